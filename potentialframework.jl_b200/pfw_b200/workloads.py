"""Seeded synthetic workloads (positions in Å, cells with columns = vectors).

The reference's benchmarks generate their systems (argon FCC in
benchmark/lennard_jones/common.jl:68-83, bcc ACE workloads); these generators
produce the evaluation configurations of this library with the stated shapes,
sizes and value distributions:

  smooth_fcc   — FCC 8×8×8 (2048 atoms), a=1.6 Å, σ=0.05 Å, H/He 50/50,
                 SmoothPair([1.0 0.7; 0.7 1.3], c=2.0)
  lj_fcc       — FCC 40³ (256,000 atoms) a=5.26 Å, σ=0.1 Å; also 64³ (1,048,576)
                 and a triclinic variant (xy tilt 0.2)
  b2           — B2 (CsCl) 20³ (16,000 atoms), a=2.9 Å, σ=0.08 Å
  batched      — 4096 periodic triclinic systems, n log-uniform in [8,256]
  fixture      — the reference test fixture generator (test/fixtures.jl:17-24)
"""
from __future__ import annotations

import math
import os

import numpy as np

SMOOTH_A = np.array([[1.0, 0.7], [0.7, 1.3]])
SMOOTH_CUTOFF = 2.0
LJ_EPS, LJ_SIGMA, LJ_CUTOFF = 0.0104, 3.4, 8.5


class System:
    """Numeric system: X (n,3) Å, H (3,3) columns = cell vectors, pbc, species channels."""

    def __init__(self, X, H, pbc, species, name=""):
        self.X = np.ascontiguousarray(X, dtype=np.float64).reshape(-1, 3)
        self.H = np.asarray(H, dtype=np.float64).reshape(3, 3)
        self.pbc = tuple(bool(b) for b in pbc)
        self.species = np.ascontiguousarray(species, dtype=np.int32)
        self.name = name

    def __len__(self):
        return self.X.shape[0]


def fixture(n, L=9.0, pbc=(True, True, True), cluster=False, mixed=True):
    """test/fixtures.jl:17-24: x[a,i] = L*mod(sin(i*(a+0.71))*437.13, 1), H/He alternating (odd → He)."""
    X = np.zeros((n, 3))
    for i in range(1, n + 1):
        for a in range(1, 4):
            v = math.sin(i * (a + 0.71)) * 437.13
            r = math.fmod(v, 1.0)  # Julia mod(v, 1)
            X[i - 1, a - 1] = L * (r + 1.0 if r < 0 else r)
    if cluster:
        X[: (n + 1) // 2] *= 0.18
    H = np.diag([L, L, L])
    species = np.array([1 if (mixed and (i % 2 == 1)) else 0 for i in range(1, n + 1)], np.int32)
    return System(X, H, pbc, species, f"fixture{n}")


def _fcc(nc, a):
    basis = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]])
    g = np.stack(np.meshgrid(np.arange(nc), np.arange(nc), np.arange(nc), indexing="ij"), -1).reshape(-1, 1, 3)
    return ((g + basis[None]) * a).reshape(-1, 3)


def smooth_fcc(seed=1, nc=8, a=1.6, sigma=0.05):
    rng = np.random.default_rng(seed)
    X = _fcc(nc, a)
    n = len(X)
    species = np.zeros(n, np.int32)
    species[rng.permutation(n)[: n // 2]] = 1
    X = X + rng.normal(0.0, sigma, X.shape)
    L = nc * a
    return System(X, np.diag([L, L, L]), (True, True, True), species, f"smooth_fcc{nc}")


def lj_fcc(seed=2, nc=40, a=5.26, sigma=0.1, shear=0.0):
    rng = np.random.default_rng(seed)
    X = _fcc(nc, a)
    X = X + rng.normal(0.0, sigma, X.shape)
    L = nc * a
    H = np.array([[L, shear * L, 0.0], [0.0, L, 0.0], [0.0, 0.0, L]])
    if shear:
        X = X @ np.array([[1, 0, 0], [shear, 1, 0], [0, 0, 1.0]])  # x += shear*y
    return System(X, H, (True, True, True), np.zeros(len(X), np.int32),
                  f"lj_fcc{nc}" + (f"_shear{shear}" if shear else ""))


def lj_1m(seed=3):
    """1,048,576 atoms = 4·64³ at the 40³ box density (a=5.26 Å)."""
    return lj_fcc(seed=seed, nc=64)


def supercell(s, nr):
    """nr×nr×nr periodic copies of a system (cell vectors scaled by nr)."""
    shifts = np.array([[a, b, c] for a in range(nr) for b in range(nr) for c in range(nr)], np.float64)
    X = (s.X[None, :, :] + (shifts @ s.H.T)[:, None, :]).reshape(-1, 3)
    return System(X, s.H * nr, s.pbc, np.tile(s.species, len(shifts)), name=f"{s.name}x{nr}")


def b2(seed=4, nc=20, a=2.9, sigma=0.08):
    """B2 (CsCl): species 0 at corners, 1 at body centres."""
    rng = np.random.default_rng(seed)
    g = np.stack(np.meshgrid(np.arange(nc), np.arange(nc), np.arange(nc), indexing="ij"), -1).reshape(-1, 3)
    X = np.concatenate([g * a, (g + 0.5) * a])
    species = np.concatenate([np.zeros(len(g), np.int32), np.ones(len(g), np.int32)])
    order = np.argsort(np.concatenate([np.arange(len(g)) * 2, np.arange(len(g)) * 2 + 1]))
    X, species = X[order], species[order]
    X = X + rng.normal(0.0, sigma, X.shape)
    L = nc * a
    return System(X, np.diag([L, L, L]), (True, True, True), species, f"b2_{nc}")


def random_triclinic_cell(rng, lo=6.0, hi=14.0, amin=70.0, amax=110.0):
    """Cell with lengths U[lo,hi] Å and angles U[amin,amax]°; lower-triangular build, columns = vectors."""
    while True:
        a, b, c = rng.uniform(lo, hi, 3)
        al, be, ga = np.radians(rng.uniform(amin, amax, 3))
        v1 = np.array([a, 0.0, 0.0])
        v2 = np.array([b * math.cos(ga), b * math.sin(ga), 0.0])
        cx = c * math.cos(be)
        cy = c * (math.cos(al) - math.cos(be) * math.cos(ga)) / math.sin(ga)
        cz2 = c * c - cx * cx - cy * cy
        if cz2 <= 0.1 * c * c:
            continue
        v3 = np.array([cx, cy, math.sqrt(cz2)])
        return np.stack([v1, v2, v3], axis=1)


def _batched_system(args):
    seq, nmin, nmax, dmin, max_density, s = args
    rng = np.random.default_rng(seq)
    n = int(round(math.exp(rng.uniform(math.log(nmin), math.log(nmax)))))
    while True:
        H = random_triclinic_cell(rng)
        V = abs(np.linalg.det(H))
        if n / V <= max_density:
            break
    X = _hardcore(rng, H, n, dmin)
    species = np.zeros(n, np.int32)
    species[rng.permutation(n)[: n // 2]] = 1
    return System(X, H, (True, True, True), species, f"batch{s}")


def batched(seed=5, nsys=4096, nmin=8, nmax=256, dmin=1.6, max_density=0.11, workers=None):
    """Periodic triclinic systems (4096 by default); n log-uniform on
    [nmin, nmax]; uniform fractional positions with hard-core rejection at
    dmin; cells are redrawn until n/V <= max_density Å⁻³.  System s draws from
    its own stream (SeedSequence(seed).spawn), so the set does not depend on
    `workers` (processes, spawned; default: all cores for large batches)."""
    seqs = np.random.SeedSequence(seed).spawn(nsys)
    args = [(seqs[s], nmin, nmax, dmin, max_density, s) for s in range(nsys)]
    if workers is None:
        workers = min(os.cpu_count() or 1, 32) if nsys >= 256 else 1
    if workers <= 1:
        return [_batched_system(a) for a in args]
    import multiprocessing as mp
    with mp.get_context("spawn").Pool(workers) as pool:
        return pool.map(_batched_system, args, chunksize=max(1, nsys // (8 * workers)))


_SHIFTS = np.array([[i, j, k] for i in (-1, 0, 1) for j in (-1, 0, 1) for k in (-1, 0, 1)], dtype=np.float64)


def _min_image_d2(H, a, b):
    """Squared minimum-image distances between fractional points a (p,3) and b (m,3)."""
    df = a[:, None, :] - b[None, :, :]
    df -= np.round(df)
    d0 = df @ H.T
    Sc = _SHIFTS @ H.T
    # |d0 + S|² = |d0|² + 2 d0·S + |S|², minimised over the 27 shifts
    d2 = (d0 * d0).sum(axis=2)[:, :, None] + 2.0 * (d0 @ Sc.T) + (Sc * Sc).sum(axis=1)[None, None, :]
    return d2.min(axis=2)


def _hardcore(rng, H, n, dmin, batch=64, max_rounds=4000):
    """Random sequential adsorption in fractional coordinates: candidates are
    drawn `batch` at a time and accepted in draw order when they stay dmin
    (minimum image) from every accepted point; dmin shrinks by 10 % after
    max_rounds rounds without completing."""
    pts = np.empty((0, 3))
    rounds = 0
    while len(pts) < n:
        rounds += 1
        if rounds > max_rounds:
            dmin *= 0.9
            rounds = 0
        d2min = dmin * dmin
        cand = rng.uniform(0, 1, (batch, 3))
        if len(pts):
            cand = cand[_min_image_d2(H, cand, pts).min(axis=1) >= d2min]
        fresh = []
        for c in cand:
            if len(pts) + len(fresh) >= n:
                break
            if fresh and _min_image_d2(H, c[None], np.array(fresh)).min() < d2min:
                continue
            fresh.append(c)
        if fresh:
            pts = np.concatenate([pts, np.array(fresh)])
    return pts @ H.T
