"""Sharding of a batch of independent systems over ranks.

The reference is single-process (README.md:327); its only parallelism is
shared-memory threading.  A batch of independent structures (the training set
of design_matrix, ACE/fitting.jl:18-67) shards without any data exchange:
every rank evaluates its own systems with one batched launch, and the
per-system results are gathered once at the end.

  system_costs   expected directed edges per system, n·(n/V)·(4/3)π c³
  shard          greedy longest-processing-time bin packing of the costs
  gather_rows    all_gather of per-system result rows (padded to the largest
                 shard) back into the original system order, on any
                 torch.distributed backend (NCCL on GPUs, gloo on CPUs)

One large periodic box decomposes into slabs instead (one exchange step):

  slab_domains      slabs along the axis with the largest face height; each
                    rank's subsystem is its owned atoms followed by ghost
                    copies (periodic images included) within `halo` of the
                    slab, with the slab axis open
  evaluate_domains  every rank evaluates its subsystem with pfw_set_owned, so
                    forces of owned atoms are exact (the halo covers their
                    neighbourhood: c for pairs, 2c for ACE, whose forces
                    gather site terms of neighbours) and energies and virials
                    count only owned shares; one all-reduce of E and W and
                    one all-gather of the owned forces assemble the result
"""
from __future__ import annotations

import heapq
import math

import numpy as np


def system_costs(systems, cutoff):
    """Expected directed neighbour count of each system (uniform density)."""
    ball = 4.0 / 3.0 * math.pi * cutoff ** 3
    out = np.zeros(len(systems))
    for k, s in enumerate(systems):
        n = len(s.species)
        V = abs(float(np.linalg.det(np.asarray(s.H, np.float64).reshape(3, 3))))
        out[k] = n * (n / V) * ball if V > 0 else n * n
    return out


def shard(costs, world):
    """Greedy LPT: systems in decreasing cost (ties by index) go to the least
    loaded rank (ties by rank).  Returns one sorted index list per rank."""
    order = sorted(range(len(costs)), key=lambda k: (-float(costs[k]), k))
    heap = [(0.0, r) for r in range(world)]
    parts = [[] for _ in range(world)]
    for k in order:
        load, r = heapq.heappop(heap)
        parts[r].append(k)
        heapq.heappush(heap, (load + float(costs[k]), r))
    return [sorted(p) for p in parts]


def gather_rows(local_rows, parts, rank, group=None, device=None):
    """local_rows [len(parts[rank]), k] float64 → [nsys, k] on every rank."""
    import torch
    import torch.distributed as dist
    world = len(parts)
    k = local_rows.shape[1] if local_rows.ndim == 2 else 1
    width = max(len(p) for p in parts)
    buf = torch.zeros((width, k), dtype=torch.float64, device=device)
    if len(parts[rank]):
        buf[: len(parts[rank])] = torch.as_tensor(np.asarray(local_rows).reshape(len(parts[rank]), k), device=device)
    bufs = [torch.zeros_like(buf) for _ in range(world)]
    dist.all_gather(bufs, buf, group=group)
    nsys = sum(len(p) for p in parts)
    out = np.zeros((nsys, k))
    for r in range(world):
        rows = bufs[r].cpu().numpy()
        for i, s in enumerate(parts[r]):
            out[s] = rows[i]
    return out


class Domain:
    """One rank's subsystem: X, species (owned first), H, pbc, the owned
    atoms' original indices."""

    def __init__(self, X, species, H, pbc, owned):
        self.X, self.species, self.H, self.pbc, self.owned = X, species, H, pbc, owned

    @property
    def n_owned(self):
        return len(self.owned)


def slab_axis(H):
    """Cell axis with the largest distance between its opposite faces."""
    H = np.asarray(H, np.float64).reshape(3, 3)
    V = abs(np.linalg.det(H))
    heights = [V / np.linalg.norm(np.cross(H[:, (a + 1) % 3], H[:, (a + 2) % 3])) for a in range(3)]
    return int(np.argmax(heights)), heights


def slab_domains(system, world, halo):
    """Slab decomposition of a fully periodic system into `world` domains."""
    H = np.asarray(system.H, np.float64).reshape(3, 3)
    if not all(system.pbc):
        raise ValueError("slab decomposition needs a fully periodic box")
    a, heights = slab_axis(H)
    d = halo / heights[a]
    if d >= 1.0:
        raise ValueError("halo thicker than the box")
    f = np.linalg.solve(H, np.asarray(system.X, np.float64).T).T
    f -= np.floor(f)
    species = np.asarray(system.species, np.int32)
    pbc = [True, True, True]
    pbc[a] = False
    out = []
    for r in range(world):
        lo, hi = r / world, (r + 1) / world
        own = np.nonzero((f[:, a] >= lo) & (f[:, a] < hi))[0]
        ghosts_f, ghosts_z = [], []
        for k in (-1.0, 0.0, 1.0):
            g = f[:, a] + k
            sel = ((g >= lo - d) & (g < lo)) | ((g >= hi) & (g < hi + d))
            if np.any(sel):
                gf = f[sel].copy()
                gf[:, a] += k
                ghosts_f.append(gf)
                ghosts_z.append(species[sel])
        F = np.concatenate([f[own]] + ghosts_f) if ghosts_f else f[own]
        Z = np.concatenate([species[own]] + ghosts_z) if ghosts_z else species[own]
        out.append(Domain(np.ascontiguousarray(F @ H.T), np.ascontiguousarray(Z, np.int32), H, tuple(pbc), own))
    return out


def evaluate_domains(h, system, model, world, halo, request=7, rank=None, group=None, device=None):
    """Energy, forces (original order) and virial of `system` from its slab
    domains.  rank None: every domain in turn on this handle (one device);
    else this rank's domain, combined over `group` with one all-reduce of E
    and W and one all-gather of the owned forces."""
    doms = slab_domains(system, world, halo)
    n = len(system.species)
    mine = range(world) if rank is None else [rank]
    E, W = 0.0, np.zeros((3, 3))
    F = np.zeros((n, 3))
    rows = None
    for r in mine:
        dm = doms[r]
        h.set_geometry(dm.X, dm.H, dm.pbc, dm.species)
        h.set_owned(dm.n_owned)
        e, f, w = h.evaluate(model, request)
        E += e
        W += w
        if f is not None:
            F[dm.owned] = f[: dm.n_owned]
            rows = f[: dm.n_owned]
    if rank is None:
        return E, F, W
    import torch
    import torch.distributed as dist
    t = torch.tensor(np.concatenate([[E], W.ravel()]), dtype=torch.float64, device=device)
    dist.all_reduce(t, group=group)
    tot = t.cpu().numpy()
    parts = [list(map(int, dm.owned)) for dm in doms]
    full = gather_rows(rows if rows is not None else np.zeros((doms[rank].n_owned, 3)), parts, rank, group, device)
    return float(tot[0]), full, tot[1:].reshape(3, 3)
