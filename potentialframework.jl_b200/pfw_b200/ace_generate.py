"""Synthetic resolved-ACE models in the schema-v1 TOML format.

The invariant basis is generated by restating the reference's construction-
time Clebsch–Gordan algebra (ACE/feature_coupling.jl:24-143):

  real_harmonic_map   Condon–Shortley complex Y → real L2 Y       (:24-33)
  complex_cg          Racah formula, exact rational arithmetic    (:34-46)
  real_cg             real coupling tensor C[r,s,t]               (:47-60)
  couple / independent multiplets, Gram–Schmidt on complete
  multiplets, products sorted by (order, key)                     (:62-143)

with one species channel in the density (species enter through the radial
channels of each species pair) and the single irrep (L=0, even).  Radial and
pair spline channels are cubic Hermite interpolants of smooth seeded
functions on 100 uniform nodes, with the Agnesi transform and envelopes of
the reference's TiAl export.  Readout WB ~ N(0, (s/(1+deg))²) where deg is
the invariant's largest Σ(n+l) over its coupled products (the rule of
ACE/fitting.jl:76-80 smoothness_prior).
"""
from __future__ import annotations

import cmath
import hashlib
import math
from fractions import Fraction

import numpy as np


# ---- Clebsch–Gordan -------------------------------------------------------
def real_harmonic_map(l):
    U = np.zeros((2 * l + 1, 2 * l + 1), dtype=complex)
    U[l, l] = 1
    s = 1 / math.sqrt(2)
    for m in range(1, l + 1):
        U[l + m, l + m] = (-1) ** m * s
        U[l + m, l - m] = s
        U[l - m, l + m] = -1j * (-1) ** m * s
        U[l - m, l - m] = 1j * s
    return U


def complex_cg(a, m, b, n, L, M):
    if m + n != M or not (abs(a - b) <= L <= a + b):
        return 0.0
    f = math.factorial
    pref2 = Fraction((2 * L + 1) * f(L + a - b) * f(L - a + b) * f(a + b - L), f(a + b + L + 1))
    pref2 *= f(L + M) * f(L - M) * f(a - m) * f(a + m) * f(b - n) * f(b + n)
    lo, hi = max(0, b - L - m, a + n - L), min(a + b - L, a - m, b + n)
    total = Fraction(0)
    for k in range(lo, hi + 1):
        total += Fraction((-1) ** k, f(k) * f(a + b - L - k) * f(a - m - k) * f(b + n - k) * f(L - b + m + k)
                          * f(L - a - n + k))
    # sqrt of an exact rational, then the exact sum
    return math.sqrt(pref2.numerator) / math.sqrt(pref2.denominator) * float(total)


_real_cg_cache = {}


def real_cg(a, b, L):
    key = (a, b, L)
    if key in _real_cg_cache:
        return _real_cg_cache[key]
    Ua, Ub, U = real_harmonic_map(a), real_harmonic_map(b), real_harmonic_map(L)
    C = np.zeros((2 * L + 1, 2 * a + 1, 2 * b + 1), dtype=complex)
    for m in range(-a, a + 1):
        for n in range(-b, b + 1):
            M = m + n
            if abs(M) > L:
                continue
            c = complex_cg(a, m, b, n, L, M) * (1j ** (a + b - L))
            if c == 0:
                continue
            C += U[:, L + M][:, None, None] * c * np.conj(Ua[:, a + m])[None, :, None] * np.conj(Ub[:, b + n])[None, None, :]
    if np.max(np.abs(C.imag)) >= 1e-12:
        raise RuntimeError("nonreal harmonic coupling")
    R = C.real.copy()
    R[np.abs(R) < 1e-14] = 0
    _real_cg_cache[key] = R
    return R


# ---- polynomial multiplets (dict: sorted key tuple -> coefficient) ---------
def _axpy(a, x, y):
    for k in sorted(x):
        y[k] = y.get(k, 0.0) + a * x[k]


def _mdot(x, y):
    s = 0.0
    for m in range(len(x)):
        ym = y[m]
        s += sum(v * ym.get(k, 0.0) for k, v in sorted(x[m].items()))
    return s / len(x)


def _independent(basis, x):
    for _ in range(2):
        for y in basis:
            c = _mdot(x, y)
            for m in range(len(x)):
                _axpy(-c, y[m], x[m])
    scale = math.sqrt(max(0.0, _mdot(x, x)))
    if not scale > 1e-10:
        return False
    for p in x:
        for k in list(p):
            v = p[k] / scale
            if abs(v) < 1e-13:
                del p[k]
            else:
                p[k] = v
    basis.append(x)
    return True


def _couple(x, y, C):
    out = [dict() for _ in range(C.shape[0])]
    nz = np.argwhere(C != 0)
    for r, s, t in nz:
        c = C[r, s, t]
        for i, v in sorted(x[s].items()):
            for j, w in sorted(y[t].items()):
                key = tuple(sorted(i + j))
                out[r][key] = out[r].get(key, 0.0) + c * v * w
    return out


def generate_feature_tables(rspec, correlation, lmax, totaldegree, irrep_L=0, irrep_parity=1):
    """Invariant (irrep) basis over density factors (r, l) with weight n+l.
    Returns (density [(r, lm)] 0-based, products [tuple of density idx], coupling rows)."""
    density, factors, vectors = [], [], []
    for r, (n, l) in enumerate(rspec):
        if not (0 <= l <= lmax):
            continue
        factors.append((r, l, n + l))
        idx = []
        for m in range(-l, l + 1):
            density.append((r, l * l + l + m))
            idx.append(len(density) - 1)
        vectors.append([{(i,): 1.0} for i in idx])
    block = []

    def visit(first, degree, order, parity, states):
        if order >= correlation:
            return
        for f in range(first, len(factors)):
            _, l, weight = factors[f]
            if degree + weight > totaldegree:
                continue
            nxt = {}
            for J in sorted(states):
                for x in states[J]:
                    for L in range(abs(J - l), J + l + 1):
                        y = _couple(x, vectors[f], real_cg(J, l, L))
                        _independent(nxt.setdefault(L, []), y)
            p = parity * (-1) ** l
            if p == irrep_parity:
                block.extend(nxt.get(irrep_L, []))
            visit(f, degree + weight, order + 1, p, nxt)

    visit(0, 0, 0, 1, {0: [[{(): 1.0}]]})
    if not block:
        raise ValueError("no invariants survive")
    keys = set()
    for x in block:
        for p in x:
            keys.update(p.keys())
    products = sorted(keys, key=lambda k: (len(k), k))
    lookup = {p: i for i, p in enumerate(products)}
    dim = 2 * irrep_L + 1
    rows, cols, vals = [], [], []
    for i, x in enumerate(block):
        for m in range(dim):
            for k, v in sorted(x[m].items()):
                rows.append(i * dim + m)
                cols.append(lookup[k])
                vals.append(v)
    return density, products, (rows, cols, vals, (dim * len(block), len(products)))


# ---- radial channels --------------------------------------------------------
def _agnesi_y(r, a, p, q, rin, r0):
    s = (r - rin) / (r0 - rin)
    return 1.0 if r <= rin else 1.0 / (1.0 + a * s ** q / (1.0 + s ** (q - p)))


def _hermite_coefficients(f, df, nodes):
    """Cubic Hermite coefficients [power][interval] in u ∈ [0,1] per interval."""
    K = len(nodes)
    c = np.zeros((4, K - 1))
    for k in range(K - 1):
        h = nodes[k + 1] - nodes[k]
        f0, f1 = f(nodes[k]), f(nodes[k + 1])
        d0, d1 = df(nodes[k]) * h, df(nodes[k + 1]) * h
        c[:, k] = [f0, d0, 3 * (f1 - f0) - 2 * d0 - d1, 2 * (f0 - f1) + d0 + d1]
    return c


def _channel(rng, spec, transform, env_kind, env, iz, jz, nknots=100, pair=False):
    nodes = np.linspace(-1.0, 1.0, nknots)
    nodes[0], nodes[-1] = -1.0, 1.0
    coeff = np.zeros((4, len(spec), nknots - 1))
    for ch, (n, l) in enumerate(spec):
        amp = 1.0 + 0.15 * (iz + jz) + 0.05 * rng.standard_normal()
        ph = 0.1 * rng.standard_normal()
        k = n - 1 + 0.5 * l

        def f(x, k=k, amp=amp, ph=ph):
            return amp * math.cos(k * math.acos(max(-1.0, min(1.0, x))) + ph * (1 - x * x))

        def df(x, f=f):
            h = 1e-6
            return (f(min(1.0, x + h)) - f(max(-1.0, x - h))) / (min(1.0, x + h) - max(-1.0, x - h))

        coeff[:, ch, :] = _hermite_coefficients(f, df, nodes)
    return {
        "centre": iz + 1, "neighbour": jz + 1, "transform": transform, "envelope_kind": env_kind,
        "envelope": env, "nodes": [float(v) for v in nodes], "coefficient_shape": [4, len(spec), nknots - 1],
        "coefficients": [float(v) for v in coeff.reshape(-1, order="F")],
    }


def generate_b2_model(seed=11, atomic_numbers=(22, 13), nmax=8, lmax=4, correlation=3, totaldegree=12, nq=8,
                      rcut=5.5, r0=2.9, wb_scale=0.05):
    """The C3 model: 2 species, radial spec {(n,l): n ≤ nmax, l ≤ lmax}, lmax 4,
    correlation order 3, total degree 12 in Σ(n+l), cutoff 5.5 Å."""
    rng = np.random.default_rng(seed)
    nz = len(atomic_numbers)
    rspec = [(n, l) for l in range(lmax + 1) for n in range(1, nmax + 1)]
    density, products, (rows, cols, vals, shape) = generate_feature_tables(rspec, correlation, lmax, totaldegree)
    # transforms (as the TiAl export): radial p=2,q=4; pair p=1,q=3
    def transform(a, p, q):
        ycut = _agnesi_y(rcut, a, p, q, 0.0, r0)
        return {"a": a, "normalization_rin": 0.0, "p": p, "q": q, "r0": r0, "rcut": rcut, "rin": 0.0,
                "ycut": ycut, "yin": 1.0}
    tr_r, tr_q = transform(0.7692307692307693, 2, 4), transform(0.2857142857142857, 1, 3)
    env_r = {"p1": 2, "p2": 2, "s": 1.0, "x1": -1.0, "x2": 1.0}
    env_q = {"p": 2, "r0": r0, "rcut": rcut}
    qspec = [(n, 0) for n in range(1, nq + 1)]
    radial = {"kind": "piecewise_cubic_agnesi", "spec": [{"n": n, "l": l} for n, l in rspec],
              "channels": [_channel(rng, rspec, tr_r, "PolyEnvelope2sX", env_r, i, j) for i in range(nz) for j in range(nz)]}
    pair = {"kind": "piecewise_cubic_agnesi", "spec": [{"n": n, "l": l} for n, l in qspec],
            "channels": [_channel(rng, qspec, tr_q, "ACE1_PolyEnvelope1sR", env_q, i, j, pair=True)
                         for i in range(nz) for j in range(nz)]}
    nB, P = shape
    # smoothness-prior degree per invariant
    weights = [rspec[r][0] + rspec[r][1] for r, _ in density]
    pdeg = [sum(weights[a] for a in prod) for prod in products]
    deg = np.ones(nB)
    for r_, c_ in zip(rows, cols):
        deg[r_] = max(deg[r_], 1 + pdeg[c_])
    WB = np.zeros((nB, nz))
    for z in range(nz):
        WB[:, z] = rng.standard_normal(nB) * wb_scale / (1.0 + deg)
    Wpair = np.zeros((nq, nz))
    for z in range(nz):
        Wpair[:, z] = rng.standard_normal(nq) * 0.2 / (1.0 + np.arange(1, nq + 1))
    D = {
        "schema": "PotentialFrameWork.resolved_ACE", "schema_version": 1,
        "species_atomic_numbers": list(atomic_numbers), "reference_eV": [-1.5, -0.75],
        "angular": {"kind": "real_spherical", "lmax": lmax, "normalization": "L2", "ordering": "l*l+l+m+1"},
        "radial": radial, "pair_radial": pair,
        "density_indices": [[r + 1, m + 1] for r, m in density],
        "products": [[a + 1 for a in p] for p in products],
        "coupling": {"shape": [nB, P], "rows": [r + 1 for r in rows], "columns": [c + 1 for c in cols],
                     "values": [float(v) for v in vals]},
        "parameters": {"ordering": "vec(WB), vec(Wpair); Julia column-major", "WB_shape": [nB, nz],
                       "Wpair_shape": [nq, nz],
                       "flat": [float(v) for v in np.concatenate([WB.reshape(-1, order="F"),
                                                                 Wpair.reshape(-1, order="F")])]},
    }
    D["source_sha256"] = hashlib.sha256(repr((seed, rspec, correlation, totaldegree)).encode()).hexdigest()
    return D


# ---- minimal TOML writer for the resolved schema ----------------------------
def _fmt(v):
    if isinstance(v, bool):
        return "true" if v else "false"
    if isinstance(v, (int, np.integer)):
        return str(int(v))
    if isinstance(v, (float, np.floating)):
        return repr(float(v))
    if isinstance(v, str):
        return '"' + v.replace("\\", "\\\\").replace('"', '\\"') + '"'
    if isinstance(v, (list, tuple)):
        return "[" + ", ".join(_fmt(x) for x in v) + "]"
    raise TypeError(type(v))


def _emit(lines, table, prefix):
    scalars = {k: v for k, v in table.items() if not isinstance(v, dict) and not _is_table_list(v)}
    for k, v in scalars.items():
        lines.append(f"{k} = {_fmt(v)}")
    for k, v in table.items():
        if isinstance(v, dict):
            lines.append("")
            lines.append(f"[{prefix}{k}]")
            _emit(lines, v, f"{prefix}{k}.")
    for k, v in table.items():
        if _is_table_list(v):
            for item in v:
                lines.append("")
                lines.append(f"[[{prefix}{k}]]")
                _emit(lines, item, f"{prefix}{k}.")


def _is_table_list(v):
    return isinstance(v, list) and v and all(isinstance(x, dict) for x in v)


def dumps_toml(D):
    lines = []
    _emit(lines, D, "")
    return "\n".join(lines) + "\n"


def write_resolved(path, D):
    with open(path, "w") as f:
        f.write(dumps_toml(D))
