"""Independent O(N²) brute-force oracles (numpy), restating the reference's
test oracles: the minimum-image oracle of test/fixtures.jl:28-51 and the fixed
±shell image sum of test/periodic_images.jl:5-28.  They share no code with
the cell-list restatement in oracle/."""
import itertools

import numpy as np


def smooth_terms(A, c, zi, zj, d):
    a = A[zi, zj]
    r2 = np.sum(d * d, axis=-1)
    q = 1 - r2 / c ** 2
    e = a * q ** 3
    g = (-6 * a * q ** 2 / c ** 2)[..., None] * d
    return e, g


def lj_terms(eps, sigma, c, d):
    r2 = np.sum(d * d, axis=-1)
    s6 = (sigma ** 2 / r2) ** 3
    sc6 = (sigma / c) ** 6
    e = 4 * eps * (s6 * s6 - s6 - sc6 * sc6 + sc6)
    g = (24 * eps * (s6 - 2 * s6 * s6) / r2)[..., None] * d
    return e, g


def image_oracle(X, H, pbc, species, terms, cutoff, shell=10):
    """Exhaustive image sum over a fixed lattice cube; returns E, F (n,3), W,
    and the set of directed (i, j, S) with S the integer shift."""
    n = len(X)
    F = np.zeros((n, 3)); W = np.zeros((3, 3)); E = 0.0
    rng = [range(-shell, shell + 1) if p else range(0, 1) for p in pbc]
    shifts = np.array(list(itertools.product(*rng)), dtype=np.float64)
    Hp = H * np.array([1.0 if p else 0.0 for p in pbc])[None, :]
    sv = shifts @ Hp.T
    pairs = set()
    for i in range(n):
        for j in range(i, n):
            d = X[j] - X[i] + sv
            r2 = np.sum(d * d, axis=1)
            mask = r2 < cutoff * cutoff
            if i == j:
                pos = np.array([tuple(s) > (0, 0, 0) for s in shifts])
                mask &= pos
            idx = np.nonzero(mask)[0]
            if len(idx) == 0:
                continue
            dd = d[idx]
            e, g = terms(species[i], species[j], dd)
            E += float(np.sum(e))
            F[i] += g.sum(0); F[j] -= g.sum(0)
            W -= dd.T @ g
            for k in idx:
                s = tuple(int(v) for v in shifts[k])
                pairs.add((i, j, s)); pairs.add((j, i, tuple(-v for v in s)))
    return E, F, W, pairs
