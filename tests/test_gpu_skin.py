"""Verlet skin reuse of the pair list (pfw_pair_set_skin): along a short
trajectory of small displacements the reused list gives the rebuild path's
energy, forces and virial (FP64, 1e-10 relative); a displacement beyond
skin/2, a new cell or a new atom count triggers a rebuild; the owned-atom
mask applies to the list path too."""
import numpy as np
import pytest

from pfw_b200 import lib
from pfw_b200 import workloads as WL

pytestmark = pytest.mark.gpu


def close(a, b, rtol=1e-10):
    a, b = np.asarray(a), np.asarray(b)
    return bool(np.all(np.abs(a - b) <= rtol * max(1.0, float(np.abs(b).max()))))


@pytest.mark.parametrize("kind", ["lj", "smooth"])
def test_trajectory_matches_rebuild(kind):
    s = WL.lj_fcc(seed=7, nc=8) if kind == "lj" else WL.smooth_fcc(seed=3)
    skin = 1.0 if kind == "lj" else 0.3
    hs, hr = lib.Handle(lib.FP64), lib.Handle(lib.FP64)
    for h in (hs, hr):
        if kind == "lj":
            h.lj(WL.LJ_EPS, WL.LJ_SIGMA, WL.LJ_CUTOFF)
        else:
            h.smooth(WL.SMOOTH_A, WL.SMOOTH_CUTOFF)
    hs.pair_skin(skin)
    rng = np.random.default_rng(0)
    X = s.X.copy()
    for step in range(6):
        X = X + rng.normal(0, 0.02 * skin, X.shape)
        hs.set_geometry(X, s.H, s.pbc, s.species)
        hr.set_geometry(X, s.H, s.pbc, s.species)
        Es, Fs, Ws = hs.evaluate(lib.MODEL_PAIR, 7)
        Er, Fr, Wr = hr.evaluate(lib.MODEL_PAIR, 7)
        assert abs(Es - Er) <= 1e-10 * max(1.0, abs(Er))
        assert close(Fs, Fr) and close(Ws, Wr)
        assert hs.pair_count() == hr.pair_count()
    builds, reuses = hs.skin_stats()
    assert builds == 1 and reuses == 5


def test_rebuild_triggers():
    s = WL.lj_fcc(seed=8, nc=8)
    h = lib.Handle(lib.FP64)
    h.lj(WL.LJ_EPS, WL.LJ_SIGMA, WL.LJ_CUTOFF)
    h.pair_skin(1.0)
    h.set_geometry(s.X, s.H, s.pbc, s.species)
    h.evaluate(lib.MODEL_PAIR, 7)
    X = s.X.copy()
    X[5] += [0.6, 0.0, 0.0]  # more than skin/2
    h.set_geometry(X, s.H, s.pbc, s.species)
    E1, F1, W1 = h.evaluate(lib.MODEL_PAIR, 7)
    assert h.skin_stats() == (2, 0)
    H2 = s.H * 1.001
    h.set_geometry(X, H2, s.pbc, s.species)
    h.evaluate(lib.MODEL_PAIR, 7)
    assert h.skin_stats() == (3, 0)
    h.set_geometry(X[:-1], H2, s.pbc, s.species[:-1])
    h.evaluate(lib.MODEL_PAIR, 7)
    assert h.skin_stats() == (4, 0)
    r = lib.Handle(lib.FP64)
    r.lj(WL.LJ_EPS, WL.LJ_SIGMA, WL.LJ_CUTOFF)
    r.set_geometry(X, s.H, s.pbc, s.species)
    E0, F0, W0 = r.evaluate(lib.MODEL_PAIR, 7)
    assert abs(E1 - E0) <= 1e-10 * abs(E0) and close(F1, F0)


def test_owned_mask_on_list_path():
    s = WL.lj_fcc(seed=9, nc=8)
    h = lib.Handle(lib.FP64)
    h.lj(WL.LJ_EPS, WL.LJ_SIGMA, WL.LJ_CUTOFF)
    h.pair_skin(1.0)
    h.set_geometry(s.X, s.H, s.pbc, s.species)
    E, F, W = h.evaluate(lib.MODEL_PAIR, 7)
    h.set_geometry(s.X, s.H, s.pbc, s.species)
    h.set_owned(len(s.species) // 2)
    Ea, Fa, Wa = h.evaluate(lib.MODEL_PAIR, 7)
    r = lib.Handle(lib.FP64)
    r.lj(WL.LJ_EPS, WL.LJ_SIGMA, WL.LJ_CUTOFF)
    r.set_geometry(s.X, s.H, s.pbc, s.species)
    r.set_owned(len(s.species) // 2)
    Eb, Fb, Wb = r.evaluate(lib.MODEL_PAIR, 7)
    assert h.skin_stats() == (1, 1)
    assert abs(Ea - Eb) <= 1e-10 * abs(Eb) and close(Fa, Fb) and close(Wa, Wb)
