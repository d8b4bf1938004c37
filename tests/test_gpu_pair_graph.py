"""Repeated pair evaluations of one structure replay a captured CUDA graph
of the whole device sequence (cell list, pair kernel, reductions): along a
trajectory every call must equal a fresh eager evaluation bit for bit, and a
change of model, request or structure must be picked up."""
import numpy as np
import pytest

from pfw_b200 import lib
from pfw_b200 import workloads as WL

pytestmark = pytest.mark.gpu


def fresh(s, X, model):
    r = lib.Handle(lib.FP64)
    if model == "lj":
        r.lj(WL.LJ_EPS, WL.LJ_SIGMA, WL.LJ_CUTOFF)
    else:
        r.smooth(WL.SMOOTH_A, WL.SMOOTH_CUTOFF)
    r.set_geometry(X, s.H, s.pbc, s.species)
    return r.evaluate(lib.MODEL_PAIR, 7)


def test_replays_equal_eager_along_trajectory():
    s = WL.lj_fcc(seed=11, nc=8)
    h = lib.Handle(lib.FP64)
    h.lj(WL.LJ_EPS, WL.LJ_SIGMA, WL.LJ_CUTOFF)
    rng = np.random.default_rng(1)
    X = s.X.copy()
    counts = []
    for step in range(5):
        X = X + rng.normal(0, 0.05, X.shape)
        h.set_geometry(X, s.H, s.pbc, s.species)
        l0 = h.launches
        E, F, W = h.evaluate(lib.MODEL_PAIR, 7)
        counts.append(h.launches - l0)
        E0, F0, W0 = fresh(s, X, "lj")
        assert E == E0 and np.array_equal(F, F0) and np.array_equal(W, W0)
    assert len(set(counts)) == 1  # replays launch the same kernels as the eager call


def test_model_request_and_structure_changes():
    s = WL.smooth_fcc(seed=4)
    h = lib.Handle(lib.FP64)
    h.lj(WL.LJ_EPS, WL.LJ_SIGMA, WL.LJ_CUTOFF)
    h.set_geometry(s.X, s.H, s.pbc, s.species)
    h.evaluate(lib.MODEL_PAIR, 7)
    h.evaluate(lib.MODEL_PAIR, 7)
    h.smooth(WL.SMOOTH_A, WL.SMOOTH_CUTOFF)
    E, F, W = h.evaluate(lib.MODEL_PAIR, 7)
    E0, F0, W0 = fresh(s, s.X, "smooth")
    assert E == E0 and np.array_equal(F, F0)
    E1, _, _ = h.evaluate(lib.MODEL_PAIR, 1)
    assert E1 == E0
    t = WL.smooth_fcc(seed=5)
    X2 = t.X[: len(t.X) // 2]
    h.set_geometry(X2, t.H, t.pbc, t.species[: len(X2)])
    E2, F2, _ = h.evaluate(lib.MODEL_PAIR, 7)
    r = lib.Handle(lib.FP64)
    r.smooth(WL.SMOOTH_A, WL.SMOOTH_CUTOFF)
    r.set_geometry(X2, t.H, t.pbc, t.species[: len(X2)])
    E3, F3, _ = r.evaluate(lib.MODEL_PAIR, 7)
    assert E2 == E3 and np.array_equal(F2, F3)
