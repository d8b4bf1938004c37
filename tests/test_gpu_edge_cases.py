"""Edge cases of the boundary on the GPU: empty systems (alone and inside a
batch), a one-system batch, and the argument errors the reference raises
(nonfinite positions, species without parameters, nonpositive cutoffs;
storage.jl:89-93,134 → ArgumentError)."""
import numpy as np
import pytest

from oracle import oracle as O
from pfw_b200 import lib
from pfw_b200 import workloads as WL
from pfw_b200.ace_model import PackedACE

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def tial():
    import os
    d = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "tial_ace.npz"))
    return PackedACE.from_npz_dict(d, "model_")


def test_empty_system_pairs_ace_snapshot(tial):
    H = np.diag([10.0, 10.0, 10.0])
    X = np.zeros((0, 3))
    z = np.zeros(0, np.int32)
    h = lib.Handle(lib.FP64)
    h.smooth(WL.SMOOTH_A, 2.0)
    h.set_geometry(X, H, (1, 1, 1), z)
    E, F, W = h.evaluate(lib.MODEL_PAIR, 7)
    assert E == 0.0 and F.shape == (0, 3) and not W.any()
    offs, j, S, R = h.neighbour_list(2.0)
    assert offs.tolist() == [0] and len(j) == 0
    h.ace(tial)
    E, F, W = h.evaluate(lib.MODEL_ACE, 7)
    assert E == 0.0 and F.shape == (0, 3) and not W.any()


def test_batch_with_empty_system(tial):
    systems = WL.batched(seed=12, nsys=3, nmin=8, nmax=40, workers=1)
    empty = WL.System(np.zeros((0, 3)), np.diag([9.0, 9.0, 9.0]), (1, 1, 1), np.zeros(0, np.int32))
    batch = [systems[0], empty, systems[1], systems[2]]
    h = lib.Handle(lib.FP64)
    h.ace(tial)
    h.set_batch(batch)
    E, F, Wv, X = h.evaluate_batch(lib.MODEL_ACE, 7, features=True)
    assert E[1] == 0.0 and not Wv[1].any() and not X[1].any()
    ace = O.AceOracle(tial)
    offs = h.batch_offsets
    for k in (0, 2, 3):
        s = batch[k]
        r = ace.evaluate(s.X, s.H, s.pbc, s.species)
        assert abs(E[k] - r["energy"]) <= 1e-10 * max(1.0, abs(r["energy"]))
        assert np.allclose(F[offs[k]:offs[k + 1]], r["forces"], rtol=0, atol=1e-10 * max(1.0, np.abs(r["forces"]).max()))
    h.smooth(WL.SMOOTH_A, 2.0)
    Ep, _, _, _ = h.evaluate_batch(lib.MODEL_PAIR, 7)
    assert Ep[1] == 0.0


def test_single_system_batch_equals_evaluate(tial):
    s = WL.batched(seed=13, nsys=1, nmin=40, nmax=60, workers=1)[0]
    h = lib.Handle(lib.FP64)
    h.ace(tial)
    h.set_batch([s])
    Eb, Fb, Wb, _ = h.evaluate_batch(lib.MODEL_ACE, 7)
    h.set_geometry(s.X, s.H, s.pbc, s.species)
    E, F, W = h.evaluate(lib.MODEL_ACE, 7)
    assert abs(Eb[0] - E) <= 1e-12 * abs(E)
    assert np.allclose(Fb, F, rtol=0, atol=1e-12 * max(1.0, np.abs(F).max()))
    assert np.allclose(Wb[0], W, rtol=0, atol=1e-12 * max(1.0, np.abs(W).max()))


def test_argument_errors():
    h = lib.Handle(lib.FP64)
    h.smooth(WL.SMOOTH_A, 2.0)
    X = np.array([[0.0, 0.0, 0.0], [1.0, np.nan, 0.0]])
    h.set_geometry(X, np.diag([10.0, 10.0, 10.0]), (1, 1, 1), [0, 1])
    with pytest.raises(lib.ArgumentError):
        h.evaluate(lib.MODEL_PAIR, 7)
    X = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0]])
    h.set_geometry(X, np.diag([10.0, 10.0, 10.0]), (1, 1, 1), [0, 5])  # no amplitudes for channel 5
    with pytest.raises(lib.ArgumentError):
        h.evaluate(lib.MODEL_PAIR, 7)
    with pytest.raises(lib.ArgumentError):
        h.smooth(WL.SMOOTH_A, 0.0)
    with pytest.raises(lib.ArgumentError):
        h.neighbour_list(-1.0)
    # the workspace stays usable after errors
    h.set_geometry(X, np.diag([10.0, 10.0, 10.0]), (1, 1, 1), [0, 1])
    E, F, W = h.evaluate(lib.MODEL_PAIR, 7)
    assert np.isfinite(E)
