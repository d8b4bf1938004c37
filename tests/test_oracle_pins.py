"""Pins the CPU oracle before it is trusted as the parity reference.

* the reference's saved 33-frame TiAl ACE oracle (data/ace_ref, via
  tests/golden/tial_ace.npz made by tests/golden/make_golden.py) at the
  tolerances of test/neighbour_saved_reference.jl:38-40;
* the analytic known answers of test/periodic_images.jl:97-104,
  test/runtests.jl:89-93,152-154 and test/neighbour_interface.jl:103-110;
* independent O(N²) brute-force sums (tests/brute.py) over the fixture
  sweeps of test/runtests.jl:66-96 and test/periodic_images.jl:61-124;
* the directed neighbour set of test/ace.jl:21-58's skew 2 Å cell at the
  5.5 Å ACE cutoff against its +-6 shell image sum.
"""
import os

import numpy as np
import pytest

from brute import image_oracle, lj_terms, smooth_terms
from oracle import oracle as O
from pfw_b200 import workloads as WL
from pfw_b200.ace_model import PackedACE

HERE = os.path.dirname(os.path.abspath(__file__))
A = WL.SMOOTH_A


def smooth(cutoff=2.0):
    return lambda zi, zj, d: smooth_terms(A, cutoff, zi, zj, d)


@pytest.fixture(scope="module")
def tial():
    d = np.load(os.path.join(HERE, "golden", "tial_ace.npz"))
    return d, PackedACE.from_npz_dict(d, "model_")


def test_tial_shapes(tial):
    # test/ace.jl:5-12: WB 123×2, Wpair 12×2, D=27, coupling 123×167
    d, m = tial
    assert m.WB.shape == (2, 123) and m.Wpair.shape == (2, 12)
    assert m.ndensity == 27 and m.nproducts == 167 and m.nbasis == 123
    assert m.cutoff == 5.5


@pytest.mark.parametrize("nthreads", [1, 4])
def test_tial_saved_oracle(tial, nthreads):
    d, m = tial
    ace = O.AceOracle(m)
    for k in range(int(d["nframes"])):
        r = ace.evaluate(d[f"f{k}_X"], d[f"f{k}_H"], (1, 1, 1), d[f"f{k}_species"], nthreads=nthreads)
        assert abs(r["energy"] - float(d[f"f{k}_energy"])) <= 1e-8
        Fref = d[f"f{k}_forces"]
        assert np.all(np.abs(r["forces"] - Fref) <= 1e-9 + 1e-10 * np.abs(Fref))
        Vref = d[f"f{k}_virial"]
        assert np.all(np.abs(r["virial"] - Vref) <= 1e-8 + 1e-10 * np.abs(Vref))


def test_kat_one_atom_chain():
    # periodic_images.jl:97-104: E = (1-(1.2/2)²)³, zero force, W11 > 0
    H = np.array([[1.2, 0, 0], [0, 0, 0], [0, 0, 0.0]])
    E, F, W, npairs = O.pair_evaluate(np.zeros((1, 3)), H, (1, 0, 0), [0], "smooth", A, 2.0)
    assert E == pytest.approx((1 - (1.2 / 2) ** 2) ** 3, rel=1e-14)
    assert np.all(F == 0)
    assert W[0, 0] > 0
    Eb, Fb, Wb, _ = image_oracle(np.zeros((1, 3)), H, (1, 0, 0), [0], smooth(), 2.0)
    assert E == pytest.approx(Eb, abs=1e-12) and np.allclose(W, Wb, atol=1e-12)


def test_kat_nm_pair():
    # runtests.jl:89-93: H at 0, He at 0.1 nm, 1 nm cell, pbc (T,F,T)
    X = np.array([[0, 0, 0], [1.0, 0, 0]])
    E, F, W, _ = O.pair_evaluate(X, np.diag([10.0, 10, 10]), (1, 0, 1), [0, 1], "smooth", A, 2.0, width=1)
    assert E == pytest.approx(0.7 * (1 - 1 / 4) ** 3, rel=1e-14)
    E2, *_ = O.pair_evaluate(X, np.zeros((3, 3)), (0, 0, 0), [0, 0], "smooth", np.ones((1, 1)), 2.0)
    assert E2 == pytest.approx((1 - 1 / 4) ** 3, rel=1e-14)


def test_kat_edge_and_coincident():
    # runtests.jl:147-154: r == c contributes nothing; coincident atoms give E = A = 1
    X = np.array([[0, 0, 0], [2.0, 0, 0]])
    H = np.diag([10.0, 10, 10])
    E, F, *_ = O.pair_evaluate(X, H, (0, 0, 0), [0, 0], "smooth", A, 2.0)
    assert E == 0 and np.all(F == 0)
    X[1] = X[0]
    E, F, *_ = O.pair_evaluate(X, H, (0, 0, 0), [0, 0], "smooth", A, 2.0)
    assert E == 1.0 and np.all(F == 0)


def test_kat_self_images_snapshot():
    # neighbour_interface.jl:103-110
    H = np.array([[1.2, 0, 0], [0, 0, 0], [0, 0, np.inf]])
    offs, j, S, R = O.neighbour_list(np.zeros((1, 3)), H, (1, 0, 0), 2.0)
    assert list(j) == [0, 0]
    assert {tuple(s) for s in S} == {(1, 0, 0), (-1, 0, 0)}
    assert sorted(R[:, 0]) == pytest.approx([-1.2, 1.2])
    assert np.all(R[:, 1:] == 0)


def _agrees(E, F, W, Eb, Fb, Wb, tol):
    assert E == pytest.approx(Eb, abs=tol, rel=tol)
    assert np.allclose(F, Fb, atol=tol, rtol=tol)
    assert np.allclose(W, Wb, atol=tol, rtol=tol)


@pytest.mark.parametrize("n", [0, 1, 2, 7, 31, 93])
@pytest.mark.parametrize("pbc", [(1, 1, 1), (1, 0, 1), (0, 0, 0)])
@pytest.mark.parametrize("cluster", [False, True])
def test_pairs_vs_bruteforce(n, pbc, cluster):
    # runtests.jl:66-96 sweep, 1e-11 agreement (runtests.jl:21-27)
    s = WL.fixture(n, pbc=pbc, cluster=cluster)
    for thr in (0, 32):
        E, F, W, npairs = O.pair_evaluate(s.X, s.H, pbc, s.species, "smooth", A, 2.0, brute_threshold=thr)
        Eb, Fb, Wb, pairs = image_oracle(s.X, s.H, pbc, s.species, smooth(), 2.0, shell=1)
        _agrees(E, F, W, Eb, Fb, Wb, 1e-11)
        assert npairs * 2 == len(pairs)


@pytest.mark.parametrize("n", [0, 1, 3, 35])
def test_skew_images_vs_bruteforce(n):
    # periodic_images.jl:116-121: skew cell smaller than the cutoff sphere
    H = np.array([[1.2, 0.4, 0.0], [0, 1.3, 0.3], [0, 0, 1.1]])
    f = np.array([[np.sin((i + 1) * (a + 1)) * 17.3 % 1.0 for a in range(3)] for i in range(n)]).reshape(n, 3)
    X = f @ H.T
    sp = np.zeros(n, np.int32)
    for thr in (0, 32):
        E, F, W, npairs = O.pair_evaluate(X, H, (1, 1, 1), sp, "smooth", A, 2.0, brute_threshold=thr)
        Eb, Fb, Wb, pairs = image_oracle(X, H, (1, 1, 1), sp, smooth(), 2.0, shell=4)
        _agrees(E, F, W, Eb, Fb, Wb, 1e-9)
        offs, j, S, R = O.neighbour_list(X, H, (1, 1, 1), 2.0, brute_threshold=thr)
        got = {(i, int(j[k]), tuple(int(v) for v in S[k])) for i in range(n) for k in range(offs[i], offs[i + 1])}
        assert got == pairs


def test_lj_vs_bruteforce():
    s = WL.lj_fcc(nc=3)
    E, F, W, _ = O.pair_evaluate(s.X, s.H, s.pbc, s.species, "lj", (WL.LJ_EPS, WL.LJ_SIGMA), WL.LJ_CUTOFF)
    # 3 cells of 5.26 Å < 2c: the oracle takes the explicit-image path
    Eb, Fb, Wb, _ = image_oracle(s.X, s.H, s.pbc, s.species,
                                 lambda zi, zj, d: lj_terms(WL.LJ_EPS, WL.LJ_SIGMA, WL.LJ_CUTOFF, d),
                                 WL.LJ_CUTOFF, shell=2)
    _agrees(E, F, W, Eb, Fb, Wb, 1e-10)


def test_snapshot_min_image_vs_bruteforce():
    s = WL.fixture(93)
    offs, j, S, R = O.neighbour_list(s.X, s.H, s.pbc, 2.0)
    _, _, _, pairs = image_oracle(s.X, s.H, s.pbc, s.species, smooth(), 2.0, shell=1)
    got = {(i, int(j[k]), tuple(int(v) for v in S[k])) for i in range(len(s)) for k in range(offs[i], offs[i + 1])}
    assert got == pairs
    # R == X[j] - X[i] + H·S  (neighbour_interface.jl:40-49)
    for i in range(len(s)):
        for k in range(offs[i], offs[i + 1]):
            assert np.allclose(R[k], s.X[j[k]] - s.X[i] + s.H @ S[k], atol=1e-12)


@pytest.mark.parametrize("pbc", [(1, 1, 1), (1, 0, 1), (0, 0, 0)])
@pytest.mark.parametrize("n", [3, 1, 0, 2])
def test_ace_environment_set_skew_cell(pbc, n):
    # test/ace.jl:21-58: a skew cell of about 2 Å against the 5.5 Å ACE cutoff,
    # the first atom placed two cell vectors outside the cell; the directed
    # (i, j, S) set equals the +-6 shell image sum
    H = np.array([[2.1, 0.6, 0.2], [0, 2.2, 0.4], [0, 0, 2.0]])
    frac = np.array([[0.1, 0.4, 0.8], [0.2, 0.6, 0.3], [0.1, 0.7, 0.5]])[:, :n]
    X = (H @ frac).T.copy()
    if n > 0:
        X[0] += 2 * H[:, 0]
    sp = np.array([0, 1, 0][:n], np.int32)
    offs, j, S, R = O.neighbour_list(X, H, pbc, 5.5)
    _, _, _, pairs = image_oracle(X, H, pbc, sp, smooth(), 5.5, shell=6)
    got = {(i, int(j[k]), tuple(int(v) for v in S[k])) for i in range(n) for k in range(offs[i], offs[i + 1])}
    assert got == pairs
    for i in range(n):
        for k in range(offs[i], offs[i + 1]):
            assert np.allclose(R[k], X[j[k]] - X[i] + H @ S[k], atol=1e-12)
