"""GPU parity of the pair path and the neighbour snapshot against the oracle.

Bars: the directed neighbour set {(i, j, S)} bit-exact (and R bit-exact, the
same arithmetic); FP64 energy/forces/virial within 1e-10 relative (forces
with a 1e-12 eV/Å absolute floor); mixed FP32 form within the stated force
RMSE (≤1e-3 eV/Å).  Sizes follow test/runtests.jl:66-96 and
test/periodic_images.jl:61-124 plus the 2048-atom SmoothPair FCC workload.
"""
import numpy as np
import pytest

from oracle import oracle as O
from pfw_b200 import lib
from pfw_b200 import workloads as WL

pytestmark = pytest.mark.gpu
A = WL.SMOOTH_A
RTOL = 1e-10


@pytest.fixture(scope="module")
def h64():
    return lib.Handle(lib.FP64)


@pytest.fixture(scope="module")
def h32():
    return lib.Handle(lib.MIXED)


def gpu_pair(h, s, kind, params, cutoff, request=7):
    h.set_geometry(s.X, s.H, s.pbc, s.species)
    if kind == "smooth":
        h.smooth(params, cutoff)
    else:
        h.lj(params[0], params[1], cutoff)
    return h.evaluate(lib.MODEL_PAIR, request)


def assert_close(E, F, W, Eo, Fo, Wo, rtol=RTOL, atol=1e-12):
    scale = max(1.0, abs(Eo))
    assert abs(E - Eo) <= rtol * scale, (E, Eo)
    fs = max(1e-300, np.abs(Fo).max()) if Fo.size else 1.0
    assert np.all(np.abs(F - Fo) <= rtol * fs + atol), np.abs(F - Fo).max()
    ws = max(1.0, np.abs(Wo).max())
    assert np.all(np.abs(W - Wo) <= rtol * ws), np.abs(W - Wo).max()


def snapshot_set(offs, j, S):
    return {(i, int(j[k]), tuple(int(v) for v in S[k])) for i in range(len(offs) - 1) for k in range(offs[i], offs[i + 1])}


def test_smooth_fcc_2048(h64):
    s = WL.smooth_fcc()
    E, F, W = gpu_pair(h64, s, "smooth", A, 2.0)
    Eo, Fo, Wo, npairs = O.pair_evaluate(s.X, s.H, s.pbc, s.species, "smooth", A, 2.0)
    assert_close(E, F, W, Eo, Fo, Wo)
    assert h64.pair_count() == npairs


def test_smooth_fcc_snapshot_bit_exact(h64):
    s = WL.smooth_fcc()
    h64.set_geometry(s.X, s.H, s.pbc, s.species)
    offs, j, S, R = h64.neighbour_list(2.0)
    oo, jo, So, Ro = O.neighbour_list(s.X, s.H, s.pbc, 2.0)
    assert np.array_equal(offs, oo)
    assert snapshot_set(offs, j, S) == snapshot_set(oo, jo, So)
    # R is produced by the same arithmetic: compare per (i, j, S) key, bit for bit
    gr = {(i, int(j[k]), tuple(S[k])): tuple(R[k]) for i in range(len(s)) for k in range(offs[i], offs[i + 1])}
    orr = {(i, int(jo[k]), tuple(So[k])): tuple(Ro[k]) for i in range(len(s)) for k in range(oo[i], oo[i + 1])}
    assert gr == orr


@pytest.mark.parametrize("n", [0, 1, 2, 7, 31, 93])
@pytest.mark.parametrize("pbc", [(1, 1, 1), (1, 0, 1), (0, 0, 0)])
@pytest.mark.parametrize("cluster", [False, True])
@pytest.mark.parametrize("thr", [0, 32])
def test_fixture_sweep(n, pbc, cluster, thr):
    h = lib.Handle(lib.FP64, bruteforce_threshold=thr)
    s = WL.fixture(n, pbc=pbc, cluster=cluster)
    E, F, W = gpu_pair(h, s, "smooth", A, 2.0)
    Eo, Fo, Wo, npairs = O.pair_evaluate(s.X, s.H, pbc, s.species, "smooth", A, 2.0, brute_threshold=thr)
    assert_close(E, F, W, Eo, Fo, Wo)
    offs, j, S, R = h.neighbour_list(2.0)
    oo, jo, So, Ro = O.neighbour_list(s.X, s.H, pbc, 2.0, brute_threshold=thr)
    assert snapshot_set(offs, j, S) == snapshot_set(oo, jo, So)


@pytest.mark.parametrize("n", [1, 3, 35, 200])
@pytest.mark.parametrize("thr", [0, 32])
def test_skew_cells(n, thr):
    # periodic_images.jl:116-121: skew cell smaller than the cutoff sphere
    h = lib.Handle(lib.FP64, bruteforce_threshold=thr)
    H = np.array([[1.2, 0.4, 0.0], [0, 1.3, 0.3], [0, 0, 1.1]])
    f = np.array([[np.sin((i + 1) * (a + 1)) * 17.3 % 1.0 for a in range(3)] for i in range(n)])
    s = WL.System(f @ H.T, H, (1, 1, 1), np.zeros(n, np.int32))
    E, F, W = gpu_pair(h, s, "smooth", A, 2.0)
    Eo, Fo, Wo, _ = O.pair_evaluate(s.X, H, s.pbc, s.species, "smooth", A, 2.0, brute_threshold=thr)
    assert_close(E, F, W, Eo, Fo, Wo)
    offs, j, S, R = h.neighbour_list(2.0)
    oo, jo, So, Ro = O.neighbour_list(s.X, H, s.pbc, 2.0, brute_threshold=thr)
    assert snapshot_set(offs, j, S) == snapshot_set(oo, jo, So)


def test_one_atom_chain_and_slab(h64):
    # periodic_images.jl:97-108
    s = WL.System(np.zeros((1, 3)), np.array([[1.2, 0, 0], [0, 0, 0], [0, 0, 0.0]]), (1, 0, 0), [0])
    E, F, W = gpu_pair(h64, s, "smooth", A, 2.0)
    assert E == pytest.approx((1 - (1.2 / 2) ** 2) ** 3, rel=1e-14)
    assert np.all(F == 0) and W[0, 0] > 0
    H = np.array([[3.0, 1.0, 0], [0, 2.5, 0], [0, 0, np.inf]])
    s = WL.System(np.array([[0.0, 0, 0], [0.5, 0.2, 0.8]]), H, (1, 1, 0), [0, 1])
    E, F, W = gpu_pair(h64, s, "smooth", A, 2.0)
    Eo, Fo, Wo, _ = O.pair_evaluate(s.X, H, s.pbc, s.species, "smooth", A, 2.0)
    assert_close(E, F, W, Eo, Fo, Wo)


def test_kats(h64):
    X = np.array([[0, 0, 0], [1.0, 0, 0]])
    s = WL.System(X, np.diag([10.0, 10, 10]), (1, 0, 1), [0, 1])
    E, _, _ = gpu_pair(h64, s, "smooth", A, 2.0)
    assert E == pytest.approx(0.7 * (1 - 1 / 4) ** 3, rel=1e-14)
    s = WL.System(np.array([[0, 0, 0], [2.0, 0, 0]]), np.diag([10.0, 10, 10]), (0, 0, 0), [0, 0])
    E, F, _ = gpu_pair(h64, s, "smooth", A, 2.0)
    assert E == 0 and np.all(F == 0)
    s.X[1] = s.X[0]
    E, F, _ = gpu_pair(h64, s, "smooth", A, 2.0)
    assert E == 1.0 and np.all(F == 0)


def test_lj_singular_origin_is_domain_error(h64):
    # gpu_pairs.jl:38-87: singular LJ origin raises DomainError
    s = WL.System(np.zeros((2, 3)), np.diag([30.0, 30, 30]), (1, 1, 1), [0, 0])
    with pytest.raises(lib.DomainError):
        gpu_pair(h64, s, "lj", (WL.LJ_EPS, WL.LJ_SIGMA), WL.LJ_CUTOFF)


@pytest.mark.parametrize("shear", [0.0, 0.2])
def test_lj_fcc(h64, shear):
    s = WL.lj_fcc(nc=8, shear=shear)
    E, F, W = gpu_pair(h64, s, "lj", (WL.LJ_EPS, WL.LJ_SIGMA), WL.LJ_CUTOFF)
    Eo, Fo, Wo, npairs = O.pair_evaluate(s.X, s.H, s.pbc, s.species, "lj", (WL.LJ_EPS, WL.LJ_SIGMA), WL.LJ_CUTOFF)
    assert_close(E, F, W, Eo, Fo, Wo)
    assert h64.pair_count() == npairs


def test_boundary_stress_bit_exact_set(h64):
    # pairs placed at |d| = c ± 1 ulp, also across the periodic boundary
    c = 2.0
    L = 12.8
    xs = []
    for k, base in enumerate([0.3, 5.0, L - 0.7]):
        for dx in (np.nextafter(c, 0), c, np.nextafter(c, 4)):
            xs.append([base, 1.0 + 2.5 * k, 1.0])
            xs.append([(base + dx) % L, 1.0 + 2.5 * k, 1.0])
    X = np.array(xs)
    s = WL.System(X, np.diag([L, L, L]), (1, 1, 1), np.zeros(len(X), np.int32))
    h64.set_geometry(s.X, s.H, s.pbc, s.species)
    offs, j, S, R = h64.neighbour_list(c)
    oo, jo, So, Ro = O.neighbour_list(s.X, s.H, s.pbc, c, brute_threshold=0)
    assert snapshot_set(offs, j, S) == snapshot_set(oo, jo, So)


def test_determinism(h64):
    s = WL.smooth_fcc(seed=7)
    r1 = gpu_pair(h64, s, "smooth", A, 2.0)
    r2 = gpu_pair(h64, s, "smooth", A, 2.0)
    assert r1[0] == r2[0] and np.array_equal(r1[1], r2[1]) and np.array_equal(r1[2], r2[2])


@pytest.mark.parametrize("kind", ["smooth", "lj"])
def test_mixed_precision_error(h32, kind):
    if kind == "smooth":
        s, params, c = WL.smooth_fcc(), A, 2.0
    else:
        s, params, c = WL.lj_fcc(nc=8), (WL.LJ_EPS, WL.LJ_SIGMA), WL.LJ_CUTOFF
    E, F, W = gpu_pair(h32, s, kind, params, c)
    Eo, Fo, Wo, _ = O.pair_evaluate(s.X, s.H, s.pbc, s.species, kind, params, c)
    rmse = float(np.sqrt(np.mean((F - Fo) ** 2)))
    assert rmse <= 1e-3, rmse
    assert abs(E - Eo) <= 1e-5 * max(1.0, abs(Eo)) * len(s)
