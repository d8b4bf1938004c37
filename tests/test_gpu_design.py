"""GPU design rows of the ACE model (design_matrix_impl, ACE/fitting.jl:18-67),
checked column by column against the CPU oracle: column c of a structure's
rows is, by linearity, the energy, forces and virial of the model whose
readout is the unit vector e_c with no reference energies — an oracle
evaluation.  Also: the stacked batch equals the single-structure rows, the
rows are deterministic, A·[vec(WB); vec(Wpair)] + baseline reproduces the
evaluation (with trainable radial scales, and for the May30 model against
the reference's cached predictions), and fit_pair=False moves the pair term
into the baseline.  FP64 bar: 1e-10 of each column's largest entry."""
import dataclasses
import os

import numpy as np
import pytest

from oracle import oracle as O
from pfw_b200 import ace_generate as G
from pfw_b200 import api
from pfw_b200 import fitting as FT
from pfw_b200 import lib
from pfw_b200 import workloads as WL
from pfw_b200.ace_model import PackedACE, read_resolved

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
RTOL = 1e-10


@pytest.fixture(scope="module")
def tial():
    d = np.load(os.path.join(HERE, "golden", "tial_ace.npz"))
    return PackedACE.from_npz_dict(d, "model_"), d


def frame(d, k):
    return WL.System(d[f"f{k}_X"], d[f"f{k}_H"], (1, 1, 1), d[f"f{k}_species"])


def rows_of(E, F, W):
    return np.concatenate([[E], np.asarray(F).ravel(), np.asarray(W).ravel(order="F")])


def unit_model(m, c):
    nz, nb, nq = m.nz, m.nbasis, m.pair.nchannels
    theta = np.zeros(nz * (nb + nq))
    theta[c] = 1.0
    WB = theta[:nz * nb].reshape(nb, nz, order="F")
    Wp = theta[nz * nb:].reshape(nq, nz, order="F")
    u = m.with_parameters({"WB": WB, "Wpair": Wp})
    return dataclasses.replace(u, reference=np.zeros_like(m.reference))


def test_columns_match_oracle_unit_readouts(tial):
    m, d = tial
    frames = [frame(d, k) for k in (32, 0, 7)]
    calc = api.ACECalculator(m)
    A = FT.design_matrix(frames, calc)["matrix"]
    nz, nb, nq = m.nz, m.nbasis, m.pair.nchannels
    assert A.shape == (sum(10 + 3 * len(f.X) for f in frames), nz * (nb + nq))
    for c in range(A.shape[1]):
        ace = O.AceOracle(unit_model(m, c))
        r0 = 0
        for f in frames:
            ref = ace.evaluate(f.X, f.H, f.pbc, f.species)
            want = rows_of(ref["energy"], ref["forces"], ref["virial"])
            got = A[r0:r0 + len(want), c]
            scale = max(1.0, float(np.abs(want).max()))
            assert np.all(np.abs(got - want) <= RTOL * scale), (c, np.abs(got - want).max())
            r0 += len(want)


def test_batch_stacks_single_rows_and_is_deterministic(tial):
    m, d = tial
    frames = [frame(d, k) for k in (32, 3, 31)]
    calc = api.ACECalculator(m)
    h = lib.Handle(lib.FP64)
    a1 = FT.design_matrix(frames, calc, handle=h)
    a2 = FT.design_matrix(frames, calc, handle=h)
    assert np.array_equal(a1["matrix"], a2["matrix"])
    r0 = 0
    for f in frames:
        s = FT.design_matrix(f, calc)
        n = s["matrix"].shape[0]
        assert np.allclose(a1["matrix"][r0:r0 + n], s["matrix"], rtol=0, atol=1e-12 * np.abs(s["matrix"]).max())
        assert np.array_equal(a1["baseline"][r0:r0 + n], s["baseline"])
        r0 += n


def test_linear_readout_reproduces_evaluation_with_scales():
    m = read_resolved(G.generate_b2_model())
    calc = api.ACECalculator(m)
    tp = api.trainable_parameters(calc, calc.parameters)
    rng = np.random.default_rng(3)
    tp["radial"]["scale"] *= rng.uniform(0.8, 1.2, tp["radial"]["scale"].shape)
    tp["pair"]["scale"] *= rng.uniform(0.8, 1.2, tp["pair"]["scale"].shape)
    tp["WB"] = tp["WB"] * rng.uniform(0.5, 1.5, tp["WB"].shape)
    calc.set_parameters(tp)
    systems = WL.batched(seed=9, nsys=5, nmin=8, nmax=48, workers=1)
    des = FT.design_matrix(systems, calc)
    pred = des["matrix"] @ FT.linear_parameters(tp) + des["baseline"]
    runtime = O.AceOracle(m.with_parameters({"WB": tp["WB"], "Wpair": tp["Wpair"]}), tp["radial"]["scale"],
                          tp["pair"]["scale"])
    r0 = 0
    for s in systems:
        ref = runtime.evaluate(s.X, s.H, s.pbc, s.species)
        want = rows_of(ref["energy"], ref["forces"], ref["virial"])
        got = pred[r0:r0 + len(want)]
        assert np.all(np.abs(got - want) <= RTOL * max(1.0, float(np.abs(want).max())))
        r0 += len(want)
    # fit_pair=False: the pair columns move into the baseline
    nb = m.nz * m.nbasis
    des2 = FT.design_matrix(systems, calc, fit_pair=False)
    assert des2["matrix"].shape[1] == nb
    pred2 = des2["matrix"] @ np.asarray(tp["WB"]).ravel(order="F") + des2["baseline"]
    assert np.allclose(pred2, pred, rtol=0, atol=1e-10 * np.abs(pred).max())
    # training rows and readout installation
    tr = FT.training_rows(FT.design_matrix(systems[0], calc), {"energy": 1.0, "forces": None,
                                                               "virial": np.eye(3)}, {"virial": 0.5})
    assert tr["matrix"].shape[0] == 10 and np.all(tr["row_weights"][1:] == 0.5)
    back = FT.install_readout(tp, FT.linear_parameters(tp))
    assert np.array_equal(back["WB"], tp["WB"]) and np.array_equal(back["Wpair"], tp["Wpair"])


def test_may30_rows_reproduce_predictions():
    path = os.path.join(HERE, "golden", "may30_model.npz")
    if not os.path.exists(path):
        pytest.skip("May30 model tables not generated")
    m = PackedACE.from_npz_dict(np.load(path), "model_")
    fr = np.load(os.path.join(HERE, "golden", "may30_frames.npz"))
    f = WL.System(fr["f0_X"], fr["f0_H"], (1, 1, 1), fr["f0_species"])
    calc = api.ACECalculator(m)
    des = FT.design_matrix(f, calc)
    pred = des["matrix"] @ FT.linear_parameters(calc.parameters) + des["baseline"]
    ref = O.AceOracle(m).evaluate(f.X, f.H, f.pbc, f.species, nthreads=4)
    want = rows_of(ref["energy"], ref["forces"], ref["virial"])
    assert np.all(np.abs(pred - want) <= RTOL * np.abs(want).max())
    # and the reference's cached ACEpotentials predictions, relative to the
    # rows' scale (a dot product over 6,495 columns)
    pf = rows_of(float(fr["f0_energy"]), fr["f0_forces"], fr["f0_virial"])
    assert np.all(np.abs(pred - pf) <= RTOL * np.abs(pf).max())


def test_open_cluster_columns_and_buffer_errors(tial):
    m, d = tial
    f = frame(d, 32)
    cl = WL.System(f.X, f.H, (0, 0, 0), f.species)  # the same atoms as an open cluster
    calc = api.ACECalculator(m)
    A = FT.design_matrix(cl, calc)["matrix"]
    rng = np.random.default_rng(11)
    for c in rng.choice(A.shape[1], 24, replace=False):
        ref = O.AceOracle(unit_model(m, int(c))).evaluate(cl.X, cl.H, cl.pbc, cl.species)
        want = rows_of(ref["energy"], ref["forces"], ref["virial"])
        assert np.all(np.abs(A[:, c] - want) <= RTOL * max(1.0, float(np.abs(want).max())))
    h = lib.Handle(lib.FP64)
    h.ace(m)
    h.set_geometry(cl.X, cl.H, cl.pbc, cl.species)
    rows, cols = h.design_shape()
    small = np.zeros((rows - 1, cols))
    with pytest.raises(lib.PFWError) as ei:
        h.check(h.L.pfw_ace_design_matrix(h.ws, small.ctypes.data_as(lib.C.POINTER(lib.C.c_double)), cols,
                                          rows - 1, None))
    assert ei.value.code == lib.ESHAPE
