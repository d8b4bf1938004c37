"""The May30 Ti–Al–V model on the GPU (real solid harmonics through l = 6,
114 radial channels on 1000 spline nodes, PolyEnvelope1sR pairs, 5652
products — a model the reference's own device packing rejects,
adaptation.jl:72,79): every frame against the reference's cached
ACEpotentials predictions at the reference's tolerances (test/ace_may30.jl:3-7)
and against the CPU oracle at 1e-10; explicit schedules (which move the
product/term tables between shared and global memory) agree; the three
frames as one batch, eager and replayed, with their fitting features."""
import os

import numpy as np
import pytest

from oracle import oracle as O
from pfw_b200 import lib
from pfw_b200 import workloads as WL
from pfw_b200.ace_model import PackedACE

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
MODEL = os.path.join(HERE, "golden", "may30_model.npz")
needs_model = pytest.mark.skipif(not os.path.exists(MODEL), reason="May30 model tables not generated")
RTOL = 1e-10


@pytest.fixture(scope="module")
def may30():
    return PackedACE.from_npz_dict(np.load(MODEL), "model_"), np.load(os.path.join(HERE, "golden", "may30_frames.npz"))


def frame(fr, k):
    return WL.System(fr[f"f{k}_X"], fr[f"f{k}_H"], (1, 1, 1), fr[f"f{k}_species"])


def close(a, b, rtol=RTOL):
    a, b = np.asarray(a), np.asarray(b)
    return bool(np.all(np.abs(a - b) <= rtol * max(1.0, float(np.abs(b).max()))))


@needs_model
@pytest.mark.parametrize("k", [0, 1, 2])
def test_frames_match_predictions_and_oracle(may30, k):
    m, fr = may30
    s = frame(fr, k)
    h = lib.Handle(lib.FP64)
    h.ace(m)
    h.set_geometry(s.X, s.H, s.pbc, s.species)
    E, F, W = h.evaluate(lib.MODEL_ACE, 7)
    assert abs(E - float(fr[f"f{k}_energy"])) <= 2e-8
    Fr, Wr = fr[f"f{k}_forces"], fr[f"f{k}_virial"]
    assert np.all(np.abs(F - Fr) <= 2e-9 + 2e-11 * np.abs(Fr))
    assert np.all(np.abs(W - Wr) <= 2e-8 + 2e-11 * np.abs(Wr))
    r = O.AceOracle(m).evaluate(s.X, s.H, s.pbc, s.species, nthreads=4)
    assert abs(E - r["energy"]) <= RTOL * abs(r["energy"])
    assert close(F, r["forces"]) and close(W, r["virial"])


@needs_model
def test_schedules_agree(may30):
    m, fr = may30
    s = frame(fr, 2)
    h = lib.Handle(lib.FP64)
    h.ace(m)
    h.set_geometry(s.X, s.H, s.pbc, s.species)
    E0, F0, W0 = h.evaluate(lib.MODEL_ACE, 7)
    for chunk, groups in ((8, 1), (8, 2), (8, 4), (16, 2)):
        h.ace_schedule(chunk, groups)
        E, F, W = h.evaluate(lib.MODEL_ACE, 7)
        assert abs(E - E0) <= 1e-12 * abs(E0)
        assert close(F, F0, 1e-12) and close(W, W0, 1e-12)


@needs_model
def test_batch_with_features_and_graph(may30):
    import torch
    m, fr = may30
    systems = [frame(fr, k) for k in range(3)]
    h = lib.Handle(lib.FP64)
    h.ace(m)
    h.set_batch(systems)
    E, F, W, X = h.evaluate_batch(lib.MODEL_ACE, 7, features=True)
    offs = h.batch_offsets
    ace = O.AceOracle(m)
    for k, s in enumerate(systems):
        r = ace.evaluate(s.X, s.H, s.pbc, s.species, features=True, nthreads=4)
        assert abs(E[k] - r["energy"]) <= RTOL * abs(r["energy"])
        assert close(F[offs[k]:offs[k + 1]], r["forces"]) and close(W[k], r["virial"])
        assert close(X[k], r["features"].sum(axis=0))
    dev = torch.device("cuda", 0)
    Eg = torch.zeros(3, dtype=torch.float64, device=dev)
    Fg = torch.zeros(h.n * 3, dtype=torch.float64, device=dev)
    Wg = torch.zeros(27, dtype=torch.float64, device=dev)
    for _ in range(2):
        h.batch_graph_launch(7, Eg.data_ptr(), Fg.data_ptr(), Wg.data_ptr(), None)
        h.batch_graph_sync()
    Ee, Fe, _, _ = h.evaluate_batch(lib.MODEL_ACE, 7)
    assert np.array_equal(Eg.cpu().numpy(), Ee) and np.array_equal(Fg.cpu().numpy().reshape(-1, 3), Fe)
