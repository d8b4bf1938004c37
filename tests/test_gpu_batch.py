"""GPU parity of batched evaluation: many independent small triclinic systems
in one launch (per-system energy, forces, virial and the energy-row fitting
features of ACE/fitting.jl:28-29), checked system by system against the CPU
oracle; the CUDA-graph replay path against the eager batch path; and the
capacity error of a replay whose environments outgrew the captured plan.
FP64 bar: 1e-10 relative."""
import numpy as np
import pytest

from oracle import oracle as O
from pfw_b200 import ace_generate as G
from pfw_b200 import lib
from pfw_b200 import workloads as WL
from pfw_b200.ace_model import read_resolved

pytestmark = pytest.mark.gpu
RTOL = 1e-10


@pytest.fixture(scope="module")
def b2model():
    return read_resolved(G.generate_b2_model())


@pytest.fixture(scope="module")
def systems():
    return WL.batched(seed=21, nsys=24, nmin=8, nmax=96)


def close(a, b, rtol=RTOL, atol=1e-12):
    a, b = np.asarray(a), np.asarray(b)
    scale = max(1.0, float(np.max(np.abs(b)))) if b.size else 1.0
    return bool(np.all(np.abs(a - b) <= rtol * scale + atol))


def test_ace_batch_matches_oracle_per_system(b2model, systems):
    h = lib.Handle(lib.FP64)
    h.ace(b2model)
    h.set_batch(systems)
    E, F, W, X = h.evaluate_batch(lib.MODEL_ACE, 7, features=True)
    ace = O.AceOracle(b2model)
    offs = h.batch_offsets
    assert X.shape == (len(systems), b2model.nz * (b2model.nbasis + b2model.pair.nchannels))
    for s, sy in enumerate(systems):
        r = ace.evaluate(sy.X, sy.H, sy.pbc, sy.species, features=True)
        assert abs(E[s] - r["energy"]) <= RTOL * max(1.0, abs(r["energy"]))
        assert close(F[offs[s]:offs[s + 1]], r["forces"])
        assert close(W[s], r["virial"])
        assert close(X[s], r["features"].sum(axis=0))


def test_batch_features_reproduce_energy(b2model, systems):
    # E_s = Σ_z WB[z]·ΣB + Wpair[z]·ΣQ + Σ_i reference[z_i]: the linear model the features feed
    h = lib.Handle(lib.FP64)
    h.ace(b2model)
    h.set_batch(systems)
    E, _, _, X = h.evaluate_batch(lib.MODEL_ACE, 1, features=True)
    nz, nB, nQ = b2model.nz, b2model.nbasis, b2model.pair.nchannels
    WB = np.asarray(b2model.WB).reshape(nz, nB)
    WP = np.asarray(b2model.Wpair).reshape(nz, nQ)
    ref = np.asarray(b2model.reference)
    for s, sy in enumerate(systems):
        lin = sum(WB[z] @ X[s, z * nB:(z + 1) * nB] + WP[z] @ X[s, nz * nB + z * nQ:nz * nB + (z + 1) * nQ]
                  for z in range(nz))
        lin += ref[sy.species].sum()
        assert abs(lin - E[s]) <= 1e-9 * max(1.0, abs(E[s]))


def test_batch_equals_single_system_calls(b2model, systems):
    h = lib.Handle(lib.FP64)
    h.ace(b2model)
    h.set_batch(systems[:6])
    E, F, W, _ = h.evaluate_batch(lib.MODEL_ACE, 7)
    offs = h.batch_offsets
    g = lib.Handle(lib.FP64)
    g.ace(b2model)
    for s, sy in enumerate(systems[:6]):
        g.set_geometry(sy.X, sy.H, sy.pbc, sy.species)
        e, f, w = g.evaluate(lib.MODEL_ACE, 7)
        assert abs(E[s] - e) <= 1e-12 * max(1.0, abs(e))
        assert close(F[offs[s]:offs[s + 1]], f, rtol=1e-12) and close(W[s], w, rtol=1e-12)


def test_pair_batch_matches_oracle(systems):
    h = lib.Handle(lib.FP64)
    h.smooth(WL.SMOOTH_A, 2.0)
    h.set_batch(systems)
    E, F, W, _ = h.evaluate_batch(lib.MODEL_PAIR, 7)
    offs = h.batch_offsets
    for s, sy in enumerate(systems):
        e, f, w, _ = O.pair_evaluate(sy.X, sy.H, sy.pbc, sy.species, "smooth", WL.SMOOTH_A, 2.0)
        assert abs(E[s] - e) <= 1e-11 * max(1.0, abs(e))
        assert close(F[offs[s]:offs[s + 1]], f, rtol=1e-11)
        assert close(W[s], w, rtol=1e-11)


def _device_outputs(torch, n, nsys, nfeat):
    dev = torch.device("cuda", 0)
    return (torch.zeros(nsys, dtype=torch.float64, device=dev), torch.zeros(n * 3, dtype=torch.float64, device=dev),
            torch.zeros(nsys * 9, dtype=torch.float64, device=dev),
            torch.zeros(nsys * nfeat, dtype=torch.float64, device=dev))


def test_graph_replay_equals_eager(b2model, systems):
    torch = pytest.importorskip("torch")
    h = lib.Handle(lib.FP64)
    h.ace(b2model)
    h.set_batch(systems)
    nfeat = h.feature_count()
    E, F, W, Xf = _device_outputs(torch, h.n, h.nsys, nfeat)
    torch.cuda.synchronize()
    rng = np.random.default_rng(3)
    X0 = np.concatenate([s.X for s in systems])
    for step in range(3):
        Xs = X0 + rng.normal(0, 0.05, X0.shape) if step else X0
        h.batch_update_positions(Xs)
        h.batch_graph_launch(7, E.data_ptr(), F.data_ptr(), W.data_ptr(), Xf.data_ptr())
        h.batch_graph_sync()
        Eg, Fg, Wg, Xg = (t.cpu().numpy().copy() for t in (E, F, W, Xf))
        Ee, Fe, We, Xe = h.evaluate_batch(lib.MODEL_ACE, 7, features=True)
        assert np.array_equal(Eg, Ee)
        assert np.array_equal(Fg.reshape(-1, 3), Fe)
        assert np.array_equal(Wg.reshape(-1, 3, 3).transpose(0, 2, 1), We)
        assert np.array_equal(Xg.reshape(h.nsys, nfeat), Xe)


def test_graph_capacity_overflow_reports_and_replans(b2model):
    torch = pytest.importorskip("torch")
    # 8 sparse systems: 64 atoms in 14 Å cubes (about 16 neighbours per atom)
    rng = np.random.default_rng(8)
    H = np.diag([14.0, 14.0, 14.0])
    systems = [WL.System(WL._hardcore(rng, H, 64, 1.6), H, (1, 1, 1), np.arange(64) % 2) for _ in range(8)]
    h = lib.Handle(lib.FP64)
    h.ace(b2model)
    h.set_batch(systems)
    E, F, W, Xf = _device_outputs(torch, h.n, h.nsys, 1)
    torch.cuda.synchronize()
    h.batch_graph_launch(7, E.data_ptr(), F.data_ptr(), W.data_ptr(), None)
    h.batch_graph_sync()
    # squeeze every system into an eighth of its cell: about 3x the environments,
    # beyond the captured plan's 25 % + 4096 headroom
    Xc = np.concatenate([0.5 * s.X for s in systems])
    h.batch_update_positions(Xc)
    h.batch_graph_launch(7, E.data_ptr(), F.data_ptr(), W.data_ptr(), None)
    with pytest.raises(lib.PFWError) as ei:
        h.batch_graph_sync()
    assert ei.value.code == lib.ECAPACITY
    # the next launch re-plans for the new positions and agrees with the eager path
    h.batch_graph_launch(7, E.data_ptr(), F.data_ptr(), W.data_ptr(), None)
    h.batch_graph_sync()
    Ee, Fe, We, _ = h.evaluate_batch(lib.MODEL_ACE, 7)
    assert np.array_equal(E.cpu().numpy(), Ee)
    assert np.array_equal(F.cpu().numpy().reshape(-1, 3), Fe)
