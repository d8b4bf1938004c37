"""The host mirror of the reference API on the GPU, checked against the CPU
oracle: evaluate_/evaluate with SmoothPair and lennard_jones, explicit
parameters, the AtomsCalculators functions (in-place variants add into the
destination), calculate with state, a Workspace with a skin, and an
ACECalculator restored from a checkpoint with tuned readout and radial
scales (the oracle applies the scales at run time, the device tables fold
them into the splines).  FP64 bar: 1e-10 relative."""
import os
from types import SimpleNamespace

import numpy as np
import pytest

import pfw_b200 as P
from oracle import oracle as O
from pfw_b200 import checkpoint as CK
from pfw_b200 import workloads as WL
from pfw_b200.ace_model import PackedACE

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
RTOL = 1e-10


def close(a, b, rtol=RTOL):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return bool(np.all(np.abs(a - b) <= rtol * max(1.0, float(np.abs(b).max(initial=0.0)))))


@pytest.fixture(scope="module")
def tial():
    d = np.load(os.path.join(HERE, "golden", "tial_ace.npz"))
    return PackedACE.from_npz_dict(d, "model_"), d


def test_smooth_pair_evaluate_and_parameters():
    s = WL.smooth_fcc(seed=3, nc=5)
    p = P.SmoothPair(["A", "B"], WL.SMOOTH_A, 2.0)
    sysl = SimpleNamespace(X=s.X, H=s.H, pbc=s.pbc, species=np.array(["AB"[z] for z in s.species]))
    r = P.evaluate(sysl, p)
    e, f, w, _ = O.pair_evaluate(s.X, s.H, s.pbc, s.species, "smooth", WL.SMOOTH_A, 2.0)
    assert abs(r["energy"] - e) <= RTOL * abs(e) and close(r["forces"], f) and close(r["virial"], w)
    # explicit parameters: upper triangle in column order (models.jl:103-110)
    A2 = np.array(WL.SMOOTH_A, np.float64) * 1.3
    tri = [A2[i, j] for j in range(2) for i in range(j + 1)]
    r2 = P.evaluate_(P.Workspace(), sysl, p, parameters={"amplitudes": tri})
    e2, _, _, _ = O.pair_evaluate(s.X, s.H, s.pbc, s.species, "smooth", A2, 2.0)
    assert abs(r2["energy"] - e2) <= RTOL * abs(e2)
    with pytest.raises(P.ArgumentError):
        P.evaluate_(P.Workspace(), sysl, p, parameters={"amplitudes": tri, "radius": 3.0})


def test_lj_atomscalculators_and_state():
    s = WL.lj_fcc(seed=4, nc=6)
    p = P.lennard_jones(0.0104, 3.4, 8.5)
    ws = P.Workspace()
    e, f, w, _ = O.pair_evaluate(s.X, s.H, s.pbc, s.species, "lj", (0.0104, 3.4), 8.5)
    assert abs(P.potential_energy(s, p, ws) - e) <= RTOL * abs(e)
    assert close(P.forces(s, p, ws), f) and close(P.virial(s, p, ws), w)
    F = np.ones_like(f)
    P.forces_(F, s, p, ws)
    assert close(F, f + 1.0)
    r = P.calculate((P.Energy(), P.Forces()), s, p, parameters={"epsilon": 0.0208, "sigma": 3.4}, state="st")
    assert set(r) == {"energy", "forces", "state"} and r["state"] == "st"
    assert abs(r["energy"] - 2 * e) <= RTOL * abs(2 * e)
    with pytest.raises(P.DimensionMismatch):
        P.forces_(np.zeros((3, 3)), s, p, ws)


def test_workspace_skin_matches_rebuild():
    s = WL.lj_fcc(seed=5, nc=6)
    p = P.lennard_jones(0.0104, 3.4, 8.5)
    ws = P.Workspace(skin=1.0)
    rng = np.random.default_rng(0)
    X = s.X.copy()
    for step in range(4):
        X = X + rng.normal(0, 0.02, X.shape)
        sk = WL.System(X, s.H, s.pbc, s.species)
        r = P.evaluate_(ws, sk, p)
        e, f, w, _ = O.pair_evaluate(X, s.H, s.pbc, s.species, "lj", (0.0104, 3.4), 8.5)
        assert abs(r["energy"] - e) <= RTOL * abs(e) and close(r["forces"], f) and close(r["virial"], w)
    builds, reuses = ws.handle.skin_stats()
    assert builds == 1 and reuses == 3
    with pytest.raises(P.ArgumentError):
        P.Workspace(skin=-1.0)


def test_ace_checkpoint_restored_calculator(tmp_path, tial):
    m, d = tial
    original = P.ACECalculator(m)
    tp = P.trainable_parameters(original, original.parameters)
    tp["WB"] *= 0.83
    tp["Wpair"] *= 1.12
    tp["radial"]["scale"][:, 0, 1] *= 0.91
    tp["pair"]["scale"][0, 1, 0] = 0.0
    path = str(tmp_path / "trained.toml")
    P.save_calculator(path, original, tp, {"epoch": np.int32(3)})
    restored = P.ACECalculator(path)
    runtime = O.AceOracle(m.with_parameters({"WB": tp["WB"], "Wpair": tp["Wpair"]}),
                          tp["radial"]["scale"], tp["pair"]["scale"])
    for k in (0, 11, 30):
        sy = WL.System(d[f"f{k}_X"], d[f"f{k}_H"], (1, 1, 1), d[f"f{k}_species"])
        ref = runtime.evaluate(sy.X, sy.H, sy.pbc, sy.species)
        r = P.energy_forces_virial(sy, restored)
        assert abs(r["energy"] - ref["energy"]) <= RTOL * abs(ref["energy"])
        assert close(r["forces"], ref["forces"]) and close(r["virial"], ref["virial"])
        # explicit parameters through calculate equal the installed ones
        c = P.calculate((P.Energy(),), sy, original, parameters=tp)
        assert abs(c["energy"] - r["energy"]) <= 1e-12 * abs(r["energy"]) and c["state"] == {}
    assert P.calculate(P.Energy(), sy, restored)["state"] == {"epoch": np.int32(3)}
    # the untouched original still reproduces the saved reference energies
    k = 5
    sy = WL.System(d[f"f{k}_X"], d[f"f{k}_H"], (1, 1, 1), d[f"f{k}_species"])
    assert abs(P.potential_energy(sy, original) - float(d[f"f{k}_energy"])) <= 1e-8
    assert CK.CHECKPOINT_SCHEMA in open(path).read()
