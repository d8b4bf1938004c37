"""GPU parity of the ACE path: the reference's saved TiAl oracle (33 frames,
test/neighbour_saved_reference.jl tolerances) and the CPU oracle on the
synthetic C3 model over minimum-image, small-box and triclinic geometries.
FP64 bar: energy/forces/virial within 1e-10 relative of the oracle."""
import os

import numpy as np
import pytest

from oracle import oracle as O
from pfw_b200 import ace_generate as G
from pfw_b200 import lib
from pfw_b200 import workloads as WL
from pfw_b200.ace_model import PackedACE, read_resolved

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def tial():
    d = np.load(os.path.join(HERE, "golden", "tial_ace.npz"))
    return d, PackedACE.from_npz_dict(d, "model_")


@pytest.fixture(scope="module")
def b2model():
    return read_resolved(G.generate_b2_model())


def gpu_ace(h, model, X, H, pbc, species, request=7):
    h.ace(model)
    h.set_geometry(X, H, pbc, species)
    return h.evaluate(lib.MODEL_ACE, request)


def close(a, b, rtol=1e-10, atol=1e-12):
    scale = max(1.0, float(np.max(np.abs(b)))) if np.size(b) else 1.0
    return np.all(np.abs(np.asarray(a) - np.asarray(b)) <= rtol * scale + atol)


def test_tial_saved_oracle(tial):
    d, m = tial
    h = lib.Handle(lib.FP64)
    ace = O.AceOracle(m)
    for k in range(int(d["nframes"])):
        X, H, z = d[f"f{k}_X"], d[f"f{k}_H"], d[f"f{k}_species"]
        E, F, W = gpu_ace(h, m, X, H, (1, 1, 1), z)
        assert abs(E - float(d[f"f{k}_energy"])) <= 1e-8
        Fr = d[f"f{k}_forces"]
        assert np.all(np.abs(F - Fr) <= 1e-9 + 1e-10 * np.abs(Fr))
        Vr = d[f"f{k}_virial"]
        assert np.all(np.abs(W - Vr) <= 1e-8 + 1e-10 * np.abs(Vr))
        r = ace.evaluate(X, H, (1, 1, 1), z, site_energies=True)
        assert abs(E - r["energy"]) <= 1e-10 * abs(r["energy"])
        assert close(F, r["forces"]) and close(W, r["virial"])
        assert close(h.site_energies(), r["site_energies"])


@pytest.mark.parametrize("nc", [3, 4, 6, 8])
def test_b2_boxes(b2model, nc):
    # nc=3: explicit images (L < 2c); 4, 6: minimum image with < 4 bins; 8: per-cell wrap
    s = WL.b2(nc=nc, seed=nc)
    h = lib.Handle(lib.FP64)
    E, F, W = gpu_ace(h, b2model, s.X, s.H, s.pbc, s.species)
    r = O.AceOracle(b2model).evaluate(s.X, s.H, s.pbc, s.species, site_energies=True)
    assert abs(E - r["energy"]) <= 1e-10 * max(1.0, abs(r["energy"]))
    assert close(F, r["forces"]) and close(W, r["virial"])
    assert close(h.site_energies(), r["site_energies"])


def test_triclinic_small_systems(b2model):
    systems = WL.batched(seed=9, nsys=6, nmin=8, nmax=64)
    h = lib.Handle(lib.FP64)
    ace = O.AceOracle(b2model)
    for s in systems:
        E, F, W = gpu_ace(h, b2model, s.X, s.H, s.pbc, s.species)
        r = ace.evaluate(s.X, s.H, s.pbc, s.species)
        assert abs(E - r["energy"]) <= 1e-10 * max(1.0, abs(r["energy"]))
        assert close(F, r["forces"]) and close(W, r["virial"])


def test_energy_only_and_determinism(b2model):
    s = WL.b2(nc=5, seed=3)
    h = lib.Handle(lib.FP64)
    E1, F1, W1 = gpu_ace(h, b2model, s.X, s.H, s.pbc, s.species)
    E2, F2, W2 = gpu_ace(h, b2model, s.X, s.H, s.pbc, s.species)
    assert E1 == E2 and np.array_equal(F1, F2) and np.array_equal(W1, W2)
    E0, _, _ = gpu_ace(h, b2model, s.X, s.H, s.pbc, s.species, request=1)
    assert abs(E0 - E1) <= 1e-12 * abs(E1)


def test_coincident_atoms_domain_error(b2model):
    X = np.array([[1.0, 1.0, 1.0], [1.0, 1.0, 1.0], [2.5, 1.0, 1.0]])
    h = lib.Handle(lib.FP64)
    with pytest.raises(lib.DomainError):
        gpu_ace(h, b2model, X, np.diag([20.0, 20, 20]), (1, 1, 1), [0, 1, 0])


def test_rotation_invariance_gpu(b2model):
    s = WL.b2(nc=4, seed=5)
    th = 0.4
    Rm = np.array([[np.cos(th), -np.sin(th), 0], [np.sin(th), np.cos(th), 0], [0, 0, 1]])
    h = lib.Handle(lib.FP64)
    E, F, W = gpu_ace(h, b2model, s.X, s.H, s.pbc, s.species)
    E2, F2, W2 = gpu_ace(h, b2model, s.X @ Rm.T, Rm @ s.H, s.pbc, s.species)
    assert abs(E - E2) <= 1e-10 * abs(E)
    assert np.abs(F2 - F @ Rm.T).max() <= 1e-9


def test_mixed_precision_form(b2model):
    # FP32 site arithmetic, FP64 energy/virial accumulation: stated force RMSE ≤ 1e-3 eV/Å
    s = WL.b2(nc=8, seed=2)
    E64, F64, W64 = gpu_ace(lib.Handle(lib.FP64), b2model, s.X, s.H, s.pbc, s.species)
    E32, F32, W32 = gpu_ace(lib.Handle(lib.MIXED), b2model, s.X, s.H, s.pbc, s.species)
    rmse = float(np.sqrt(np.mean((F32 - F64) ** 2)))
    assert rmse <= 1e-3, rmse
    assert abs(E32 - E64) <= 1e-5 * abs(E64)


def test_autotune_picks_fastest_and_caches(b2model, tmp_path):
    from pfw_b200 import autotune
    s = WL.b2(nc=6, seed=7)
    h = lib.Handle(lib.FP64)
    h.ace(b2model)
    h.set_geometry(s.X, s.H, s.pbc, s.species)
    path = str(tmp_path / "tune.json")
    c, g, ms = autotune.tune(h, b2model, lambda: h.evaluate(lib.MODEL_ACE, 7), len(s.species), path=path, reps=2)
    assert f"{c}x{g}" == min(ms, key=ms.get) and len(ms) >= 3
    E1, F1, W1 = h.evaluate(lib.MODEL_ACE, 7)
    r = O.AceOracle(b2model).evaluate(s.X, s.H, s.pbc, s.species)
    assert close(F1, r["forces"]) and abs(E1 - r["energy"]) <= 1e-10 * abs(r["energy"])
    c2, g2, ms2 = autotune.tune(h, b2model, lambda: None, len(s.species), path=path)
    assert (c2, g2) == (c, g) and ms2 == ms
