"""compare_precision (ACE/precision.jl:33-121): the FP32-against-FP64 report of
the GPU evaluators — per-structure and pooled maxima and RMS against a direct
computation from the two workspaces, tolerance statuses, and the failure
record of a structure whose evaluation raises."""
import math
import os

import numpy as np
import pytest

from pfw_b200 import api
from pfw_b200 import precision as PR
from pfw_b200 import workloads as WL
from pfw_b200.ace_model import PackedACE

HERE = os.path.dirname(os.path.abspath(__file__))


def test_tolerances_are_validated_before_any_evaluation():
    with pytest.raises(api.ArgumentError):
        PR.compare_precision(api.lennard_jones(), [], tolerances={"energy": -1.0})
    with pytest.raises(api.ArgumentError):
        PR.compare_precision(api.lennard_jones(), [], tolerances={"stress": 1.0})


@pytest.mark.gpu
def test_ace_report_matches_direct_differences():
    d = np.load(os.path.join(HERE, "golden", "tial_ace.npz"))
    calc = api.ACECalculator(PackedACE.from_npz_dict(d, "model_"))
    frames = [WL.System(d[f"f{k}_X"], d[f"f{k}_H"], (1, 1, 1), d[f"f{k}_species"]) for k in (32, 5, 31)]
    rep = PR.compare_precision(calc, frames)
    assert rep["aggregate"]["status"] == "descriptive" and len(rep["records"]) == 3
    w64, w32 = api.Workspace(), api.Workspace(precision="mixed")
    sq, cnt, fmax = 0.0, 0, 0.0
    for rec, f in zip(rep["records"], frames):
        a, b = api.evaluate_(w64, f, calc), api.evaluate_(w32, f, calc)
        df = b["forces"] - a["forces"]
        assert rec["metrics"]["forces"]["maximum"] == pytest.approx(np.abs(df).max(), rel=1e-12, abs=0)
        assert rec["metrics"]["energy"]["per_atom"] == pytest.approx(abs(b["energy"] - a["energy"]) / len(f.X))
        assert rec["metrics"]["forces"]["max_atom_vector"] == pytest.approx(np.sqrt((df ** 2).sum(axis=1)).max())
        sq += float((df ** 2).sum())
        cnt += df.size
        fmax = max(fmax, float(np.abs(df).max()))
    agg = rep["aggregate"]["forces"]
    assert agg["maximum"] == pytest.approx(fmax) and agg["pooled_rms"] == pytest.approx(math.sqrt(sq / cnt))
    assert 0 < agg["maximum"] < 4e-3  # the reference's FP32 bar for GPU ACE forces
    strict = PR.compare_precision(calc, frames[:1], tolerances={"forces": 1e-14})
    assert strict["aggregate"]["status"] == "failed"
    loose = PR.compare_precision(calc, frames[:1], tolerances={"forces": 1.0, "energy": 1.0, "virial": 10.0})
    assert loose["aggregate"]["status"] == "passed"


@pytest.mark.gpu
def test_pair_report_and_failed_structure():
    p = api.lennard_jones(0.0104, 3.4, 8.5)
    good = WL.lj_fcc(seed=3, nc=5)
    X = good.X.copy()
    X[1] = X[0]  # coincident atoms: LJ is singular there → DomainError in both precisions
    bad = WL.System(X, good.H, good.pbc, good.species)
    rep = PR.compare_precision(p, [good, bad], properties=(api.Energy(), api.Forces()))
    assert rep["records"][0]["status"] == "descriptive"
    assert rep["records"][1]["status"] == "failed" and rep["records"][1]["errors"]
    assert rep["aggregate"]["status"] == "failed" and math.isinf(rep["aggregate"]["forces"]["maximum"])
    assert set(rep["records"][0]["metrics"]) == {"energy", "forces"}
