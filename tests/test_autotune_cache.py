"""Autotuner bookkeeping without a GPU: model keys are content hashes,
workload keys bucket the atom count, and the JSON cache round-trips."""
import numpy as np

from pfw_b200 import ace_generate as G
from pfw_b200 import autotune as A
from pfw_b200.ace_model import read_resolved


def test_model_key_is_content_hash():
    m = read_resolved(G.generate_b2_model())
    k1 = A.model_key(m)
    m.WB = m.WB.copy()
    assert A.model_key(m) == k1
    m.WB[0, 0] += 1e-12
    assert A.model_key(m) != k1


def test_workload_key_buckets():
    assert A.workload_key(16000) == A.workload_key(16384) == "n16384_s1"
    assert A.workload_key(16385) == "n32768_s1"
    assert A.workload_key(290502, 4096) == "n524288_s4096"


def test_cache_roundtrip(tmp_path):
    p = str(tmp_path / "sub" / "tune.json")
    assert A._load(p) == {}
    A._store(p, {"k": {"schedule": [16, 4], "ms": {"16x4": 1.5}}})
    assert A._load(p)["k"]["schedule"] == [16, 4]
