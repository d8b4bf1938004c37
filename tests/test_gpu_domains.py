"""Slab domain decomposition of one periodic box (pfw_b200/parallel.py) on
one GPU: every domain evaluated in turn with pfw_set_owned, owned forces
assembled and energies/virials summed, must equal the single-box evaluation
(FP64, 1e-10 relative) for Lennard-Jones, SmoothPair and ACE, with 2 to 4
slabs."""
import numpy as np
import pytest

from pfw_b200 import ace_generate as G
from pfw_b200 import lib
from pfw_b200 import parallel as PAR
from pfw_b200 import workloads as WL
from pfw_b200.ace_model import read_resolved

pytestmark = pytest.mark.gpu


def close(a, b, rtol=1e-10):
    a, b = np.asarray(a), np.asarray(b)
    return bool(np.all(np.abs(a - b) <= rtol * max(1.0, float(np.abs(b).max()))))


def check(h, s, model, world, halo):
    h.set_geometry(s.X, s.H, s.pbc, s.species)
    E0, F0, W0 = h.evaluate(model, 7)
    E, F, W = PAR.evaluate_domains(h, s, model, world, halo)
    assert abs(E - E0) <= 1e-10 * max(1.0, abs(E0))
    assert close(F, F0) and close(W, W0)


@pytest.mark.parametrize("world", [2, 3, 4])
def test_lj_slabs(world):
    s = WL.lj_fcc(seed=5, nc=10)
    h = lib.Handle(lib.FP64)
    h.lj(WL.LJ_EPS, WL.LJ_SIGMA, WL.LJ_CUTOFF)
    check(h, s, lib.MODEL_PAIR, world, WL.LJ_CUTOFF)


@pytest.mark.parametrize("world", [2, 3])
def test_smooth_slabs(world):
    s = WL.smooth_fcc(seed=2)
    h = lib.Handle(lib.FP64)
    h.smooth(WL.SMOOTH_A, WL.SMOOTH_CUTOFF)
    check(h, s, lib.MODEL_PAIR, world, WL.SMOOTH_CUTOFF)


def test_ace_slabs():
    m = read_resolved(G.generate_b2_model())
    s = WL.b2(seed=6, nc=8)
    h = lib.Handle(lib.FP64)
    h.ace(m)
    check(h, s, lib.MODEL_ACE, 2, 2.0 * m.cutoff)


def test_owned_count_validation():
    s = WL.smooth_fcc(seed=2)
    h = lib.Handle(lib.FP64)
    h.set_geometry(s.X, s.H, s.pbc, s.species)
    with pytest.raises(lib.ArgumentError):
        h.set_owned(len(s.species) + 1)
