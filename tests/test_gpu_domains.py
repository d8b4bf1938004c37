"""Slab domain decomposition of one periodic box (pfw_b200/parallel.py) on
one GPU: every domain evaluated in turn with pfw_set_owned, owned forces
assembled and energies/virials summed, must equal the single-box evaluation
(FP64, 1e-10 relative) for Lennard-Jones, SmoothPair and ACE, with 2 to 4
slabs.  The device-resident form (SlabPlan / SlabRank, bands selected by
pfw_slab_bands and assembled on the GPU) must give the same, with 1, 2 and
4 slabs, and its bands must equal the numpy selection."""
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


def exchange_check(h, s, model, world, halo):
    """The device-resident decomposition (SlabPlan / SlabRank): bands selected
    by pfw_slab_bands, exchanged by indexing, owned + ghosts assembled on the
    device; every rank in turn on this GPU."""
    import ctypes

    import torch
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(device=dev)  # the library and torch in one stream
    h.set_stream(ctypes.c_void_p(stream.cuda_stream))
    try:
        with torch.cuda.stream(stream):
            h.set_geometry(s.X, s.H, s.pbc, s.species)
            E0, F0, W0 = h.evaluate(model, 7)
            plan = PAR.SlabPlan(s, world, halo)
            assert sorted(np.concatenate(plan.owned).tolist()) == list(range(len(s.species)))
            ranks = [PAR.SlabRank(h, plan, r, dev) for r in range(world)]
            E = torch.zeros(1, dtype=torch.float64, device=dev)
            W = torch.zeros(9, dtype=torch.float64, device=dev)
            F = torch.zeros((3 * len(s.species), 3), dtype=torch.float64, device=dev)
            Ex, Fx, Wx = PAR.slab_step_local(ranks, E, F, W, model)
            # a second step on the same buffers gives the same result (scratch reuse)
            Ey, Fy, Wy = PAR.slab_step_local(ranks, E, F, W, model)
    finally:
        torch.cuda.synchronize(dev)
        h.set_stream(None)
    assert Ex == Ey and np.array_equal(Fx, Fy) and np.array_equal(Wx, Wy)
    assert abs(Ex - E0) <= 1e-10 * max(1.0, abs(E0))
    assert close(Fx, F0) and close(Wx, W0)


@pytest.mark.parametrize("world", [1, 2, 4])
def test_lj_slab_exchange_on_device(world):
    s = WL.lj_fcc(seed=5, nc=10)
    h = lib.Handle(lib.FP64)
    h.lj(WL.LJ_EPS, WL.LJ_SIGMA, WL.LJ_CUTOFF)
    exchange_check(h, s, lib.MODEL_PAIR, world, WL.LJ_CUTOFF)


def test_ace_slab_exchange_on_device():
    m = read_resolved(G.generate_b2_model())
    s = WL.b2(seed=6, nc=8)
    h = lib.Handle(lib.FP64)
    h.ace(m)
    exchange_check(h, s, lib.MODEL_ACE, 2, 2.0 * m.cutoff)


def test_slab_bands_match_numpy_selection():
    import ctypes

    import torch
    s = WL.lj_fcc(seed=8, nc=8)
    plan = PAR.SlabPlan(s, 3, WL.LJ_CUTOFF)
    h = lib.Handle(lib.FP64)
    dev = torch.device("cuda", 0)
    for r in range(3):
        rk = PAR.SlabRank(h, plan, r, dev)
        c = rk.bands()
        torch.cuda.synchronize(dev)  # the library's own stream
        c = c.cpu().numpy()
        X = plan.X[plan.owned[r]]
        f = X @ plan.frac_row
        lo, hi = plan.bounds(r)
        sl, su = plan.shifts(r)
        for band, sel, sh, k in ((rk.lower, f < lo + plan.d, sl, 0), (rk.upper, f >= hi - plan.d, su, 1)):
            assert c[k] == sel.sum()
            got = band[: c[k]].cpu().numpy()
            assert np.allclose(got[:, :3], X[sel] + sh, rtol=0, atol=1e-12)
            assert np.array_equal(got[:, 3], plan.species[plan.owned[r]][sel])
    with pytest.raises(lib.ArgumentError):
        h.slab_bands(4, ctypes.c_void_p(0), ctypes.c_void_p(0), plan.frac_row, 0.5, 0.25, 0.1, sl, su,
                     ctypes.c_void_p(0), ctypes.c_void_p(0), ctypes.c_void_p(0))
