"""pfw_pair_evaluate_noalloc, the entry point for callers that cannot call
cudaMalloc (a host runtime that owns all device memory through its own pool,
or code that must not trigger an allocation's device-wide synchronisation).

It is checked through the C ABI against the ordinary entry point
(pfw_evaluate, which allocates its workspace) on the same systems, twice in
a row, since consecutive calls share the library's static scratch array.
Errors that depend on the data arrive through the device status word; the
argument checks return before anything is queued.  This file is collected
last so that a run stopping at the first failure has already run every other
test; it also passes when run alone.
"""
import ctypes

import numpy as np
import pytest

from pfw_b200 import lib
from pfw_b200 import workloads as WL

pytestmark = pytest.mark.gpu
RTOL = 1e-10
dp = ctypes.POINTER(ctypes.c_double)
u8p = ctypes.POINTER(ctypes.c_uint8)


def noalloc_fn():
    L = lib.load()
    f = L.pfw_pair_evaluate_noalloc
    f.argtypes = [ctypes.c_int32, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p, dp, u8p,
                  ctypes.c_int32, ctypes.c_int32, dp, ctypes.c_double, ctypes.c_uint32, ctypes.c_void_p,
                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int32]
    f.restype = ctypes.c_int
    return f


def host_args(s, params, kind):
    Hf = np.asarray(s.H, dtype=np.float64).ravel(order="F").copy()
    pb = np.array([1 if b else 0 for b in s.pbc], np.uint8)
    prm = np.ascontiguousarray(params, dtype=np.float64).ravel()
    nz = int(round(np.sqrt(prm.size))) if kind == 0 else 1
    return Hf, pb, prm, nz


def call_noalloc(s, kind, params, cutoff, request=7, with_forces=True):
    """Returns (rc, status, E, F, W); status is the device status word."""
    import torch
    f = noalloc_fn()
    dev = torch.device("cuda", 0)
    X = torch.from_numpy(np.ascontiguousarray(s.X)).to(dev)
    sp = torch.from_numpy(np.ascontiguousarray(s.species, dtype=np.int32)).to(dev)
    E = torch.full((1,), np.nan, dtype=torch.float64, device=dev)
    F = torch.full((max(len(s), 1), 3), np.nan, dtype=torch.float64, device=dev)
    W = torch.full((9,), np.nan, dtype=torch.float64, device=dev)
    status = torch.full((1,), -1, dtype=torch.int32, device=dev)
    Hf, pb, prm, nz = host_args(s, params, kind)
    err = ctypes.create_string_buffer(256)
    stream = torch.cuda.current_stream(dev).cuda_stream
    rc = f(0, ctypes.c_void_p(stream), len(s), ctypes.c_void_p(X.data_ptr()), ctypes.c_void_p(sp.data_ptr()),
           Hf.ctypes.data_as(dp), pb.ctypes.data_as(u8p), kind, nz, prm.ctypes.data_as(dp), float(cutoff), request,
           ctypes.c_void_p(E.data_ptr()), ctypes.c_void_p(F.data_ptr()) if with_forces else None,
           ctypes.c_void_p(W.data_ptr()), ctypes.c_void_p(status.data_ptr()), err, 256)
    torch.cuda.synchronize()
    return (rc, int(status.item()), float(E.item()), F.cpu().numpy()[: len(s)],
            W.cpu().numpy().reshape(3, 3, order="F"), err.value)


def call_allocating(s, kind, params, cutoff):
    h = lib.Handle(lib.FP64)
    h.set_geometry(s.X, s.H, s.pbc, s.species)
    if kind == 0:
        h.smooth(params, cutoff)
    else:
        h.lj(params[0], params[1], cutoff)
    out = h.evaluate(lib.MODEL_PAIR, 7)
    h.close()
    return out


def assert_close(a, b):
    E, F, W = a
    Eo, Fo, Wo = b
    assert abs(E - Eo) <= RTOL * max(1.0, abs(Eo))
    if Fo.size:
        assert np.abs(F - Fo).max() <= RTOL * max(1e-300, np.abs(Fo).max()) + 1e-12
    assert np.abs(W - Wo).max() <= RTOL * max(1.0, np.abs(Wo).max())


def two_species_slab():
    """Two species, one open axis (z), positions spread over the slab."""
    s = WL.smooth_fcc(seed=11, nc=6)
    s.X[:, 2] *= 1.7  # stretch along the open axis
    return WL.System(s.X, np.diag([9.6, 9.6, 1.0]), (True, True, False), s.species, "slab")


CASES = {
    "smooth_fcc": lambda: (WL.smooth_fcc(seed=3), 0, WL.SMOOTH_A, WL.SMOOTH_CUTOFF),
    "lj_fcc": lambda: (WL.lj_fcc(nc=8, seed=4), 1, np.array([WL.LJ_EPS, WL.LJ_SIGMA]), WL.LJ_CUTOFF),
    "smooth_two_species_slab": lambda: (two_species_slab(), 0, WL.SMOOTH_A, WL.SMOOTH_CUTOFF),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_noalloc_matches_allocating_entry_point_twice(case):
    s, kind, params, c = CASES[case]()
    ref = call_allocating(s, kind, params, c)
    for _ in range(2):
        rc, status, E, F, W, err = call_noalloc(s, kind, params, c)
        assert rc == 0, err.decode()
        assert status == lib.OK
        assert_close((E, F, W), ref)


def test_noalloc_empty_system_has_zero_energy_and_virial():
    s = WL.System(np.zeros((0, 3)), np.diag([10.0, 10.0, 10.0]), (True, True, True), np.zeros(0, np.int32))
    rc, status, E, F, W, err = call_noalloc(s, 0, WL.SMOOTH_A, WL.SMOOTH_CUTOFF)
    assert rc == 0 and status == lib.OK
    assert E == 0.0 and np.all(W == 0.0)


def test_noalloc_reports_species_outside_the_model():
    s = WL.smooth_fcc(seed=5)
    s.species[17] = 2  # the amplitude table has channels 0 and 1
    rc, status, *_ = call_noalloc(s, 0, WL.SMOOTH_A, WL.SMOOTH_CUTOFF)
    assert rc == 0 and status == lib.EINVAL
    # the next call on valid data reads OK again (the status word is cleared per call)
    s.species[17] = 1
    rc, status, *_ = call_noalloc(s, 0, WL.SMOOTH_A, WL.SMOOTH_CUTOFF)
    assert rc == 0 and status == lib.OK


def test_noalloc_reports_coincident_lennard_jones_atoms():
    s = WL.System(np.array([[1.0, 2.0, 3.0], [1.0, 2.0, 3.0], [5.0, 5.0, 5.0]]), np.diag([30.0, 30.0, 30.0]),
                  (True, True, True), np.zeros(3, np.int32))
    rc, status, *_ = call_noalloc(s, 1, np.array([WL.LJ_EPS, WL.LJ_SIGMA]), WL.LJ_CUTOFF)
    assert rc == 0 and status == lib.EDOMAIN


def rejected(s, kind, params, cutoff, request=7, with_forces=True):
    """Argument errors return before any device work: no device memory needed."""
    f = noalloc_fn()
    Hf, pb, prm, nz = host_args(s, params, kind)
    err = ctypes.create_string_buffer(256)
    fake = ctypes.c_void_p(16)  # never dereferenced: the call must return first
    rc = f(0, None, len(s), fake, fake, Hf.ctypes.data_as(dp), pb.ctypes.data_as(u8p), kind, nz,
           prm.ctypes.data_as(dp), float(cutoff), request, fake, fake if with_forces else None, fake, None, err, 256)
    return rc, err.value


def test_noalloc_rejects_bad_arguments_before_queueing_work():
    s = WL.smooth_fcc()
    rc, msg = rejected(s, 0, WL.SMOOTH_A, WL.SMOOTH_CUTOFF, with_forces=False)
    assert rc == lib.EINVAL and b"force buffer" in msg
    rc, msg = rejected(s, 0, np.array([[1.0, 0.7], [0.6, 1.3]]), WL.SMOOTH_CUTOFF)
    assert rc == lib.EINVAL and b"symmetric" in msg
    sheared = WL.System(s.X, np.array([[12.8, 2.0, 0.0], [0.0, 12.8, 0.0], [0.0, 0.0, 12.8]]), s.pbc, s.species)
    rc, msg = rejected(sheared, 0, WL.SMOOTH_A, WL.SMOOTH_CUTOFF)
    assert rc == lib.EINVAL and b"orthorhombic" in msg
    short = WL.System(s.X, np.diag([12.8, 3.9, 12.8]), s.pbc, s.species)
    rc, msg = rejected(short, 0, WL.SMOOTH_A, WL.SMOOTH_CUTOFF)
    assert rc == lib.EINVAL and b"twice the cutoff" in msg


def test_noalloc_rejects_oversize_system():
    f = noalloc_fn()
    n = 8193
    H = np.diag([100.0, 100.0, 100.0]).ravel(order="F").copy()
    pb = np.ones(3, np.uint8)
    prm = np.ones(1)
    err = ctypes.create_string_buffer(256)
    rc = f(0, None, n, None, None, H.ctypes.data_as(dp), pb.ctypes.data_as(u8p), 0, 1, prm.ctypes.data_as(dp),
           2.0, 7, None, None, None, None, err, 256)
    assert rc == lib.EINVAL
    assert b"8192" in err.value


def test_noalloc_leaves_the_current_device_alone():
    import torch
    before = torch.cuda.current_device()
    s, kind, params, c = CASES["smooth_fcc"]()
    rc, status, *_ = call_noalloc(s, kind, params, c)
    assert rc == 0 and status == lib.OK
    assert torch.cuda.current_device() == before
