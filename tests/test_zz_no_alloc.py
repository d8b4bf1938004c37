"""pfw_pair_evaluate_noalloc, the entry point for callers that cannot call
cudaMalloc (a host runtime that owns all device memory through its own pool,
or code that must not trigger an allocation's device-wide synchronisation).

It is checked through the C ABI against the ordinary entry point
(pfw_evaluate, which allocates its workspace) on the same systems, twice in
a row, since consecutive calls share the library's static scratch array.
This file is collected last so that a run stopping at the first failure has
already run every other test; it also passes when run alone.
"""
import ctypes

import numpy as np
import pytest

from pfw_b200 import lib
from pfw_b200 import workloads as WL

pytestmark = pytest.mark.gpu
RTOL = 1e-10


def noalloc_fn():
    L = lib.load()
    f = L.pfw_pair_evaluate_noalloc
    f.argtypes = [ctypes.c_int32, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p,
                  ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_uint8), ctypes.c_int32, ctypes.c_int32,
                  ctypes.POINTER(ctypes.c_double), ctypes.c_double, ctypes.c_uint32, ctypes.c_void_p,
                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int32]
    f.restype = ctypes.c_int
    return f


def call_noalloc(s, kind, params, cutoff):
    import torch
    f = noalloc_fn()
    dev = torch.device("cuda", 0)
    X = torch.from_numpy(np.ascontiguousarray(s.X)).to(dev)
    sp = torch.from_numpy(np.ascontiguousarray(s.species, dtype=np.int32)).to(dev)
    E = torch.full((1,), np.nan, dtype=torch.float64, device=dev)
    F = torch.full((len(s), 3), np.nan, dtype=torch.float64, device=dev)
    W = torch.full((9,), np.nan, dtype=torch.float64, device=dev)
    Hf = np.asarray(s.H, dtype=np.float64).ravel(order="F").copy()
    pb = np.array([1 if b else 0 for b in s.pbc], np.uint8)
    prm = np.ascontiguousarray(params, dtype=np.float64).ravel()
    nz = int(round(np.sqrt(prm.size))) if kind == 0 else 1
    err = ctypes.create_string_buffer(256)
    stream = torch.cuda.current_stream(dev).cuda_stream
    rc = f(0, ctypes.c_void_p(stream), len(s), ctypes.c_void_p(X.data_ptr()), ctypes.c_void_p(sp.data_ptr()),
           Hf.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), pb.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)),
           kind, nz, prm.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
           float(cutoff), 7, ctypes.c_void_p(E.data_ptr()), ctypes.c_void_p(F.data_ptr()),
           ctypes.c_void_p(W.data_ptr()), err, 256)
    torch.cuda.synchronize()
    assert rc == 0, err.value.decode()
    return float(E.item()), F.cpu().numpy(), W.cpu().numpy().reshape(3, 3, order="F")


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
    assert np.abs(F - Fo).max() <= RTOL * max(1e-300, np.abs(Fo).max()) + 1e-12
    assert np.abs(W - Wo).max() <= RTOL * max(1.0, np.abs(Wo).max())


@pytest.mark.parametrize("case", ["smooth_fcc", "lj_fcc"])
def test_noalloc_matches_allocating_entry_point_twice(case):
    if case == "smooth_fcc":
        s, kind, params, c = WL.smooth_fcc(seed=3), 0, WL.SMOOTH_A, WL.SMOOTH_CUTOFF
    else:
        s, kind, params, c = WL.lj_fcc(nc=8, seed=4), 1, np.array([WL.LJ_EPS, WL.LJ_SIGMA]), WL.LJ_CUTOFF
    ref = call_allocating(s, kind, params, c)
    first = call_noalloc(s, kind, params, c)
    second = call_noalloc(s, kind, params, c)
    assert_close(first, ref)
    assert_close(second, ref)


def test_noalloc_rejects_oversize_system():
    f = noalloc_fn()
    n = 8193
    H = np.diag([100.0, 100.0, 100.0]).ravel(order="F").copy()
    pb = np.ones(3, np.uint8)
    prm = np.ones(1)
    err = ctypes.create_string_buffer(256)
    rc = f(0, None, n, None, None, H.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
           pb.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), 0, 1, prm.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
           2.0, 7, None, None, None, err, 256)
    assert rc == lib.EINVAL
    assert b"8192" in err.value
