"""ctypes binding of the CPU oracle (libpfw_oracle.so) — TEST INFRASTRUCTURE.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module.  It never stands in for the CUDA library.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libpfw_oracle.so")
_lib = None

REQ_E, REQ_F, REQ_V = 1, 2, 4


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


_simd = None


def lib_simd():
    """The timed CPU baseline's build (-O3 -march=native, SIMD lanes), compiled
    for this host on first use into a temporary directory (never shipped: the
    instruction set must be the running machine's)."""
    global _simd
    if _simd is None:
        import tempfile
        out = os.path.join(tempfile.gettempdir(), f"pfw_oracle_simd_{os.uname().nodename}_{os.getpid()}.so")
        flags = ["-O3", "-march=native", "-std=c++17", "-fPIC", "-ffp-contract=off", "-pthread", "-Wno-psabi", "-shared"]
        subprocess.run([os.environ.get("CXX", "g++"), *flags, "-o", out, os.path.join(HERE, "pfw_oracle.cpp")],
                       check=True, capture_output=True)
        _simd = _bind(C.CDLL(out))
    return _simd


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        _lib = _bind(C.CDLL(LIB))
    return _lib


def _bind(L):
    """Argument and result types of the oracle's C entry points."""
    dp, ip, i32p, u8p = C.POINTER(C.c_double), C.POINTER(C.c_int64), C.POINTER(C.c_int32), C.POINTER(C.c_uint8)
    L.pfo_last_error.restype = C.c_char_p
    L.pfo_pair_evaluate.argtypes = [C.c_int64, dp, dp, u8p, i32p, C.c_int32, C.c_int32, dp, C.c_double,
                                    C.c_int32, C.c_int32, C.c_uint32, C.c_int32, dp, dp, dp, ip]
    L.pfo_neighbour_list.argtypes = [C.c_int64, dp, dp, u8p, C.c_double, C.c_int32, C.c_int64, ip, i32p,
                                     i32p, dp, ip]
    L.pfo_ace_model_create.restype = C.c_void_p
    L.pfo_ace_model_create.argtypes = [C.c_void_p]
    L.pfo_ace_model_destroy.argtypes = [C.c_void_p]
    L.pfo_ace_evaluate.argtypes = [C.c_void_p, C.c_int64, dp, dp, u8p, i32p, C.c_int32, C.c_uint32, C.c_int32,
                                   dp, dp, dp, dp, dp]
    L.pfo_ace_set_scales.argtypes = [C.c_void_p, dp, dp]
    L.pfo_radial_ed.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_double, dp, dp]
    L.pfo_angular_ed.argtypes = [C.c_int32, dp, dp, dp]
    L.pfo_solid_ed.argtypes = [C.c_int32, dp, dp, dp]
    return L


class OracleError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"oracle error {code}: {msg}")
        self.code = code


def _check(rc):
    if rc != 0:
        raise OracleError(rc, lib().pfo_last_error().decode())


def _p(a, t):
    return None if a is None else a.ctypes.data_as(C.POINTER(t))


def _geom(X, H, pbc, species):
    X = np.ascontiguousarray(np.asarray(X, dtype=np.float64).reshape(-1, 3))
    H = np.asfortranarray(np.asarray(H, dtype=np.float64).reshape(3, 3)).ravel(order="F").copy()
    pbc = np.asarray([1 if b else 0 for b in pbc], dtype=np.uint8)
    sp = None if species is None else np.ascontiguousarray(species, dtype=np.int32)
    return X, H, pbc, sp


def pair_evaluate(X, H, pbc, species, kind, params, cutoff, *, width=4, brute_threshold=32,
                  request=7, nthreads=1, simd=False):
    """Restated evaluate!(Workspace(width, bruteforce_threshold), sys, p; request).

    X: (n,3) positions, H: 3×3 with columns = cell vectors, kind 'smooth'
    (params = symmetric nz×nz amplitudes) or 'lj' (params = (eps, sigma)).
    simd: the timed-baseline build with the W = 4 lanes as SIMD vectors.
    Returns (E, F (n,3), W (3,3), npairs)."""
    X, Hf, pbc, sp = _geom(X, H, pbc, species)
    n = X.shape[0]
    if sp is None:
        sp = np.zeros(n, np.int32)
    if kind == "smooth":
        A = np.ascontiguousarray(params, dtype=np.float64)
        k, nz = 0, A.shape[0]
    else:
        A = np.asarray(params, dtype=np.float64)
        k, nz = 1, 1
    E = np.zeros(1)
    F = np.zeros((n, 3))
    W = np.zeros(9)
    npairs = np.zeros(1, np.int64)
    L = lib_simd() if simd else lib()
    _check(L.pfo_pair_evaluate(n, _p(X, C.c_double), _p(Hf, C.c_double), _p(pbc, C.c_uint8),
                                   _p(sp, C.c_int32), k, nz, _p(A, C.c_double), float(cutoff), -4 if simd else width,
                                   brute_threshold, request, nthreads, _p(E, C.c_double), _p(F, C.c_double),
                                   _p(W, C.c_double), _p(npairs, C.c_int64)))
    return float(E[0]), F, W.reshape(3, 3, order="F"), int(npairs[0])


def neighbour_list(X, H, pbc, cutoff, *, brute_threshold=32):
    """Restated neighbour_list + neighbours: returns (offsets, j, S (M,3), R (M,3))."""
    X, Hf, pbc, _ = _geom(X, H, pbc, None)
    n = X.shape[0]
    total = np.zeros(1, np.int64)
    args = (n, _p(X, C.c_double), _p(Hf, C.c_double), _p(pbc, C.c_uint8), float(cutoff), brute_threshold)
    _check(lib().pfo_neighbour_list(*args, 0, None, None, None, None, _p(total, C.c_int64)))
    M = int(total[0])
    offs = np.zeros(n + 1, np.int64)
    j = np.zeros(M, np.int32)
    S = np.zeros((M, 3), np.int32)
    R = np.zeros((M, 3))
    _check(lib().pfo_neighbour_list(*args, M, _p(offs, C.c_int64), _p(j, C.c_int32), _p(S, C.c_int32),
                                    _p(R, C.c_double), _p(total, C.c_int64)))
    return offs, j, S, R


class AceOracle:
    """Restated ACE CPU executor on a PackedACE model."""

    def __init__(self, packed, radial_scale=None, pair_scale=None):
        """radial_scale [nR, nz, nz] / pair_scale [nQ, nz, nz]: the trainable
        scales ps.radial.scale / ps.pair.scale (ACE/serial.jl:12-17), applied
        to the radial values at run time as the reference does."""
        self.packed = packed
        self._t = packed.tables()
        self.handle = lib().pfo_ace_model_create(C.byref(self._t))
        if not self.handle:
            raise OracleError(1, lib().pfo_last_error().decode())
        if radial_scale is not None or pair_scale is not None:
            nz = packed.nz
            rs = None if radial_scale is None else np.asarray(radial_scale, np.float64).reshape(
                packed.radial.nchannels, nz, nz).ravel(order="F").copy()
            qs = None if pair_scale is None else np.asarray(pair_scale, np.float64).reshape(
                packed.pair.nchannels, nz, nz).ravel(order="F").copy()
            _check(lib().pfo_ace_set_scales(self.handle, _p(rs, C.c_double), _p(qs, C.c_double)))

    def __del__(self):
        if getattr(self, "handle", None) and _lib is not None:
            _lib.pfo_ace_model_destroy(self.handle)
            self.handle = None

    def evaluate(self, X, H, pbc, species, *, request=7, nthreads=1, brute_threshold=32,
                 site_energies=False, features=False):
        X, Hf, pbc, sp = _geom(X, H, pbc, species)
        n = X.shape[0]
        E = np.zeros(1)
        F = np.zeros((n, 3))
        W = np.zeros(9)
        es = np.zeros(n) if site_energies else None
        nfeat = self.packed.nz * (self.packed.nbasis + self.packed.pair.nchannels)
        feats = np.zeros((n, nfeat)) if features else None
        _check(lib().pfo_ace_evaluate(self.handle, n, _p(X, C.c_double), _p(Hf, C.c_double), _p(pbc, C.c_uint8),
                                      _p(sp, C.c_int32), brute_threshold, request, nthreads, _p(E, C.c_double),
                                      _p(F, C.c_double), _p(W, C.c_double), _p(es, C.c_double),
                                      _p(feats, C.c_double)))
        out = dict(energy=float(E[0]), forces=F, virial=W.reshape(3, 3, order="F"))
        if site_energies:
            out["site_energies"] = es
        if features:
            out["features"] = feats
        return out

    def radial_ed(self, family, iz, jz, r):
        fam = self.packed.radial if family == 0 else self.packed.pair
        v = np.zeros(fam.nchannels)
        d = np.zeros(fam.nchannels)
        _check(lib().pfo_radial_ed(self.handle, family, iz, jz, float(r), _p(v, C.c_double), _p(d, C.c_double)))
        return v, d


def angular_ed(lmax, d, solid=False):
    """BlockAngular values and Cartesian gradients; solid: r^l·Y_lm."""
    d = np.ascontiguousarray(d, dtype=np.float64)
    nY = (lmax + 1) ** 2
    Y = np.zeros(nY)
    dY = np.zeros((nY, 3))
    fn = lib().pfo_solid_ed if solid else lib().pfo_angular_ed
    _check(fn(lmax, _p(d, C.c_double), _p(Y, C.c_double), _p(dY, C.c_double)))
    return Y, dY
