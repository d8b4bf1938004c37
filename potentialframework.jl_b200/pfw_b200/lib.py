"""ctypes binding of libpfw_b200.so (the C ABI declared in include/pfw_b200.h).

The library is built in-tree (potentialframework.jl_b200/lib/).  Loading
fails loudly when it is missing or when no CUDA device is present: there is
no CPU fallback anywhere in the product path.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .ace_model import pfw_ace_tables

PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBPATH = os.path.join(PKG, "lib", "libpfw_b200.so")

from .errors import (ECAPACITY, ECUDA, EDOMAIN, EINVAL, ESHAPE, ESTATE, ETIMEDOUT, OK,  # noqa: F401
                     ArgumentError, DimensionMismatch, DomainError, PFWError)
REQ_E, REQ_F, REQ_V = 1, 2, 4
FP64, MIXED = 0, 1
MODEL_PAIR, MODEL_ACE, MODEL_SURROGATE = 0, 1, 2


class pfw_options(C.Structure):
    _fields_ = [("precision", C.c_int32), ("bruteforce_threshold", C.c_int32), ("device", C.c_int32),
                ("reserved", C.c_int32)]


_ERRORS = {EINVAL: ArgumentError, EDOMAIN: DomainError, ESHAPE: DimensionMismatch}
_lib = None

dp = C.POINTER(C.c_double)
i32p = C.POINTER(C.c_int32)
i64p = C.POINTER(C.c_int64)
u8p = C.POINTER(C.c_uint8)
vp = C.c_void_p


def load():
    """Load the CUDA library (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIBPATH):
        raise RuntimeError(f"libpfw_b200.so not built: run `python -m pfw_b200.build` in {PKG}")
    L = C.CDLL(LIBPATH)
    L.pfw_version.restype = C.c_char_p
    L.pfw_ws_create.argtypes = [C.POINTER(pfw_options), C.POINTER(vp)]
    L.pfw_ws_destroy.argtypes = [vp]
    L.pfw_ws_destroy.restype = None
    L.pfw_last_error.argtypes = [vp]
    L.pfw_last_error.restype = C.c_char_p
    L.pfw_set_geometry.argtypes = [vp, C.c_int64, dp, dp, u8p, i32p]
    L.pfw_set_geometry_device.argtypes = [vp, C.c_int64, vp, dp, u8p, vp]
    L.pfw_pair_model_smooth.argtypes = [vp, C.c_int32, dp, C.c_double]
    L.pfw_pair_model_lj.argtypes = [vp, C.c_double, C.c_double, C.c_double]
    L.pfw_ace_model_load.argtypes = [vp, C.POINTER(pfw_ace_tables)]
    L.pfw_ace_set_schedule.argtypes = [vp, C.c_int32, C.c_int32]
    L.pfw_evaluate.argtypes = [vp, C.c_int32, C.c_uint32, dp, dp, dp]
    L.pfw_evaluate_device.argtypes = [vp, C.c_int32, C.c_uint32, vp, vp, vp]
    L.pfw_site_energies.argtypes = [vp, dp]
    L.pfw_last_pair_count.argtypes = [vp, i64p]
    L.pfw_neighbour_count.argtypes = [vp, C.c_double, i64p]
    L.pfw_neighbour_fill.argtypes = [vp, i64p, i32p, i32p, dp]
    L.pfw_probe_fp64_peak.argtypes = [vp, dp]
    L.pfw_launch_count.argtypes = [vp]
    L.pfw_launch_count.restype = C.c_uint64
    L.pfw_set_stream.argtypes = [vp, vp]
    L.pfw_set_diagnostics.argtypes = [vp, C.c_int32]
    L.pfw_stage_times.argtypes = [vp, dp, C.c_int32]
    L.pfw_stage_times.restype = C.c_int32
    L.pfw_set_batch.argtypes = [vp, C.c_int32, i64p, dp, dp, u8p, i32p]
    L.pfw_set_batch_device.argtypes = [vp, C.c_int32, i64p, vp, dp, u8p, vp]
    L.pfw_batch_update_positions.argtypes = [vp, vp, C.c_int32]
    L.pfw_ace_feature_count.argtypes = [vp, i32p]
    L.pfw_ace_design_shape.argtypes = [vp, i64p, i64p]
    L.pfw_ace_design_matrix.argtypes = [vp, dp, C.c_int64, C.c_int64, dp]
    L.pfw_ace_design_matrix_device.argtypes = [vp, vp, C.c_int64, C.c_int64, vp]
    L.pfw_evaluate_batch.argtypes = [vp, C.c_int32, C.c_uint32, dp, dp, dp, dp]
    L.pfw_evaluate_batch_device.argtypes = [vp, C.c_int32, C.c_uint32, vp, vp, vp, vp]
    L.pfw_batch_graph_launch.argtypes = [vp, C.c_uint32, vp, vp, vp, vp]
    L.pfw_batch_graph_sync.argtypes = [vp]
    L.pfw_set_owned.argtypes = [vp, C.c_int64]
    L.pfw_slab_bands.argtypes = [vp, C.c_int64, vp, vp, dp, C.c_double, C.c_double, C.c_double, dp, dp, vp, vp, vp]
    L.pfw_pair_set_skin.argtypes = [vp, C.c_double]
    L.pfw_pair_skin_stats.argtypes = [vp, i64p, i64p]
    L.pfw_surrogate_load.argtypes = [vp, C.POINTER(pfw_ace_tables), vp]
    L.pfw_surrogate_features.argtypes = [vp, dp]
    L.pfw_surrogate_stats.argtypes = [vp, i64p, i64p]
    L.pfw_mlp_param_grad.argtypes = [vp, vp, C.POINTER(C.c_float), C.c_int64, C.POINTER(C.c_float),
                                     C.POINTER(C.c_float), i32p, dp, C.POINTER(C.c_float)]
    L.pfw_mlp_train.argtypes = [vp, vp, C.POINTER(C.c_float), C.c_int64, C.POINTER(C.c_float),
                                C.POINTER(C.c_float), i32p, vp, C.POINTER(C.c_float)]
    L.pfw_mlp_ef_step.argtypes = [vp, vp, vp, vp, vp, C.c_int64, vp, vp, i32p, vp, vp, C.c_float, C.c_float,
                                  C.c_int64, vp, dp]
    L.pfw_mlp_input_grad.argtypes = [vp, vp, vp, C.c_int64, vp, i32p, vp]
    L.pfw_surrogate_pullback.argtypes = [vp, vp, vp]
    _lib = L
    return L


def ptr(a, t):
    return None if a is None else a.ctypes.data_as(C.POINTER(t))


class Handle:
    """Owns one pfw_ws (one per host thread; not reentrant)."""

    def __init__(self, precision=FP64, bruteforce_threshold=32, device=0):
        L = load()
        opt = pfw_options(int(precision), int(bruteforce_threshold), int(device), 0)
        h = vp()
        rc = L.pfw_ws_create(C.byref(opt), C.byref(h))
        if rc != OK:
            raise PFWError(rc, "pfw_ws_create failed (no CUDA device, or invalid options)")
        self.ws = h
        self.L = L
        self.device = int(device)

    def check(self, rc):
        if rc != OK:
            msg = self.L.pfw_last_error(self.ws).decode()
            raise _ERRORS.get(rc, PFWError)(rc, msg)

    def close(self):
        if getattr(self, "ws", None):
            self.L.pfw_ws_destroy(self.ws)
            self.ws = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def launches(self):
        return int(self.L.pfw_launch_count(self.ws))

    # --- thin wrappers ---------------------------------------------------
    def set_geometry(self, X, H, pbc, species):
        X = np.ascontiguousarray(X, dtype=np.float64).reshape(-1, 3)
        Hf = np.asarray(H, dtype=np.float64).reshape(3, 3).ravel(order="F").copy()
        pb = np.array([1 if b else 0 for b in pbc], dtype=np.uint8)
        sp = np.ascontiguousarray(species, dtype=np.int32)
        self.check(self.L.pfw_set_geometry(self.ws, X.shape[0], ptr(X, C.c_double), ptr(Hf, C.c_double),
                                           ptr(pb, C.c_uint8), ptr(sp, C.c_int32)))
        self.n = X.shape[0]

    def set_geometry_device(self, n, X_dev_ptr, H, pbc, species_dev_ptr):
        Hf = np.asarray(H, dtype=np.float64).reshape(3, 3).ravel(order="F").copy()
        pb = np.array([1 if b else 0 for b in pbc], dtype=np.uint8)
        self.check(self.L.pfw_set_geometry_device(self.ws, int(n), X_dev_ptr, ptr(Hf, C.c_double),
                                                  ptr(pb, C.c_uint8), species_dev_ptr))
        self.n = int(n)

    def set_owned(self, n_owned):
        self.check(self.L.pfw_set_owned(self.ws, int(n_owned)))

    def slab_bands(self, n, X_ptr, species_ptr, frac_row, lo, hi, d, shift_lower, shift_upper, lower_ptr,
                   upper_ptr, counts_ptr):
        """pfw_slab_bands on device buffers (pointers); queued on the workspace's stream."""
        fr = np.ascontiguousarray(frac_row, dtype=np.float64).reshape(3)
        sl = np.ascontiguousarray(shift_lower, dtype=np.float64).reshape(3)
        su = np.ascontiguousarray(shift_upper, dtype=np.float64).reshape(3)
        self.check(self.L.pfw_slab_bands(self.ws, int(n), X_ptr, species_ptr, ptr(fr, C.c_double), float(lo),
                                         float(hi), float(d), ptr(sl, C.c_double), ptr(su, C.c_double), lower_ptr,
                                         upper_ptr, counts_ptr))

    def pair_skin(self, skin):
        self.check(self.L.pfw_pair_set_skin(self.ws, float(skin)))

    def skin_stats(self):
        a = np.zeros(2, np.int64)
        self.check(self.L.pfw_pair_skin_stats(self.ws, ptr(a[:1], C.c_int64), ptr(a[1:], C.c_int64)))
        return int(a[0]), int(a[1])

    def smooth(self, A, cutoff):
        A = np.ascontiguousarray(A, dtype=np.float64)
        self.check(self.L.pfw_pair_model_smooth(self.ws, A.shape[0], ptr(A, C.c_double), float(cutoff)))

    def lj(self, eps, sigma, cutoff):
        self.check(self.L.pfw_pair_model_lj(self.ws, float(eps), float(sigma), float(cutoff)))

    def ace(self, packed):
        self._ace_tables = packed.tables()
        self._ace_packed = packed
        self.check(self.L.pfw_ace_model_load(self.ws, C.byref(self._ace_tables)))

    def ace_schedule(self, chunk=0, groups=0):
        self.check(self.L.pfw_ace_set_schedule(self.ws, int(chunk), int(groups)))

    def evaluate(self, model=MODEL_PAIR, request=7):
        E = np.zeros(1)
        W = np.zeros(9)
        F = np.zeros((self.n, 3)) if request & REQ_F else None
        self.check(self.L.pfw_evaluate(self.ws, model, request, ptr(E, C.c_double), ptr(F, C.c_double),
                                       ptr(W, C.c_double)))
        return float(E[0]), F, W.reshape(3, 3, order="F")

    def evaluate_device(self, model, request, E_ptr, F_ptr, W_ptr):
        self.check(self.L.pfw_evaluate_device(self.ws, model, request, E_ptr, F_ptr, W_ptr))

    def site_energies(self):
        e = np.zeros(self.n)
        self.check(self.L.pfw_site_energies(self.ws, ptr(e, C.c_double)))
        return e

    def pair_count(self):
        v = np.zeros(1, np.int64)
        self.check(self.L.pfw_last_pair_count(self.ws, ptr(v, C.c_int64)))
        return int(v[0])

    def neighbour_list(self, cutoff):
        tot = np.zeros(1, np.int64)
        self.check(self.L.pfw_neighbour_count(self.ws, float(cutoff), ptr(tot, C.c_int64)))
        M = int(tot[0])
        offs = np.zeros(self.n + 1, np.int64)
        j = np.zeros(M, np.int32)
        S = np.zeros((M, 3), np.int32)
        R = np.zeros((M, 3))
        self.check(self.L.pfw_neighbour_fill(self.ws, ptr(offs, C.c_int64), ptr(j, C.c_int32), ptr(S, C.c_int32),
                                             ptr(R, C.c_double)))
        return offs, j, S, R

    # --- batches of independent systems --------------------------------
    @staticmethod
    def _batch_arrays(systems):
        offs = np.zeros(len(systems) + 1, np.int64)
        offs[1:] = np.cumsum([len(s.species) for s in systems])
        H = np.concatenate([np.asarray(s.H, np.float64).reshape(3, 3).ravel(order="F") for s in systems])
        pbc = np.array([[1 if b else 0 for b in s.pbc] for s in systems], np.uint8).ravel()
        return offs, H, pbc

    def set_batch(self, systems):
        """systems: sequence of workloads.System-like objects (X n×3, H with columns = cell vectors, pbc, species)."""
        offs, H, pbc = self._batch_arrays(systems)
        X = np.ascontiguousarray(np.concatenate([np.asarray(s.X, np.float64).reshape(-1, 3) for s in systems]))
        sp = np.ascontiguousarray(np.concatenate([np.asarray(s.species, np.int32) for s in systems]))
        self.check(self.L.pfw_set_batch(self.ws, len(systems), ptr(offs, C.c_int64), ptr(X, C.c_double),
                                        ptr(H, C.c_double), ptr(pbc, C.c_uint8), ptr(sp, C.c_int32)))
        self.n = int(offs[-1])
        self.nsys = len(systems)
        self.batch_offsets = offs

    def set_batch_device(self, systems, X_dev_ptr, species_dev_ptr):
        offs, H, pbc = self._batch_arrays(systems)
        self.check(self.L.pfw_set_batch_device(self.ws, len(systems), ptr(offs, C.c_int64), X_dev_ptr,
                                               ptr(H, C.c_double), ptr(pbc, C.c_uint8), species_dev_ptr))
        self.n = int(offs[-1])
        self.nsys = len(systems)
        self.batch_offsets = offs

    def batch_update_positions(self, X=None, X_dev_ptr=None):
        if X_dev_ptr is not None:
            self.check(self.L.pfw_batch_update_positions(self.ws, X_dev_ptr, 1))
        else:
            X = np.ascontiguousarray(X, dtype=np.float64).reshape(-1, 3)
            self.check(self.L.pfw_batch_update_positions(self.ws, X.ctypes.data, 0))

    def feature_count(self):
        v = np.zeros(1, np.int32)
        self.check(self.L.pfw_ace_feature_count(self.ws, ptr(v, C.c_int32)))
        return int(v[0])

    def design_shape(self):
        r = np.zeros(2, np.int64)
        self.check(self.L.pfw_ace_design_shape(self.ws, ptr(r[:1], C.c_int64), ptr(r[1:], C.c_int64)))
        return int(r[0]), int(r[1])

    def design_matrix(self):
        """Stacked design rows [rows × cols] of the current geometry or batch
        and the per-system reference-energy baselines [nsys]."""
        rows, cols = self.design_shape()
        A = np.zeros((rows, cols))
        nsys = (rows - 3 * self.n) // 10
        base = np.zeros(max(nsys, 1))
        self.check(self.L.pfw_ace_design_matrix(self.ws, ptr(A, C.c_double), cols, rows, ptr(base, C.c_double)))
        return A, base[:nsys]

    def design_matrix_device(self, A_ptr, ld, rows_capacity, base_ptr=None):
        self.check(self.L.pfw_ace_design_matrix_device(self.ws, A_ptr, ld, rows_capacity, base_ptr))

    def evaluate_batch(self, model=MODEL_ACE, request=7, features=False):
        """Per-system E [nsys], F [N×3], W [nsys×3×3] and (ACE) fitting features [nsys×nfeat]."""
        E = np.zeros(self.nsys)
        W = np.zeros((self.nsys, 9))
        F = np.zeros((self.n, 3)) if request & REQ_F else None
        X = np.zeros((self.nsys, self.feature_count())) if features else None
        self.check(self.L.pfw_evaluate_batch(self.ws, model, request, ptr(E, C.c_double), ptr(F, C.c_double),
                                             ptr(W, C.c_double), ptr(X, C.c_double)))
        return E, F, W.reshape(self.nsys, 3, 3).transpose(0, 2, 1), X

    def evaluate_batch_device(self, model, request, E_ptr, F_ptr, W_ptr, feat_ptr=None):
        self.check(self.L.pfw_evaluate_batch_device(self.ws, model, request, E_ptr, F_ptr, W_ptr, feat_ptr))

    def batch_graph_launch(self, request, E_ptr, F_ptr, W_ptr, feat_ptr=None):
        self.check(self.L.pfw_batch_graph_launch(self.ws, request, E_ptr, F_ptr, W_ptr, feat_ptr))

    def batch_graph_sync(self):
        self.check(self.L.pfw_batch_graph_sync(self.ws))

    def set_stream(self, stream_ptr):
        self.check(self.L.pfw_set_stream(self.ws, stream_ptr))

    # --- learned surrogate ----------------------------------------------
    def surrogate(self, feature_model, sur=None, tau=None):
        """Load the feature model and (optionally) a trained surrogate.Surrogate."""
        self._sur_tables = feature_model.tables()
        self._sur_model = feature_model
        self._sur_struct = sur.mlp_struct(tau) if sur is not None else None
        arg = C.byref(self._sur_struct) if sur is not None else None
        self.check(self.L.pfw_surrogate_load(self.ws, C.byref(self._sur_tables), arg))
        self.sur_nin = feature_model.nbasis + feature_model.pair.nchannels

    def surrogate_features(self):
        out = np.zeros((self.n, self.sur_nin))
        self.check(self.L.pfw_surrogate_features(self.ws, ptr(out, C.c_double)))
        return out

    def surrogate_stats(self):
        a = np.zeros(2, np.int64)
        self.check(self.L.pfw_surrogate_stats(self.ws, ptr(a[:1], C.c_int64), ptr(a[1:], C.c_int64)))
        return int(a[0]), int(a[1])

    def _mlp_shape(self, P, nin):
        from .surrogate import HIDDEN, pfw_mlp_shape
        nz, M, _ = P.shape
        self._shape = pfw_mlp_shape(nz, M, nin, HIDDEN)
        return self._shape

    def mlp_param_grad(self, P, X, y, Z):
        P = np.ascontiguousarray(P, np.float32)
        X = np.ascontiguousarray(X, np.float32)
        y = np.ascontiguousarray(y, np.float32)
        Z = np.ascontiguousarray(Z, np.int32)
        shape = self._mlp_shape(P, X.shape[1])
        loss = np.zeros(P.shape[0] * P.shape[1])
        grad = np.zeros_like(P)
        self.check(self.L.pfw_mlp_param_grad(self.ws, C.byref(shape), ptr(P, C.c_float), len(y), ptr(X, C.c_float),
                                             ptr(y, C.c_float), ptr(Z, C.c_int32), ptr(loss, C.c_double),
                                             ptr(grad, C.c_float)))
        return loss.reshape(P.shape[:2]), grad

    def mlp_train(self, P, X, y, Z, *, epochs, batch, lr, lr_final, seed):
        """Train in place (P: FP32 [nz, M, nparams]); returns the per-epoch mean loss."""
        from .surrogate import pfw_mlp_train_options
        assert P.dtype == np.float32 and P.flags.c_contiguous
        X = np.ascontiguousarray(X, np.float32)
        y = np.ascontiguousarray(y, np.float32)
        Z = np.ascontiguousarray(Z, np.int32)
        shape = self._mlp_shape(P, X.shape[1])
        opt = pfw_mlp_train_options(int(epochs), int(batch), float(lr), float(lr_final), int(seed))
        hist = np.zeros(int(epochs), np.float32)
        self.check(self.L.pfw_mlp_train(self.ws, C.byref(shape), ptr(P, C.c_float), len(y), ptr(X, C.c_float),
                                        ptr(y, C.c_float), ptr(Z, C.c_int32), C.byref(opt),
                                        ptr(hist, C.c_float)))
        return hist

    # --- energy + force training on device buffers (torch tensors) -------
    def mlp_ef_step(self, shape, P, m1, m2, X, y, Z, V, c, *, wE, lr, step, grad=None, with_loss=False):
        """One full-batch Adam step (or, with grad, the gradient only); tensors
        on the workspace's device, Z a host int32 array."""
        Z = np.ascontiguousarray(Z, np.int32)
        loss = np.zeros(shape.nz * shape.members) if with_loss else None
        vp_ = lambda t: None if t is None else C.c_void_p(t.data_ptr())
        self.check(self.L.pfw_mlp_ef_step(self.ws, C.byref(shape), vp_(P), vp_(m1), vp_(m2), len(Z), vp_(X), vp_(y),
                                          ptr(Z, C.c_int32), vp_(V), vp_(c), float(wE), float(lr), int(step),
                                          vp_(grad), ptr(loss, C.c_double)))
        return loss

    def mlp_input_grad(self, shape, P, X, Z, G):
        """∂y/∂x of every member at every sample into G (device tensor [members, n, nin])."""
        Z = np.ascontiguousarray(Z, np.int32)
        self.check(self.L.pfw_mlp_input_grad(self.ws, C.byref(shape), C.c_void_p(P.data_ptr()), len(Z),
                                             C.c_void_p(X.data_ptr()), ptr(Z, C.c_int32), C.c_void_p(G.data_ptr())))

    def surrogate_pullback(self, dEdx, F):
        """Forces (device tensor n×3) of a per-site dE/dfeature field (device tensor n×nin)."""
        self.check(self.L.pfw_surrogate_pullback(self.ws, C.c_void_p(dEdx.data_ptr()), C.c_void_p(F.data_ptr())))

    def probe_fp64(self):
        v = np.zeros(1)
        self.check(self.L.pfw_probe_fp64_peak(self.ws, ptr(v, C.c_double)))
        return float(v[0])
