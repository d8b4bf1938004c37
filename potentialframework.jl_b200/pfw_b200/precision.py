"""FP32-against-FP64 error report of the GPU evaluators (ACE/precision.jl:33-121).

compare_precision(model, systems, properties=(Energy, Forces, Virial),
tolerances=None) evaluates every system in an FP64 workspace and in the
mixed workspace (FP32 arithmetic, FP64 wrap and Kahan FP64 energy/virial)
and reports, per structure and pooled over all of them, the largest absolute
difference and the RMS of each requested property, where it occurs, the
energy error per atom and the largest per-atom force-vector error — the
reference's PrecisionReport fields.  With tolerances, a property whose
largest error exceeds its tolerance fails the structure and the report;
without, the statuses are "descriptive".  A structure whose evaluation raises
or returns nonfinite values fails with infinite errors and its message.

model: an ACECalculator, SmoothPair or LennardJones (the pair models run the
mixed pair kernel, ACE the mixed site kernel).
"""
from __future__ import annotations

import hashlib
import math

import numpy as np

from . import api
from . import lib as _lib
from .errors import argument_error

_KEYS = {"energy": _lib.REQ_E, "forces": _lib.REQ_F, "virial": _lib.REQ_V}


def _props(properties):
    bits = api._request_bits(properties)
    return [k for k, b in _KEYS.items() if bits & b]


def _evaluate(ws, sys, model, keys):
    r = api.evaluate_(ws, sys, model, request=tuple({"energy": api.Energy(), "forces": api.Forces(),
                                                    "virial": api.Virial()}[k] for k in keys))
    out = {}
    for k in keys:
        v = np.asarray(r[k], np.float64)
        if not np.all(np.isfinite(v)):
            raise ArithmeticError("nonfinite output")
        out[k] = v
    return out


def compare_precision(model, systems, properties=(api.Energy(), api.Forces(), api.Virial()), tolerances=None):
    tolerances = dict(tolerances or {})
    for k, v in tolerances.items():
        if k not in _KEYS or not (isinstance(v, (int, float)) and math.isfinite(v) and v >= 0):
            raise argument_error("tolerances must be finite nonnegative property errors")
    keys = _props(properties)
    if hasattr(systems, "X"):
        systems = [systems]
    ws = {64: api.Workspace(precision="Float64"), 32: api.Workspace(precision="mixed")}
    records, totals, failed = [], {}, False
    for index, sys in enumerate(systems, start=1):
        n = len(sys.X)
        results, errors = {}, []
        for prec in (64, 32):
            try:
                results[prec] = _evaluate(ws[prec], sys, model, keys)
            except Exception as e:  # the reference records the message and fails the structure
                errors.append(f"Float{prec}: {e}")
        bad = bool(errors)
        failed |= bad
        metrics = {}
        for key in keys:
            if bad:
                metrics[key] = dict(status="failed", maximum=math.inf, rms=math.inf, component=None)
                totals[key] = dict(maximum=math.inf, squares=math.inf, count=0, worst_structure=index, component=None)
                continue
            x, y = results[64][key].ravel(), results[32][key].ravel()
            if key == "virial":  # column-major 3×3, as vec(virial)
                x, y = results[64][key].ravel(order="F"), results[32][key].ravel(order="F")
            diff = y - x
            absd = np.abs(diff)
            maxerr = float(absd.max()) if diff.size else 0.0
            component = int(absd.argmax()) + 1 if diff.size else None  # 1-based as vec index
            rms = float(np.sqrt(np.mean(diff ** 2))) if diff.size else 0.0
            ok = key not in tolerances or maxerr <= tolerances[key]
            status = ("passed" if ok else "failed") if key in tolerances else "descriptive"
            failed |= not ok
            m = dict(status=status, maximum=maxerr, rms=rms, component=component)
            if key == "energy":
                m.update(location=dict(structure=index), absolute=maxerr, per_atom=0.0 if n == 0 else maxerr / n)
            elif key == "forces":
                vec = np.sqrt((diff.reshape(-1, 3) ** 2).sum(axis=1)) if diff.size else np.zeros(0)
                m.update(location=dict(structure=index, atom=None if component is None else (component - 1) // 3 + 1,
                                       axis=None if component is None else (component - 1) % 3 + 1),
                         max_atom_vector=float(vec.max()) if vec.size else 0.0)
            else:
                m.update(location=dict(structure=index, row=None if component is None else (component - 1) % 3 + 1,
                                       column=None if component is None else (component - 1) // 3 + 1))
            metrics[key] = m
            old = totals.get(key, dict(maximum=-math.inf, squares=0.0, count=0, worst_structure=index, component=None))
            worse = maxerr > old["maximum"]
            totals[key] = dict(maximum=max(old["maximum"], maxerr), squares=old["squares"] + float((diff ** 2).sum()),
                               count=old["count"] + diff.size, worst_structure=index if worse else old["worst_structure"],
                               component=component if worse else old["component"])
        X = np.asarray(sys.X, np.float64)
        H = np.asarray(sys.H, np.float64)
        rounding = float(np.abs(X.astype(np.float32).astype(np.float64) - X).max()) if X.size else 0.0
        Hf = H[np.isfinite(H)]
        cell_rounding = float(np.abs(Hf.astype(np.float32).astype(np.float64) - Hf).max()) if Hf.size else 0.0
        identity = hashlib.sha256(X.tobytes() + H.tobytes() + np.asarray(sys.species).tobytes()).hexdigest()
        status = "failed" if bad or any(v["status"] == "failed" for v in metrics.values()) else \
            ("descriptive" if not tolerances else "passed")
        records.append(dict(index=index, identity=identity, atoms=n, status=status,
                            position_rounding_max_A=rounding, cell_rounding_max_A=cell_rounding, errors=errors,
                            metrics=metrics))
    aggregate = dict(status="empty" if not records else ("failed" if failed else
                                                          ("descriptive" if not tolerances else "passed")))
    for key, v in totals.items():
        aggregate[key] = dict(maximum=v["maximum"],
                              pooled_rms=(0.0 if v["count"] == 0 else math.sqrt(v["squares"] / v["count"]))
                              if math.isfinite(v["squares"]) else math.inf,
                              components=v["count"], worst_structure=v["worst_structure"], component=v["component"])
    if "energy" in aggregate:
        aggregate["energy"]["maximum_per_atom"] = max((r["metrics"]["energy"].get("per_atom", math.inf)
                                                       for r in records), default=0.0)
    if "forces" in aggregate:
        vecs = [r["metrics"]["forces"].get("max_atom_vector", math.inf) for r in records]
        aggregate["forces"]["maximum_atom_vector"] = max(vecs, default=0.0)
        aggregate["forces"]["worst_vector_structure"] = int(np.argmax(vecs)) + 1 if vecs else None
    return dict(records=records, aggregate=aggregate,
                metadata=dict(properties=tuple(keys), tolerances=tolerances,
                              units=dict(energy="eV", forces="eV/Å", virial="eV"),
                              weighting="pooled components; failed cases propagate Inf"))
