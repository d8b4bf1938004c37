"""ACECalculator checkpoints: the reference's self-contained TOML format.

Restates ACE/persistence.jl:1-167 for the host mirror:

  encode / decode       checkpoint_encode / checkpoint_decode (persistence.jl:6-52):
                        nested named tuples (Python dicts with str keys), tuples,
                        nothing (None), strings, Bool scalars (Python bool), and
                        numeric scalars/arrays of the
                        Julia types Float32/64, Int8-64, UInt8-32 and Bool, with
                        shapes and element types kept (arrays stored column-major)
  dumps                 a TOML writer (Python reads TOML but ships no writer)
  save_calculator       save_calculator (persistence.jl:139-167): schema
                        "PotentialFrameWork.ACECalculator" version 2 with the
                        resolved model tree, the parameters and the state; the
                        destination is replaced only after a complete write
  load                  ACECalculator(path) (persistence.jl:101-124): a
                        checkpoint (versions 1 and 2) or a resolved TOML export

Nothing device-side is stored: geometry, schedules and workspaces are rebuilt
when a checkpoint is loaded.  Recipe JSON files need ACEpotentials and are
refused with an ArgumentError, as are custom (callable) radial channels.
"""
from __future__ import annotations

import math
import os
import re
import tempfile
import tomllib

import numpy as np

from .ace_model import PackedACE, read_resolved
from .errors import argument_error, dimension_mismatch

CHECKPOINT_SCHEMA = "PotentialFrameWork.ACECalculator"
WRITER = "pfw_b200"

# Julia element type name ↔ numpy dtype (CHECKPOINT_TYPES, persistence.jl:3-4)
_TYPES = {"Float32": np.float32, "Float64": np.float64, "Int8": np.int8, "Int16": np.int16, "Int32": np.int32,
          "Int64": np.int64, "UInt8": np.uint8, "UInt16": np.uint16, "UInt32": np.uint32, "Bool": np.bool_}
_NAMES = {np.dtype(v): k for k, v in _TYPES.items()}


# ---- checkpoint_encode / checkpoint_decode ---------------------------------
def _type_name(dtype):
    name = _NAMES.get(np.dtype(dtype))
    if name is None:
        raise argument_error(f"unsupported checkpoint numeric type {dtype}; save ordinary numeric parameters")
    return name


def _plain(v, dtype):
    if dtype == np.bool_:
        return bool(v)
    if np.issubdtype(dtype, np.integer):
        return int(v)
    return float(v)


def encode(x):
    """checkpoint_encode: a nested value → the tagged tree of the format."""
    if isinstance(x, dict) or hasattr(x, "_asdict"):
        d = x._asdict() if hasattr(x, "_asdict") else x
        if not all(isinstance(k, str) for k in d):
            raise argument_error("checkpoint named tuples need string field names")
        return {"kind": "namedtuple", "names": list(d.keys()), "items": [encode(v) for v in d.values()]}
    if isinstance(x, tuple):
        return {"kind": "tuple", "items": [encode(v) for v in x]}
    if x is None:
        return {"kind": "nothing"}
    if isinstance(x, str):
        return {"kind": "string", "value": x}
    if isinstance(x, (bool, np.bool_)):
        return {"kind": "scalar", "eltype": "Bool", "value": bool(x)}
    if isinstance(x, (int, float)) and not isinstance(x, np.generic):
        x = np.int64(x) if isinstance(x, int) else np.float64(x)
    if isinstance(x, np.generic):
        name = _type_name(x.dtype)
        if not np.isfinite(x):
            raise argument_error("nonfinite checkpoint values")
        return {"kind": "scalar", "eltype": name, "value": _plain(x, x.dtype)}
    if isinstance(x, (np.ndarray, list)):
        a = np.asarray(x)
        name = _type_name(a.dtype)
        if a.size and not np.all(np.isfinite(a)):
            raise argument_error("nonfinite checkpoint values")
        return {"kind": "array", "eltype": name, "shape": [int(s) for s in a.shape],
                "values": [_plain(v, a.dtype) for v in a.ravel(order="F")]}
    raise argument_error(f"unsupported checkpoint value {type(x).__name__}; use nested dicts/tuples, "
                         "numeric arrays/scalars, strings or None")


def decode(d):
    """checkpoint_decode: the tagged tree → nested dicts, tuples, None, str
    and numpy scalars/arrays of the saved element types and shapes."""
    kind = d.get("kind") if isinstance(d, dict) else None
    if kind == "namedtuple":
        names, items = d["names"], d["items"]
        if not (len(names) == len(items) and len(set(names)) == len(names)):
            raise argument_error("invalid checkpoint field names")
        return {str(k): decode(v) for k, v in zip(names, items)}
    if kind == "tuple":
        return tuple(decode(v) for v in d["items"])
    if kind == "nothing":
        return None
    if kind == "string":
        return str(d["value"])
    if kind in ("array", "scalar"):
        T = _TYPES.get(d.get("eltype"))
        if T is None:
            raise argument_error("unsupported checkpoint numeric type")
        if kind == "scalar":
            if T is np.bool_:
                return bool(d["value"])
            v = T(d["value"])
            if not np.isfinite(v):
                raise argument_error("nonfinite checkpoint value")
            return v
        shape = tuple(int(s) for s in d["shape"])
        if not all(s >= 0 for s in shape):
            raise dimension_mismatch("negative checkpoint array dimension")
        vals = np.array(d["values"], dtype=T)
        if math.prod(shape) != vals.size:
            raise dimension_mismatch("checkpoint array shape")
        if vals.size and not np.all(np.isfinite(vals)):
            raise argument_error("nonfinite checkpoint array")
        return vals.reshape(shape, order="F")
    raise argument_error(f"unsupported checkpoint value kind {kind}")


# ---- TOML writer -------------------------------------------------------------
_BARE = re.compile(r"^[A-Za-z0-9_-]+$")


def _key(k):
    return k if _BARE.match(k) else _string(k)


def _string(s):
    out = ['"']
    for ch in s:
        if ch == '"':
            out.append('\\"')
        elif ch == "\\":
            out.append("\\\\")
        elif ch == "\n":
            out.append("\\n")
        elif ch == "\t":
            out.append("\\t")
        elif ord(ch) < 0x20 or ord(ch) == 0x7F:
            out.append(f"\\u{ord(ch):04X}")
        else:
            out.append(ch)
    out.append('"')
    return "".join(out)


def _value(v):
    if isinstance(v, (bool, np.bool_)):
        return "true" if v else "false"
    if isinstance(v, (int, np.integer)):
        return str(int(v))
    if isinstance(v, (float, np.floating)):
        f = float(v)
        if not math.isfinite(f):
            raise argument_error("nonfinite value in TOML output")
        r = repr(f)
        return r if any(c in r for c in ".en") else r + ".0"
    if isinstance(v, str):
        return _string(v)
    if isinstance(v, (list, tuple, np.ndarray)):
        return "[" + ", ".join(_value(e) for e in v) + "]"
    if isinstance(v, dict):
        return "{" + ", ".join(f"{_key(k)} = {_value(e)}" for k, e in sorted(v.items())) + "}"
    raise argument_error(f"cannot write {type(v).__name__} to TOML")


def _is_table_array(v):
    return isinstance(v, list) and len(v) > 0 and all(isinstance(e, dict) for e in v)


def _emit(table, path, out):
    keys = sorted(table)
    for k in keys:
        v = table[k]
        if not isinstance(v, dict) and not _is_table_array(v):
            out.append(f"{_key(k)} = {_value(v)}")
    for k in keys:
        v = table[k]
        sub = path + [_key(k)]
        if isinstance(v, dict):
            out.append("")
            out.append("[" + ".".join(sub) + "]")
            _emit(v, sub, out)
        elif _is_table_array(v):
            for e in v:
                out.append("")
                out.append("[[" + ".".join(sub) + "]]")
                _emit(e, sub, out)


def dumps(d: dict) -> str:
    """TOML text of a tree of dicts, lists, strings, ints, floats and bools
    (keys sorted, as TOML.print(io, d; sorted=true))."""
    out = []
    _emit(d, [], out)
    return "\n".join(out).lstrip("\n") + "\n"


# ---- save / load -------------------------------------------------------------
def _model_with_parameters(model_dict, ps):
    """checkpoint_read_model (persistence.jl:82-99): validate the readout and
    scale shapes against the model tree and read it with these parameters."""
    if not (isinstance(ps, dict) and "WB" in ps and "Wpair" in ps):
        raise argument_error("checkpoint parameters require WB and Wpair")
    nz = len(model_dict["species_atomic_numbers"])
    m = int(model_dict["coupling"]["shape"][0])
    nq = len(model_dict["pair_radial"]["spec"])
    WB, Wp = np.asarray(ps["WB"]), np.asarray(ps["Wpair"])
    if WB.shape != (m, nz) or Wp.shape != (nq, nz):
        raise dimension_mismatch("checkpoint readout dimensions")
    for key, n in (("radial", len(model_dict["radial"]["spec"])), ("pair", nq)):
        if key in ps:
            block = ps[key]
            if not (isinstance(block, dict) and "scale" in block and np.asarray(block["scale"]).shape == (n, nz, nz)):
                raise dimension_mismatch(f"checkpoint {key} scale dimensions")
    if model_dict.get("radial", {}).get("kind") == "interface_channels_v1" or \
            model_dict.get("pair_radial", {}).get("kind") == "interface_channels_v1":
        raise argument_error("custom radial channels are not packed for the device")
    data = dict(model_dict)
    data["parameters"] = {"WB_shape": [m, nz], "Wpair_shape": [nq, nz],
                          "ordering": "vec(WB), vec(Wpair); Julia column-major",
                          "flat": [float(v) for v in np.concatenate([WB.astype(np.float64).ravel(order="F"),
                                                                     Wp.astype(np.float64).ravel(order="F")])]}
    return read_resolved(data)


def save_calculator(path, calc, parameters=None, state=None):
    """save_calculator(path, calc; parameters=calc.parameters, state=calc.state).

    Everything is encoded and validated before the destination is touched;
    the file is written to a temporary sibling and moved over the destination,
    so a failed save leaves an existing checkpoint intact.  Saving does not
    modify the calculator.  Returns path."""
    parameters = calc.parameters if parameters is None else parameters
    state = calc.state if state is None else state
    p = encode(parameters)
    s = encode(state)
    m = calc.model.resolved_dict()
    _model_with_parameters(m, parameters)  # the loader's own validation
    text = dumps({"schema": CHECKPOINT_SCHEMA, "schema_version": 2, "writer": WRITER,
                  "model": m, "parameters": p, "state": s})
    destination = os.path.abspath(path)
    fd, tmp = tempfile.mkstemp(dir=os.path.dirname(destination), prefix=".pfw_ckpt_")
    try:
        with os.fdopen(fd, "w", encoding="utf-8") as f:
            f.write(text)
        os.replace(tmp, destination)
    finally:
        if os.path.exists(tmp):
            os.remove(tmp)
    return path


def load(path):
    """(model, parameters, state) of a checkpoint or a resolved TOML export;
    the file's content, not its extension, decides which (persistence.jl:113-124)."""
    with open(path, "rb") as f:
        raw = f.read()
    if raw.lstrip().startswith(b"{"):
        raise argument_error("recipe JSON needs ACEpotentials; load its resolved TOML export instead")
    try:
        d = tomllib.loads(raw.decode("utf-8"))
    except (tomllib.TOMLDecodeError, UnicodeDecodeError) as e:
        raise argument_error(f"not a TOML checkpoint or resolved model: {e}") from None
    if d.get("schema") == CHECKPOINT_SCHEMA:
        if d.get("schema_version") not in (1, 2):
            raise argument_error("unsupported ACECalculator checkpoint version")
        ps = decode(d["parameters"])
        st = decode(d["state"])
        model = _model_with_parameters(d["model"], ps)
        return model, ps, st
    model = read_resolved(d)
    return model, model.default_parameters(), {}


def trainable_parameters(model: PackedACE, ps):
    """trainable_parameters (ACE/serial.jl:12-16): ps plus unit radial and
    pair scales where ps has none."""
    out = {k: (np.array(v) if isinstance(v, np.ndarray) else v) for k, v in ps.items()}
    nz = model.nz
    if "radial" not in out:
        out["radial"] = {"scale": np.ones((model.radial.nchannels, nz, nz))}
    if "pair" not in out:
        out["pair"] = {"scale": np.ones((model.pair.nchannels, nz, nz))}
    return out
