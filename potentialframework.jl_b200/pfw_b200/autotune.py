"""Autotuner of the ACE site kernel's schedule (edges per chunk × site groups
per CTA), with a JSON cache.

The reference tunes its GPU ACE launch by hand (GPUConfig workgroup sizes,
NeighbourList/gpu.jl:61-73; the chunk executor's sizes, ACE/chunks.jl); here
every schedule that fits the model in shared memory is timed on the caller's
own workload and the fastest is kept, keyed by device, model and workload
shape.  The cache file defaults to $PFW_B200_CACHE or
~/.cache/pfw_b200/autotune.json.
"""
from __future__ import annotations

import hashlib
import json
import os
import time

import numpy as np

from . import lib

# (edges per chunk, site groups per CTA); schedules the library rejects for
# its site-group size or the model's shared memory are skipped
CANDIDATES = ((8, 1), (8, 2), (8, 4), (8, 8), (16, 1), (16, 2), (16, 3), (16, 4), (16, 6), (16, 8), (32, 1),
              (32, 2), (32, 3), (32, 4))


def cache_path():
    p = os.environ.get("PFW_B200_CACHE")
    if p:
        return p
    return os.path.join(os.path.expanduser("~"), ".cache", "pfw_b200", "autotune.json")


def model_key(packed):
    """Content hash of the packed model tables (shape and values)."""
    h = hashlib.sha256()
    for k, v in sorted(packed.to_npz_dict().items()):
        a = np.ascontiguousarray(v)
        h.update(k.encode())
        h.update(str(a.dtype).encode() + str(a.shape).encode())
        h.update(a.tobytes())
    return h.hexdigest()[:16]


def workload_key(n, nsys=1):
    """Atom count rounded to a power of two, and the number of systems."""
    return f"n{1 << max(0, int(np.ceil(np.log2(max(n, 1)))))}_s{nsys}"


def device_key():
    import torch
    return torch.cuda.get_device_name(0).replace(" ", "_")


def _load(path):
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(path, table):
    os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(table, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def tune(h, packed, run, n, nsys=1, *, candidates=CANDIDATES, reps=3, path=None, use_cache=True):
    """Choose and set the fastest schedule for `run()` (one evaluation on the
    handle's current geometry and model).  Returns (chunk, groups, timings)."""
    path = path or cache_path()
    key = f"{device_key()}|{model_key(packed)}|{workload_key(n, nsys)}"
    table = _load(path) if use_cache else {}
    if use_cache and key in table:
        c, g = table[key]["schedule"]
        h.ace_schedule(c, g)
        return c, g, table[key].get("ms", {})
    timings = {}
    for c, g in candidates:
        try:
            h.ace_schedule(c, g)
        except lib.PFWError:
            continue  # does not fit this model in shared memory
        run()  # warm-up (also captures any per-schedule graph)
        best = np.inf
        for _ in range(reps):
            t = time.perf_counter()
            run()
            best = min(best, time.perf_counter() - t)
        timings[f"{c}x{g}"] = best * 1e3
    if not timings:
        raise RuntimeError("no ACE schedule fits this model")
    c, g = map(int, min(timings, key=timings.get).split("x"))
    h.ace_schedule(c, g)
    if use_cache:
        table[key] = dict(schedule=[c, g], ms=timings)
        _store(path, table)
    return c, g, timings
