"""Generate tests/golden fixtures from the reference's own data files.

Reads (text only, never executes) the reference checkout's
data/ace_ref/resolved_model_v1.toml, reference_results.xyz and
reloaded_predictions.toml — the saved 33-frame TiAl oracle of
test/neighbour_saved_reference.jl — and writes tial_ace.npz: the packed model
tables, the 33 frames (positions, cells, species channels) and the saved
ACEpotentials-0.10.2 energies, forces and virials.

Usage: python tests/golden/make_golden.py [/path/to/reference]
"""
import hashlib
import os
import re
import sys
import tomllib

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "potentialframework.jl_b200"))
from pfw_b200.ace_model import load_resolved  # noqa: E402

SYMBOLS = {"Ti": 22, "Al": 13}


def read_frames(path):
    frames = []
    with open(path) as f:
        lines = f.read().splitlines()
    k = 0
    while k < len(lines) and lines[k].strip():
        n = int(lines[k]); header = lines[k + 1]
        lat = re.search(r'Lattice="([^"]+)"', header)
        assert lat and "pbc=[T, T, T]" in header
        H = np.array([float(v) for v in lat.group(1).split()]).reshape(3, 3).T  # columns = vectors
        X = np.zeros((n, 3)); z = []
        for i in range(n):
            fields = lines[k + 2 + i].split()
            z.append(SYMBOLS[fields[0]]); X[i] = [float(v) for v in fields[1:4]]
        frames.append((X, H, z))
        k += n + 2
    return frames


def main(ref):
    d = os.path.join(ref, "data", "ace_ref")
    model = load_resolved(os.path.join(d, "resolved_model_v1.toml"))
    pred = tomllib.load(open(os.path.join(d, "reloaded_predictions.toml"), "rb"))
    geo = os.path.join(d, "reference_results.xyz")
    assert hashlib.sha256(open(geo, "rb").read()).hexdigest() == pred["geometry_sha256"]
    frames = read_frames(geo)
    assert len(frames) == len(pred["frames"]) == 33
    out = model.to_npz_dict("model_")
    out["nframes"] = np.array(len(frames))
    for k, ((X, H, z), p) in enumerate(zip(frames, pred["frames"])):
        out[f"f{k}_X"] = X
        out[f"f{k}_H"] = H
        out[f"f{k}_species"] = np.array([model.channel_of(v) for v in z], np.int32)
        out[f"f{k}_energy"] = np.array(p["energy_eV"])
        out[f"f{k}_forces"] = np.array(p["forces_eV_per_A"])              # (n, 3)
        out[f"f{k}_virial"] = np.array(p["virial_eV_columns"]).T          # columns -> 3x3
    out["model_sha256"] = np.array(pred["model_sha256"])
    np.savez_compressed(os.path.join(HERE, "tial_ace.npz"), **out)
    print("wrote", os.path.join(HERE, "tial_ace.npz"), "frames", len(frames))


def reference_dir(arg=None):
    """The reference checkout: the command-line argument, else $PFW_REFERENCE_DIR,
    else the read-only checkout at /root/reference."""
    return arg or os.environ.get("PFW_REFERENCE_DIR") or "/root/reference"


if __name__ == "__main__":
    main(reference_dir(sys.argv[1] if len(sys.argv) > 1 else None))
