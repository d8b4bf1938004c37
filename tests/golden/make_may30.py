"""Generate the May30 Ti–Al–V fixtures from the reference's own data files.

Reads (text only, never executes) the reference checkout's data/may30/:
resolved.toml — the fitted degree-10, order-3 model with real solid harmonics
through l = 6, 114 radial channels on 1000 spline nodes and PolyEnvelope1sR
pair channels — and the three structures bcc-128, hcp-150 and omega-240 with
their splined ACEpotentials predictions (test/ace_may30.jl compares against
them at atol 2e-8 eV for energies and virials, 2e-9 eV/Å for forces).

Writes
  may30_frames.npz  the three structures and predictions (small; committed)
  may30_model.npz   the packed model tables (33 MB of spline coefficients;
                    not committed — regenerated by __graft_entry__.build()
                    whenever the reference checkout is present)

Usage: python tests/golden/make_may30.py [/path/to/reference]
"""
import os
import sys
import tomllib

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "potentialframework.jl_b200"))
from pfw_b200.ace_model import load_resolved  # noqa: E402

NAMES = ("bcc-128", "hcp-150", "omega-240")


def main(ref, frames_only=False):
    d = os.path.join(ref, "data", "may30")
    out = {}
    Z = [22, 13, 23]
    for k, name in enumerate(NAMES):
        t = tomllib.load(open(os.path.join(d, name + ".toml"), "rb"))
        n = len(t["species"])
        out[f"f{k}_name"] = np.array(name)
        out[f"f{k}_X"] = np.array(t["positions"], np.float64).reshape(n, 3)        # 3×n column-major
        out[f"f{k}_H"] = np.array(t["cell"], np.float64).reshape(3, 3).T          # columns = cell vectors
        out[f"f{k}_species"] = np.array([Z.index(z) for z in t["species"]], np.int32)
        out[f"f{k}_energy"] = np.array(t["energy"])
        out[f"f{k}_forces"] = np.array(t["forces"], np.float64).reshape(n, 3)
        out[f"f{k}_virial"] = np.array(t["virial"], np.float64).reshape(3, 3).T   # column-major 3×3
    out["nframes"] = np.array(len(NAMES))
    np.savez_compressed(os.path.join(HERE, "may30_frames.npz"), **out)
    if frames_only:
        return
    model = load_resolved(os.path.join(d, "resolved.toml"))
    assert model.atomic_numbers == Z and model.angular_kind == 1 and model.lmax == 6
    np.savez(os.path.join(HERE, "may30_model.npz"), **model.to_npz_dict("model_"))
    print("wrote may30_frames.npz and may30_model.npz:", model.nbasis, "invariants,", model.nproducts,
          "products,", model.ndensity, "densities,", model.radial.nchannels, "radial channels")


def reference_dir(arg=None):
    """The reference checkout: the command-line argument, else $PFW_REFERENCE_DIR,
    else the read-only checkout at /root/reference."""
    return arg or os.environ.get("PFW_REFERENCE_DIR") or "/root/reference"


if __name__ == "__main__":
    main(reference_dir(sys.argv[1] if len(sys.argv) > 1 else None))
