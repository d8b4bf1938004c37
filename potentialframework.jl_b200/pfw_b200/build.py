"""Build libpfw_b200.so for sm_100a in-tree with nvcc.

    python -m pfw_b200.build            (from potentialframework.jl_b200/)

The geometry that decides the neighbour set is written with explicit
round-to-nearest intrinsics, so the whole library can be compiled with FMA
contraction enabled; host code is compiled with -ffp-contract=off so the
host-side cell decisions round exactly like the reference's.
"""
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(PKG, "csrc")
OUT = os.path.join(PKG, "lib", "libpfw_b200.so")
SOURCES = ["geometry.cu", "pair.cu", "snapshot.cu", "ace.cu", "capi.cu"]


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def needs_build():
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(PKG, "..", "include", "pfw_b200.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(verbose=False, force=False, extra=()):
    if not force and not needs_build():
        return OUT
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    cmd = [nvcc(), "-O3", "-std=c++17", "-shared", "-Xcompiler", "-fPIC,-ffp-contract=off",
           "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "--expt-relaxed-constexpr",
           "--extended-lambda", "-Xptxas", "-warn-spills", "-o", OUT + ".tmp"]
    cmd += list(extra)
    cmd += [os.path.join(CSRC, s) for s in SOURCES]
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed")
    if verbose and (r.stdout or r.stderr):
        print(r.stdout + r.stderr)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    extra = sys.argv[1:]
    print(build(verbose=True, force=True, extra=extra))
