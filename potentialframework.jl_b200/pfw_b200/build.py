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
SOURCES = ["geometry.cu", "reduce.cu", "pair.cu", "pair_half.cu", "snapshot.cu", "ace.cu", "capi.cu", "noalloc.cu", "mlp.cu", "skin.cu", "slab.cu"]


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


FLAGS = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC,-ffp-contract=off", "-gencode",
         "arch=compute_100a,code=sm_100a", "-lineinfo", "--expt-relaxed-constexpr", "--extended-lambda",
         "-Xptxas", "-warn-spills"]


def build(verbose=False, force=False, extra=(), out=None):
    """Compile every source to an object in parallel, then link the shared library."""
    out = out or OUT
    if not force and out == OUT and not needs_build():
        return out
    objdir = os.path.join(PKG, "lib", "obj")
    os.makedirs(objdir, exist_ok=True)
    procs = []
    for s in SOURCES:
        obj = os.path.join(objdir, s.replace(".cu", ".o"))
        cmd = [nvcc(), *FLAGS, *extra, "-c", os.path.join(CSRC, s), "-o", obj]
        if verbose:
            print(" ".join(cmd))
        procs.append((s, obj, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
    objs, failed = [], False
    for s, obj, p in procs:
        text = p.communicate()[0]
        if p.returncode != 0:
            sys.stderr.write(text)
            failed = True
        elif verbose and text.strip():
            print(text)
        objs.append(obj)
    if failed:
        raise RuntimeError("nvcc failed")
    link = [nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", out + ".tmp", *objs]
    r = subprocess.run(link, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc link failed")
    os.replace(out + ".tmp", out)
    return out


if __name__ == "__main__":
    extra = sys.argv[1:]
    print(build(verbose=True, force=True, extra=extra))
