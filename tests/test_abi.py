"""CPU-side checks of the C ABI: the library builds, loads, and exports every
symbol that include/pfw_b200.h declares; without a GPU it fails loudly."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = []
    for fn in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if fn.endswith(".h"):
            src = open(os.path.join(ROOT, "include", fn)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names += re.findall(r"\b(pfw_[a-z0-9_]+)\s*\(", src)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    from pfw_b200 import build, lib
    build.build()
    L = ctypes.CDLL(lib.LIBPATH)
    syms = declared_symbols()
    assert "pfw_evaluate" in syms and "pfw_neighbour_fill" in syms
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing


def test_no_silent_cpu_fallback_without_gpu():
    from conftest import gpu_available
    if gpu_available():
        pytest.skip("GPU present")
    from pfw_b200 import lib
    with pytest.raises(lib.PFWError):
        lib.Handle()


def test_version():
    from pfw_b200 import lib
    assert lib.load().pfw_version().decode().count(".") == 2
