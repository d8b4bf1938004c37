"""CPU-side checks of the C ABI: the library builds, loads, and exports every
symbol that include/pfw_b200.h declares; without a GPU it fails loudly; the
Julia binding's struct mirrors match the header's structs and its ccalls the
declared argument counts."""
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


C_TO_JULIA = {"int32_t": "Int32", "double": "Float64", "uint8_t": "UInt8"}


def c_struct_fields(name):
    src = open(os.path.join(ROOT, "include", "pfw_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    body = re.search(r"typedef struct " + name + r"\s*\{(.*?)\}\s*" + name + ";", src, re.S).group(1)
    out = []
    for decl in body.split(";"):
        decl = decl.strip()
        if not decl:
            continue
        m = re.match(r"(?:const\s+)?(\w+)\s*(\*?)\s*(\w+)$", decl)
        ctype, ptr, field = m.groups()
        jl = C_TO_JULIA.get(ctype, {"pfw_radial_family": "RadialFamilyC"}.get(ctype, ctype))
        out.append((field, f"Ptr{{{jl}}}" if ptr else jl))
    return out


def julia_struct_fields(name):
    src = open(os.path.join(ROOT, "potentialframework.jl_b200", "julia", "PFWB200.jl")).read()
    body = re.search(r"\nstruct " + name + r"\n(.*?)\nend\n", src, re.S).group(1)
    return [tuple(x.strip() for x in line.split("#")[0].split("::")) for line in body.strip().splitlines()]


def test_julia_binding_structs_match_the_header():
    """The Julia binding passes pfw_options, pfw_radial_family and
    pfw_ace_tables by reference: its isbits mirrors must list the same
    fields, in the same order, with the same types."""
    assert julia_struct_fields("Options") == c_struct_fields("pfw_options")
    assert julia_struct_fields("RadialFamilyC") == c_struct_fields("pfw_radial_family")
    assert julia_struct_fields("ACETablesC") == c_struct_fields("pfw_ace_tables")


def header_arity():
    src = open(os.path.join(ROOT, "include", "pfw_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    out = {}
    for name, args in re.findall(r"\b(pfw_[a-z0-9_]+)\s*\(([^)]*)\)\s*;", src):
        args = args.strip()
        out[name] = 0 if args in ("", "void") else args.count(",") + 1
    return out


def test_julia_ccalls_match_the_header_arity():
    src = open(os.path.join(ROOT, "potentialframework.jl_b200", "julia", "PFWB200.jl")).read()
    calls = re.findall(r"ccall\(\(:(pfw_[a-z0-9_]+), libpfw\),\s*\w+(?:\{\w+\})?,\s*\(([^()]*(?:\([^()]*\))?[^()]*)\)", src)
    assert len(calls) == src.count("ccall(")  # every ccall parsed
    arity = header_arity()
    for name, types in calls:
        n = len([t for t in types.split(",") if t.strip()])
        assert name in arity, name
        assert n == arity[name], (name, n, arity[name])
