"""The ISO_C_BINDING shim (wam_b200/fortran/wamgpu_binding.f90) against the C
ABI it binds (include/wamgpu.h): every BIND(C) name is declared in the header
with the same number of arguments, and the BIND(C) derived type has the
fields of struct wamgpu_config in the same order and kinds.  No Fortran
compiler exists on these machines, so this is a source-level check."""
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
F90 = os.path.join(ROOT, "wam_b200", "fortran", "wamgpu_binding.f90")
HDR = os.path.join(ROOT, "include", "wamgpu.h")


def _fortran_functions():
    src = open(F90).read().replace("&\n&", " ").replace("&\n", " ")
    out = {}
    for m in re.finditer(r"FUNCTION\s+(\w+)\s*\(([^)]*)\)\s*(?:&\s*)?BIND\(C,\s*NAME='(\w+)'\)", src):
        args = [a.strip() for a in m.group(2).split(",") if a.strip()]
        out[m.group(3)] = args
    return out


def _c_prototypes():
    src = re.sub(r"/\*.*?\*/", "", open(HDR).read(), flags=re.S)
    out = {}
    for m in re.finditer(r"WAMGPU_API\s+[\w\s\*]+?\b(wamgpu_\w+)\s*\(([^)]*)\)\s*;", src):
        args = [a.strip() for a in m.group(2).split(",") if a.strip() and a.strip() != "void"]
        out[m.group(1)] = args
    return out


def test_every_bound_name_is_declared_with_its_arity():
    f = _fortran_functions()
    c = _c_prototypes()
    assert len(f) >= 20
    for name, args in f.items():
        assert name in c, f"{name} is bound in the shim but not declared in wamgpu.h"
        assert len(args) == len(c[name]), f"{name}: {len(args)} Fortran arguments, {len(c[name])} in C"


def test_config_type_matches_struct():
    src = open(F90).read()
    body = re.search(r"TYPE, BIND\(C\) :: WAMGPU_CONFIG(.*?)END TYPE", src, re.S).group(1)
    fields = []
    for line in body.splitlines():
        m = re.match(r"\s*(INTEGER\(C_INT\)|REAL\(C_DOUBLE\))\s*::\s*(.*)", line)
        if m:
            kind = "int" if "INTEGER" in m.group(1) else "double"
            fields += [(n.strip().lower(), kind) for n in m.group(2).split(",")]
    from wam_b200._lib import WamgpuConfig
    import ctypes
    want = [(n, "int" if t is ctypes.c_int else "double") for n, t in WamgpuConfig._fields_]
    assert fields == want
