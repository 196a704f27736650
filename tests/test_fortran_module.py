"""The Fortran module (iso_c_binding interfaces for the reference's driver)
binds every entry point that include/psdns_gpu.h declares, under the same C
name and with the same number of arguments.  No Fortran compiler exists in
this image, so the module is checked as text."""
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def c_decls():
    h = open(os.path.join(ROOT, "include", "psdns_gpu.h")).read()
    h = re.sub(r"/\*.*?\*/", "", h, flags=re.S)
    out = {}
    for m in re.finditer(r"\bint\s+(psdns_gpu_\w+)\s*\(([^)]*)\)\s*;", h):
        args = [a for a in m.group(2).split(",") if a.strip() and a.strip() != "void"]
        out[m.group(1)] = len(args)
    return out


def f_decls():
    f = open(os.path.join(ROOT, "nasa-bluewater-psdns-benchmark-minsky_b200", "fortran", "psdns_gpu_mod.f90")).read()
    f = f.replace("&\n", " ")
    out = {}
    for m in re.finditer(r"function\s+(\w+)\s*\(([^)]*)\)\s*bind\s*\(\s*c\s*,\s*name\s*=\s*'(\w+)'", f, flags=re.I):
        args = [a for a in m.group(2).split(",") if a.strip()]
        out[m.group(3)] = len(args)
    return out


def test_every_entry_point_has_a_fortran_interface():
    c, f = c_decls(), f_decls()
    assert len(c) > 40
    assert sorted(set(c) - set(f)) == []
    assert sorted(set(f) - set(c)) == []
    assert {k: c[k] for k in c if c[k] != f[k]} == {}
