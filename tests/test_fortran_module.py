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


# ---------------------------------------------------------------------------
# Argument-level agreement: how each argument is passed (by value or by
# reference), its kind, and read-only pointers bound as intent(in); and the
# field sequence of the bind(c) psdns_params type against the C struct.
# ---------------------------------------------------------------------------
def _c_args():
    h = open(os.path.join(ROOT, "include", "psdns_gpu.h")).read()
    h = re.sub(r"/\*.*?\*/", "", h, flags=re.S)
    out = {}
    for m in re.finditer(r"\bint\s+(psdns_gpu_\w+)\s*\(([^)]*)\)\s*;", h):
        args = []
        for a in m.group(2).split(","):
            a = " ".join(a.split())
            if not a or a == "void":
                continue
            a = re.sub(r"\*\s*const\b", "*", a)   # pointer to const pointers
            stars = a.count("*")
            mm = re.match(r"(const\s+)?(\w+)\s+(\w+)$", " ".join(a.replace("*", " ").split()))
            assert mm, a
            args.append({"const": bool(mm.group(1)), "type": mm.group(2), "ptr": stars, "name": mm.group(3)})
        out[m.group(1)] = args
    return out


def _f_args():
    f = open(os.path.join(ROOT, "nasa-bluewater-psdns-benchmark-minsky_b200", "fortran", "psdns_gpu_mod.f90")).read()
    f = re.sub(r"!.*", "", f).replace("&\n", " ")
    out = {}
    for m in re.finditer(r"function\s+(\w+)\s*\(([^)]*)\)\s*bind\s*\(\s*c\s*,\s*name\s*=\s*'(\w+)'\s*\)(.*?)end\s+function",
                         f, flags=re.I | re.S):
        names = [a.strip().lower() for a in m.group(2).split(",") if a.strip()]
        decl = {}
        for line in m.group(4).splitlines():
            if "::" not in line or line.strip().lower().startswith("import"):
                continue
            spec, vars_ = line.split("::", 1)
            spec = spec.strip().lower()
            for v in re.findall(r"(\w+)\s*(\([^)]*\))?", vars_):
                if v[0]:
                    decl[v[0].lower()] = {"spec": spec, "array": bool(v[1])}
        out[m.group(3)] = [(n, decl.get(n)) for n in names]
    return out


# C scalar passed by value -> Fortran kind; C pointee -> Fortran kinds that may bind it
_BY_VALUE = {"int32_t": "integer(c_int32_t)", "int64_t": "integer(c_int64_t)", "size_t": "integer(c_size_t)",
             "double": "real(c_double)"}
_BY_REF = {"double": ("real(c_double)", "complex(c_double_complex)"), "float": ("real(c_float)",),
           "int32_t": ("integer(c_int32_t)",),
           "int64_t": ("integer(c_int64_t)",), "char": ("character(kind=c_char)",),
           "psdns_params": ("type(psdns_params)",), "void": ("type(c_ptr)",)}


def test_each_argument_is_bound_with_the_right_kind_and_passing_mode():
    c, f = _c_args(), _f_args()
    problems = []
    for name, cargs in c.items():
        fargs = f[name]
        assert len(fargs) == len(cargs), name
        for ca, (fn, fd) in zip(cargs, fargs):
            where = f"{name}({ca['name']} <-> {fn})"
            if fd is None:
                problems.append(where + ": no declaration")
                continue
            spec = fd["spec"].replace(" ", "")
            is_value = ",value" in spec
            kind = spec.split(",")[0]
            intent_in = "intent(in)" in spec
            if ca["ptr"] == 0:
                # scalars are passed by value with the matching kind
                if not (is_value and kind == _BY_VALUE[ca["type"]].replace(" ", "")):
                    problems.append(where + f": C {ca['type']} by value, Fortran {spec}")
            elif ca["type"] == "void" and ca["ptr"] == 1:
                # an opaque address (context, device array, stream, pinned array)
                if not (is_value and kind == "type(c_ptr)"):
                    problems.append(where + f": void* must be type(c_ptr), value; got {spec}")
            elif ca["type"] == "void" and ca["ptr"] == 2:
                if is_value or kind != "type(c_ptr)":
                    problems.append(where + f": void** must be type(c_ptr) by reference; got {spec}")
            else:
                # typed pointer: bound by reference with the pointee's kind, or
                # as an address (type(c_ptr), value) that may be null
                if is_value:
                    if kind != "type(c_ptr)":
                        problems.append(where + f": pointer bound by value as {spec}")
                elif kind not in _BY_REF[ca["type"]]:
                    problems.append(where + f": C {ca['type']}* bound as {spec}")
                elif ca["const"] and "intent(out)" in spec or ca["const"] and "intent(inout)" in spec:
                    problems.append(where + ": const pointer bound with intent(out/inout)")
                elif not ca["const"] and intent_in:
                    problems.append(where + ": writable pointer bound as intent(in)")
    assert problems == []


def _c_struct_fields():
    h = open(os.path.join(ROOT, "include", "psdns_gpu.h")).read()
    h = re.sub(r"/\*.*?\*/", "", h, flags=re.S)
    body = re.search(r"typedef\s+struct\s+psdns_params\s*\{(.*?)\}\s*psdns_params\s*;", h, flags=re.S).group(1)
    out = []
    for stmt in body.split(";"):
        stmt = " ".join(stmt.split())
        if not stmt:
            continue
        typ, rest = stmt.split(" ", 1)
        for v in rest.split(","):
            v = v.strip()
            mm = re.match(r"(\w+)(\[(\d+)\])?$", v)
            out.append((typ, mm.group(1), int(mm.group(3) or 1)))
    return out


def _f_type_fields():
    f = open(os.path.join(ROOT, "nasa-bluewater-psdns-benchmark-minsky_b200", "fortran", "psdns_gpu_mod.f90")).read()
    f = re.sub(r"!.*", "", f)
    body = re.search(r"type\s*,\s*bind\s*\(\s*c\s*\)\s*::\s*psdns_params(.*?)end\s+type", f, flags=re.I | re.S).group(1)
    out = []
    for line in body.splitlines():
        if "::" not in line:
            continue
        spec, vars_ = line.split("::", 1)
        for v in re.findall(r"(\w+)\s*(?:\((\d+)\))?", vars_):
            if v[0]:
                out.append((spec.strip().lower().replace(" ", ""), v[0].lower(), int(v[1] or 1)))
    return out


def test_params_type_matches_the_c_struct_field_by_field():
    kinds = {"int32_t": "integer(c_int32_t)", "double": "real(c_double)"}
    c = [(kinds[t], n.lower(), k) for t, n, k in _c_struct_fields()]
    f = _f_type_fields()
    assert len(c) > 20
    assert c == f
    # the ctypes mirror has the same layout
    import sys
    sys.path.insert(0, os.path.join(ROOT, "nasa-bluewater-psdns-benchmark-minsky_b200"))
    import ctypes
    import psdns_gpu
    ct = {ctypes.c_int32: "integer(c_int32_t)", ctypes.c_double: "real(c_double)"}
    py = []
    for n, t in psdns_gpu.Params._fields_:
        if hasattr(t, "_length_"):
            py.append((ct[t._type_], n.lower(), t._length_))
        else:
            py.append((ct[t], n.lower(), 1))
    assert py == c
    assert ctypes.sizeof(psdns_gpu.Params) == 4 * 16 + 8 * 22
