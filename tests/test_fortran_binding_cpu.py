"""The Fortran binding module (include/m_qsgw_b200.f90) cannot be compiled
here (no Fortran compiler), so it is checked against the C header as text:
every bind(C) function names a declared entry point with the same number of
arguments, and the bind(C) types (qsgw_sxcf_args, qsgw_zmel_atom,
qsgw_zmel_ipw_args) list the C structs' fields in the same order with
matching kinds, as do the ctypes mirrors."""
import os
import re

import pytest

from ecalj_b200 import lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "qsgw_b200.h")
MODULE = os.path.join(ROOT, "include", "m_qsgw_b200.f90")


def _c_prototypes():
    src = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    out = {}
    for m in re.finditer(r"\b(?:int|long long)\s+(qsgw_[a-z0-9_]+)\s*\(([^)]*)\)\s*;", src):
        args = m.group(2).strip()
        out[m.group(1)] = 0 if args in ("", "void") else len(args.split(","))
    return out


def _fortran_functions():
    src = open(MODULE).read()
    src = re.sub(r"&\s*\n\s*", " ", src)                      # join continuation lines
    src = re.sub(r"!.*", "", src)
    out = {}
    for m in re.finditer(r"function\s+(qsgw_[a-z0-9_]+)\s*\(([^)]*)\)\s*bind\(C,\s*name='([a-z0-9_]+)'\)", src):
        name, args, cname = m.group(1), m.group(2).strip(), m.group(3)
        assert name == cname, (name, cname)
        out[name] = 0 if not args else len(args.split(","))
    return out


def test_every_fortran_binding_matches_a_c_prototype():
    c, f = _c_prototypes(), _fortran_functions()
    assert len(f) >= 30
    for name, nargs in f.items():
        assert name in c, f"{name} is bound in the Fortran module but not declared in the header"
        assert nargs == c[name], f"{name}: {nargs} Fortran arguments, {c[name]} in C"


def _c_struct_fields(name):
    src = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    body = re.search(r"typedef struct %s\s*\{(.*?)\}" % name, src, flags=re.S).group(1)
    fields = []
    for decl in body.split(";"):
        decl = decl.strip()
        if not decl:
            continue
        kind = "ptr" if "*" in decl else ("int" if decl.startswith("int") else "double")
        names = re.sub(r"^(const\s+)?(int|double)\s*", "", decl).replace("*", "")
        for n in names.split(","):
            m = re.match(r"\s*(\w+)\s*(?:\[(\d+)\])?", n)
            fields.append((m.group(1), kind + (f"[{m.group(2)}]" if m.group(2) else "")))
    return fields


def _fortran_type_fields(name):
    src = open(MODULE).read()
    body = re.search(r"type, bind\(C\) :: %s\n(.*?)end type" % name, src, flags=re.S).group(1)
    kinds = {"integer(c_int)": "int", "real(c_double)": "double", "type(c_ptr)": "ptr"}
    fields = []
    for line in body.strip().splitlines():
        k, names = line.split("::")
        for n in names.split(","):
            m = re.match(r"\s*(\w+)\s*(?:\((\d+)\))?", n)
            fields.append((m.group(1), kinds[k.strip()] + (f"[{m.group(2)}]" if m.group(2) else "")))
    return fields


def _ctypes_fields(struct):
    def kind(t):
        if t is lib.c_vp:
            return "ptr"
        if t is lib.c_int:
            return "int"
        if t is lib.c_dbl:
            return "double"
        if getattr(t, "_type_", None) is lib.c_int and hasattr(t, "_length_"):
            return f"int[{t._length_}]"
        raise AssertionError(t)
    return [(n, kind(t)) for n, t in struct._fields_]


@pytest.mark.parametrize("name,mirror", [("qsgw_sxcf_args", "SxcfArgs"), ("qsgw_zmel_atom", "ZmelAtom"),
                                         ("qsgw_zmel_ipw_args", "ZmelIpwArgs")])
def test_struct_layouts_match(name, mirror):
    c = _c_struct_fields(name)
    assert len(c) >= 10
    assert _fortran_type_fields(name) == c
    assert _ctypes_fields(getattr(lib, mirror)) == c
