"""The Fortran binding module (include/m_qsgw_b200.f90) cannot be compiled
here (no Fortran compiler), so it is checked against the C header as text:
every bind(C) function names a declared entry point with the same number of
arguments, and the bind(C) type qsgw_sxcf_args lists the C struct's fields
in the same order with matching kinds (and so does the ctypes mirror)."""
import os
import re

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


def _c_struct_fields():
    src = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    body = re.search(r"typedef struct qsgw_sxcf_args\s*\{(.*?)\}", src, flags=re.S).group(1)
    fields = []
    for decl in body.split(";"):
        decl = decl.strip()
        if not decl:
            continue
        kind = "ptr" if "*" in decl else ("int" if decl.startswith("int") else "double")
        names = re.sub(r"^(const\s+)?(int|double)\s*", "", decl).replace("*", "")
        fields += [(n.strip(), kind) for n in names.split(",")]
    return fields


def _fortran_type_fields():
    src = open(MODULE).read()
    body = re.search(r"type, bind\(C\) :: qsgw_sxcf_args(.*?)end type", src, flags=re.S).group(1)
    kinds = {"integer(c_int)": "int", "real(c_double)": "double", "type(c_ptr)": "ptr"}
    fields = []
    for line in body.strip().splitlines():
        k, names = line.split("::")
        fields += [(n.strip(), kinds[k.strip()]) for n in names.split(",")]
    return fields


def test_sxcf_args_layout_matches():
    c = _c_struct_fields()
    assert _fortran_type_fields() == c
    mirror = [(n, "ptr" if t is lib.c_vp else ("int" if t is lib.c_int else "double"))
              for n, t in lib.SxcfArgs._fields_]
    assert mirror == c
