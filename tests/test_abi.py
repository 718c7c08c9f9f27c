"""The C-ABI library loads and exports every entry point that
include/qsgw_b200.h declares; argument checks that run before any CUDA call
behave (no GPU needed)."""
import os
import re
import subprocess

import pytest

from ecalj_b200 import lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "qsgw_b200.h")


def _declared():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(qsgw_[a-z0-9_]+)\s*\(", src)))


@pytest.fixture(scope="module")
def so():
    if not os.path.exists(lib.LIBPATH):
        from ecalj_b200 import build
        build.build()
    return lib.load()


def test_header_lists_entry_points():
    names = _declared()
    assert "qsgw_x0gemm" in names and "qsgw_sxcf_correlation_d" in names
    assert set(names) == set(lib.exported_symbols()), set(names) ^ set(lib.exported_symbols())


def test_library_exports_every_declared_symbol(so):
    out = subprocess.run(["nm", "-D", "--defined-only", lib.LIBPATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (qsgw_\w+)", out))
    missing = [n for n in _declared() if n not in exported]
    assert not missing, missing
    for n in _declared():
        assert hasattr(so, n)


def test_calls_before_init_fail_cleanly(so):
    if lib.initialized():
        pytest.skip("a GPU test initialised the library earlier in this process")
    assert so.qsgw_synchronize() == -4
    assert "qsgw_init" in lib.last_error()
    assert so.qsgw_x0gemm(None, 1, 1, 1, 1, 1, 1, 1, None, 1, 1, 1, 1, 1, 1,
                          None, None, None, None, None, None, None, 0) == -4


def test_precision_switch_validates(so):
    if lib.initialized():
        pytest.skip("a GPU test initialised the library earlier in this process")
    assert so.qsgw_set_precision(7, 2) == -1
    assert so.qsgw_set_precision(1, 3) == -1
    assert so.qsgw_set_precision(1, 2) == 0
    assert lib.get_precision() == (1, 2)
    assert so.qsgw_set_precision(0, 1) == 0


def _cabi_caller(tmp_path):
    exe = tmp_path / "cabi_caller"
    src = os.path.join(ROOT, "tests", "cabi_caller.cpp")
    libdir = os.path.dirname(lib.LIBPATH)
    subprocess.run(["g++", "-O1", "-std=c++17", "-I", os.path.join(ROOT, "include"), src, "-o", str(exe),
                    "-L", libdir, "-lqsgw_b200", f"-Wl,-rpath,{libdir}"], check=True)
    return exe


def test_cpp_caller_before_init(so, tmp_path):
    """A C++ host program compiled against the header links and gets clean
    status codes before qsgw_init."""
    r = subprocess.run([str(_cabi_caller(tmp_path))], capture_output=True, text=True)
    assert r.returncode == 0 and "OK cpu" in r.stdout, r.stdout + r.stderr


@pytest.mark.gpu
def test_cpp_caller_gpu(so, tmp_path):
    """The same program multiplies Fortran-layout matrices through qsgw_zmm."""
    r = subprocess.run([str(_cabi_caller(tmp_path)), "gpu"], capture_output=True, text=True)
    assert r.returncode == 0 and "OK gpu" in r.stdout, r.stdout + r.stderr


def test_header_is_plain_c(tmp_path):
    """The header compiles as strict C99 (the Fortran ISO_C_BINDING side and C
    callers see it without a C++ compiler), structs included."""
    src = tmp_path / "hdr.c"
    src.write_text('#include "qsgw_b200.h"\n'
                   "int main(void) { qsgw_sxcf_args a; qsgw_zmel_atom z; qsgw_zmel_ipw_args p;\n"
                   "  (void)a; (void)z; (void)p; return 0; }\n")
    r = subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-pedantic", "-I",
                        os.path.join(ROOT, "include"), "-c", str(src), "-o", str(tmp_path / "hdr.o")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
