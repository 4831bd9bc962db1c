"""The C-ABI libraries load and export every symbol the headers declare (CPU only:
no compute call is made)."""
import ctypes
import os
import re
import subprocess

import pytest

from conftest import ROOT

HDR = os.path.join(ROOT, "include", "mms_b200.h")


def declared_functions(path):
    src = open(path).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = set(re.findall(r"^\s*(?:const\s+)?[\w\s\*]+?\b(mms_\w+)\s*\(", src, flags=re.M))
    return sorted(n for n in names if not n.endswith("_cb"))


@pytest.fixture(scope="module")
def built():
    import mmsb200
    mmsb200.build()
    return mmsb200


def test_header_declares_the_abi():
    names = declared_functions(HDR)
    for must in ("mms_ctx_create", "mms_potential_dev", "mms_hfield_host", "mms_run_fixed", "mms_march"):
        assert must in names


def test_library_exports_every_declared_symbol(built):
    lib = ctypes.CDLL(built.LIB_PATH)
    missing = [n for n in declared_functions(HDR) if not hasattr(lib, n)]
    assert not missing, missing
    # the python binding covers the whole ABI
    assert set(declared_functions(HDR)) <= set(built.SIGNATURES)
    assert lib.mms_abi_version() == 1


def test_error_path_without_gpu_work(built):
    lib = built.load()
    # a NULL output pointer is rejected before any CUDA call
    st = lib.mms_ctx_create(None, None, None, None, None)
    assert st == built.MMS_ERR_ARG
    assert b"NULL" in lib.mms_last_error() or lib.mms_last_error()


def test_reference_signatures_exported(built):
    """libmms_refapi.so exports the reference's C++ entry points with the
    reference's mangled names (fptype = float, Vector3, byte = unsigned char)"""
    out = subprocess.run(["nm", "-D", "--defined-only", built.REFAPI_PATH], capture_output=True, text=True).stdout
    syms = set(l.split()[-1] for l in out.splitlines() if l.strip())
    demangled = subprocess.run(["c++filt"], input="\n".join(sorted(syms)), capture_output=True,
                               text=True).stdout.splitlines()
    want = [
        "fmm_calc(float const*, float*, int, int, int, float, float, float, int, int, int)",
        "calc_potential_exact(float const*, int, int, int, float, float, float, float*, int, int)",
        "calc_potential_exact_gpu(float const*, int, int, int, float, float, float, float*)",
        "Hfield(Vector3 const*, Vector3*, float*, float*, float, int, int, int, float, float, float, int, float, "
        "float, float, int, int, int, int, int, int)",
        "time_marching(unsigned char*, Vector3*, float, float, int, int, int, float, float, float, int, float, "
        "float, float, float, float, int, int, int, int, int, char const*, int)",
        "rk4_step(float, float, float*, unsigned char const*, Vector3 const*, Vector3*, Vector3*, Vector3*, "
        "Vector3*, float*, float*, int, int, int, float, float, float, int, float, float, float, float, float, "
        "int, int, int, int, int, int, int)",
    ]
    for w in want:
        assert w in demangled, w
