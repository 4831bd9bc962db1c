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


def test_struct_layouts_match_the_header(tmp_path):
    """the ctypes mirrors of the header's structs have the C compiler's size
    and field offsets (a field added in place of a reserved slot, such as
    mms_solver.near_mode, must not move the others)"""
    import mmsb200
    from mmsb200.ensemble import EnsInstance
    mirrors = {"mms_grid": mmsb200.Grid, "mms_params": mmsb200.Params, "mms_solver": mmsb200.Solver,
               "mms_controller": mmsb200.Controller, "mms_record": mmsb200.Record,
               "mms_ens_instance": EnsInstance}
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "mms_b200.h"', "int main(void) {"]
    for cname, py in mirrors.items():
        lines.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'printf("{cname}.{fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = dict(l.split() for l in subprocess.run([str(exe)], capture_output=True, text=True,
                                                 check=True).stdout.splitlines())
    for cname, py in mirrors.items():
        assert int(got[cname]) == ctypes.sizeof(py), cname
        for fname, _ in py._fields_:
            assert int(got[f"{cname}.{fname}"]) == getattr(py, fname).offset, f"{cname}.{fname}"
