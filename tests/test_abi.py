"""C-ABI checks that need no GPU: the library loads, exports every symbol the
public header declares, and reports a missing device as a status code."""
import ctypes as C
import os
import re
import subprocess

import numpy as np

import fftsvd_b200 as F
from fftsvd_b200 import _abi
from fftsvd_b200.lib import EXPORTED, LIB_PATH

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "fftsvd_b200.h")


def declared_functions():
    with open(HEADER) as f:
        text = f.read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = set(re.findall(r"\b(fftsvd_b200_\w+)\s*\(", text))
    names |= set(re.findall(r"\bvoid\s+(solveSurfaceOperator|generateRHS|collectPotentials)\s*\(", text))
    return names


def test_library_exports_every_declared_symbol():
    out = subprocess.run(["nm", "-D", "--defined-only", LIB_PATH], capture_output=True, text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    declared = declared_functions()
    assert declared, "no declarations parsed"
    assert declared <= exported, sorted(declared - exported)
    assert set(EXPORTED) == declared


def test_version_and_error_string():
    lib = F.load()
    assert lib.fftsvd_b200_version() >= 100
    assert isinstance(lib.fftsvd_b200_last_error(), bytes)


def test_struct_sizes_match_header_layout():
    # pointer-heavy structs: every field 8-byte aligned on LP64
    assert C.sizeof(_abi.RegionMap) == 6 * 8
    assert C.sizeof(_abi.PrecondCSC) == 4 * 8
    assert C.sizeof(_abi.SolveInfo) == 3 * 4 + 4 + 3 * 8


def test_null_arguments_are_rejected_without_crashing():
    lib = F.load()
    assert lib.fftsvd_b200_matvec(None, 0, None, None) == _abi.FFTSVD_ERR_ARGUMENT
    assert lib.fftsvd_b200_solve(None, 0, None, None, 1e-6, 10, None) == _abi.FFTSVD_ERR_ARGUMENT
    # the block least-squares hook checks its sizes and pointers before any device call
    for k, m, ptr in ((0, 1, 8), (257, 1, 8), (8, 0, 8), (8, 1, None)):
        p = C.c_void_p(ptr)
        assert lib.fftsvd_b200_block_ls_device(k, m, p, p, p, p, p) == _abi.FFTSVD_ERR_ARGUMENT


def test_create_without_device_reports_status():
    from conftest import has_gpu
    if has_gpu():
        return
    lib = F.load()
    h = C.c_void_p()
    n = 4
    pre = F.two_region_precond(np.ones(2), np.ones(2), 0.05)
    P = _abi.PrecondCSC(n, F.lib.ptr(F.lib.i32(pre["col_ptr"]), C.c_int32), None, None)
    rc = lib.fftsvd_b200_surface_create_flat(n, 0, None, None, C.byref(P), 0, None, None, 1.0, C.byref(h))
    assert rc in (_abi.FFTSVD_ERR_NO_DEVICE, _abi.FFTSVD_ERR_ARGUMENT)
    assert not h.value


def test_missing_library_fails_loudly(tmp_path):
    """No fallback: without the built library the package refuses to run."""
    code = ("import fftsvd_b200.lib as L\n"
            f"L.LIB_PATH = {str(tmp_path / 'absent.so')!r}\n"
            "L._lib = None\n"
            "try:\n    L.load()\nexcept ImportError as e:\n    print('raised', e)\n")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([os.sys.executable, "-c", code], cwd=root, capture_output=True, text=True, check=True)
    assert out.stdout.startswith("raised") and "is missing" in out.stdout
