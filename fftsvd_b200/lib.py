"""ctypes binding of libfftsvd_b200.so (the in-tree CUDA library).

The library is required: importing this module on a machine without the
built .so raises immediately, and every call that needs a GPU fails with
FFTSVDError(FFTSVD_ERR_NO_DEVICE) instead of falling back to host code.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _abi
from ._abi import PrecondCSC, Problem, RegionMap, SolveInfo, TreeFlat

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libfftsvd_b200.so")

_f64p = C.POINTER(C.c_double)
_i32p = C.POINTER(C.c_int32)

# every symbol declared in include/fftsvd_b200.h
EXPORTED = [
    "fftsvd_b200_last_error", "fftsvd_b200_version", "fftsvd_b200_surface_create",
    "fftsvd_b200_surface_create_flat", "fftsvd_b200_surface_free", "fftsvd_b200_surface_num_unknowns",
    "fftsvd_b200_matvec", "fftsvd_b200_matvec_device", "fftsvd_b200_precond_solve", "fftsvd_b200_solve",
    "fftsvd_b200_solve_device", "fftsvd_b200_set_geometry", "fftsvd_b200_rhs", "fftsvd_b200_rhs_device",
    "fftsvd_b200_reaction_potentials", "fftsvd_b200_reaction_potentials_device", "fftsvd_b200_energy",
    "fftsvd_b200_matvec_bytes", "fftsvd_b200_surface_stats", "fftsvd_b200_host_setup",
    "fftsvd_b200_host_operator_tree", "fftsvd_b200_device_setup", "fftsvd_b200_host_setup_batched",
    "fftsvd_b200_host_operator_timings", "fftsvd_b200_host_operator_precond", "fftsvd_b200_host_operator_free",
    "fftsvd_b200_matvec_kernel_bytes", "fftsvd_b200_translate_smem_bytes", "fftsvd_b200_profile_matvec", "fftsvd_b200_surface_stream",
    "fftsvd_b200_launch_count", "fftsvd_b200_device_alloc_count", "fftsvd_b200_bounded_wait_selftest", "fftsvd_b200_dense_gemm_device",
    "fftsvd_b200_dense_trsm_device", "fftsvd_b200_block_ls_device", "fftsvd_b200_reaction_potentials_noalloc",
    "solveSurfaceOperator", "generateRHS",
    "collectPotentials",
    "fftsvd_b200_matvec_batch_device", "fftsvd_b200_matvec_batch_tensor_device", "fftsvd_b200_solve_batch_device",
    "fftsvd_b200_solve_batch",
    "fftsvd_b200_rhs_groups_device", "fftsvd_b200_group_energies_device",
    "fftsvd_b200_set_charges", "fftsvd_b200_matvec_transpose", "fftsvd_b200_matvec_transpose_device",
    "fftsvd_b200_adjoint", "fftsvd_b200_solve_many", "fftsvd_b200_surface_autotune",
    "fftsvd_b200_surface_set_tile_limits", "fftsvd_b200_solve_block_device", "fftsvd_b200_solve_block",
]


class FFTSVDError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"[{code}] {message}")
        self.code = code


_lib = None


def load():
    """Load the CUDA library (once).  Raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m fftsvd_b200.build`")
    lib = C.CDLL(LIB_PATH)
    lib.fftsvd_b200_last_error.restype = C.c_char_p
    lib.fftsvd_b200_version.restype = C.c_int
    sp = C.c_void_p
    lib.fftsvd_b200_surface_create.argtypes = [C.POINTER(Problem), C.POINTER(sp)]
    lib.fftsvd_b200_surface_create_flat.argtypes = [C.c_int32, C.c_int32, C.POINTER(TreeFlat), C.POINTER(RegionMap),
                                                    C.POINTER(PrecondCSC), C.c_int32, _f64p, _f64p, C.c_double,
                                                    C.POINTER(sp)]
    lib.fftsvd_b200_surface_free.argtypes = [sp]
    lib.fftsvd_b200_surface_num_unknowns.argtypes = [sp]
    lib.fftsvd_b200_surface_num_unknowns.restype = C.c_int32
    for name in ("fftsvd_b200_matvec", "fftsvd_b200_matvec_device"):
        getattr(lib, name).argtypes = [sp, C.c_int32, C.c_void_p, C.c_void_p]
    lib.fftsvd_b200_precond_solve.argtypes = [sp, _f64p, _f64p]
    for name in ("fftsvd_b200_solve", "fftsvd_b200_solve_device"):
        getattr(lib, name).argtypes = [sp, C.c_int32, C.c_void_p, C.c_void_p, C.c_double, C.c_int32,
                                       C.POINTER(SolveInfo)]
    lib.fftsvd_b200_set_geometry.argtypes = [sp, C.c_int32, _f64p, _i32p, _i32p]
    lib.fftsvd_b200_rhs.argtypes = [sp, _f64p]
    lib.fftsvd_b200_rhs_device.argtypes = [sp, C.c_void_p]
    lib.fftsvd_b200_reaction_potentials.argtypes = [sp, _f64p, _f64p]
    lib.fftsvd_b200_reaction_potentials_device.argtypes = [sp, C.c_void_p, C.c_void_p]
    lib.fftsvd_b200_energy.argtypes = [sp, _f64p, _f64p]
    lib.fftsvd_b200_matvec_bytes.argtypes = [sp, C.c_int32, _f64p]
    lib.fftsvd_b200_surface_stats.argtypes = [sp, C.POINTER(_abi.SurfaceStats)]
    lib.fftsvd_b200_host_setup.argtypes = [C.POINTER(Problem), C.POINTER(sp)]
    lib.fftsvd_b200_device_setup.argtypes = [C.POINTER(Problem), C.POINTER(sp)]
    lib.fftsvd_b200_host_setup_batched.argtypes = [C.POINTER(Problem), C.POINTER(sp)]
    lib.fftsvd_b200_host_operator_timings.argtypes = [sp, _f64p]
    lib.fftsvd_b200_host_operator_tree.argtypes = [sp, C.c_int32, C.POINTER(TreeFlat)]
    lib.fftsvd_b200_host_operator_precond.argtypes = [sp, C.POINTER(PrecondCSC)]
    lib.fftsvd_b200_host_operator_free.argtypes = [sp]
    lib.fftsvd_b200_matvec_kernel_bytes.argtypes = [sp, C.c_int32, _f64p]
    lib.fftsvd_b200_translate_smem_bytes.argtypes = [sp, C.c_int32, _f64p]
    lib.fftsvd_b200_profile_matvec.argtypes = [sp, C.c_int32, C.c_void_p, C.c_void_p, C.c_int32, _f64p]
    lib.fftsvd_b200_surface_stream.argtypes = [sp]
    lib.fftsvd_b200_surface_stream.restype = C.c_void_p
    lib.fftsvd_b200_launch_count.restype = C.c_longlong
    lib.fftsvd_b200_device_alloc_count.restype = C.c_longlong
    lib.fftsvd_b200_bounded_wait_selftest.argtypes = [C.c_int32]
    lib.fftsvd_b200_dense_gemm_device.argtypes = [C.c_int, C.c_int64, C.c_int32, C.c_int64, C.c_double, C.c_void_p,
                                                  C.c_int64, C.c_void_p, C.c_int64, C.c_double, C.c_void_p, C.c_int64]
    lib.fftsvd_b200_dense_trsm_device.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_int64, C.c_void_p,
                                                  C.c_void_p]
    lib.fftsvd_b200_block_ls_device.argtypes = [C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                                C.c_void_p]
    lib.fftsvd_b200_reaction_potentials_noalloc.argtypes = [sp, C.c_void_p, C.c_void_p]
    lib.fftsvd_b200_matvec_batch_device.argtypes = [sp, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p]
    lib.fftsvd_b200_matvec_batch_tensor_device.argtypes = [sp, C.c_int32, C.c_void_p, C.c_void_p]
    for name in ("fftsvd_b200_solve_batch_device", "fftsvd_b200_solve_batch", "fftsvd_b200_solve_block_device",
                 "fftsvd_b200_solve_block"):
        getattr(lib, name).argtypes = [sp, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_double, C.c_int32,
                                       C.POINTER(SolveInfo)]
    lib.fftsvd_b200_rhs_groups_device.argtypes = [sp, C.c_int32, _i32p, C.c_void_p]
    lib.fftsvd_b200_group_energies_device.argtypes = [sp, C.c_int32, _i32p, C.c_void_p, _f64p]
    lib.fftsvd_b200_set_charges.argtypes = [sp, C.c_int32, _f64p, _f64p]
    lib.fftsvd_b200_solve_many.argtypes = [C.c_int32, C.POINTER(sp), C.POINTER(C.c_void_p), C.POINTER(C.c_void_p),
                                           C.c_int32, C.c_double, C.c_int32, C.POINTER(SolveInfo)]
    lib.fftsvd_b200_matvec_transpose.argtypes = [sp, C.c_int32, _f64p, _f64p]
    lib.fftsvd_b200_surface_autotune.argtypes = [sp, C.POINTER(_abi.TuneInfo)]
    lib.fftsvd_b200_surface_set_tile_limits.argtypes = [sp, C.c_int32, C.c_int32, C.c_int32]
    lib.fftsvd_b200_matvec_transpose_device.argtypes = [sp, C.c_int32, C.c_void_p, C.c_void_p]
    lib.fftsvd_b200_adjoint.argtypes = [sp, C.c_int32, C.c_double, C.c_int32, _f64p, _f64p, _f64p,
                                        C.POINTER(SolveInfo)]
    _lib = lib
    return lib


def check(rc: int) -> None:
    if rc != _abi.FFTSVD_OK:
        msg = load().fftsvd_b200_last_error()
        raise FFTSVDError(rc, msg.decode() if msg else "")


def f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def i32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.int32)


def ptr(a: np.ndarray, ctype=C.c_double):
    return a.ctypes.data_as(C.POINTER(ctype))
