"""ctypes mirrors of the plain-C structures declared in include/fftsvd_b200.h."""
from __future__ import annotations

import ctypes as C

import numpy as np

FFTSVD_MAX_DEPTH = 16

FFTSVD_OK = 0
FFTSVD_ERR_ARGUMENT = 1
FFTSVD_ERR_CUDA = 2
FFTSVD_ERR_NO_DEVICE = 3
FFTSVD_ERR_SINGULAR = 4
FFTSVD_ERR_NOT_CONVERGED = 5
FFTSVD_ERR_NONFINITE = 6
FFTSVD_ERR_TIMEOUT = 7
FFTSVD_ERR_UNSUPPORTED = 8

PREC_FP64 = 0
PREC_MIXED = 1
PREC_FP32 = 2

_i32p = C.POINTER(C.c_int32)
_i64p = C.POINTER(C.c_int64)
_f64p = C.POINTER(C.c_double)


class TreeFlat(C.Structure):
    _fields_ = [
        ("num_panels", C.c_int32), ("num_points", C.c_int32), ("depth", C.c_int32),
        ("grid", C.c_int32 * FFTSVD_MAX_DEPTH),
        ("num_leaves", C.c_int32),
        ("leaf_row_ptr", _i32p), ("leaf_rows", _i32p), ("leaf_col_ptr", _i32p), ("leaf_cols", _i32p),
        ("leaf_d_ptr", _i64p), ("d_single", _f64p), ("d_double", _f64p),
        ("num_cubes", C.c_int32),
        ("cube_level", _i32p), ("cube_index", _i32p),
        ("cube_panel_ptr", _i32p), ("cube_panels", _i32p),
        ("cube_point_ptr", _i32p), ("cube_points", _i32p),
        ("cube_row_rank", _i32p), ("cube_col_rank", _i32p),
        ("cube_vt_ptr", _i64p), ("vt", _f64p),
        ("cube_pv_ptr", _i64p), ("pv_single", _f64p), ("pv_double", _f64p),
        ("cube_uti_ptr", _i64p), ("uti", _f64p),
        ("cube_u_ptr", _i64p), ("u", _f64p),
        ("inter_ptr", _i32p), ("inter_cubes", _i32p),
        ("t_level_ptr", _i64p), ("t_ops", _f64p),
    ]


class RegionMap(C.Structure):
    _fields_ = [("phi_index", _i32p), ("phi_scale", _f64p), ("dphi_index", _i32p), ("dphi_scale", _f64p),
                ("out_index", _i32p), ("jump", _f64p)]


class PrecondCSC(C.Structure):
    _fields_ = [("n", C.c_int32), ("col_ptr", _i32p), ("row_index", _i32p), ("value", _f64p)]


class Problem(C.Structure):
    _fields_ = [
        ("num_panels", C.c_int32), ("vertices", _f64p),
        ("num_charges", C.c_int32), ("charge_pos", _f64p), ("charge", _f64p),
        ("eps_in", C.c_double), ("eps_out", C.c_double), ("kappa", C.c_double), ("svd_tol", C.c_double),
        ("max_panels_per_leaf", C.c_int32), ("grid_points", C.c_int32), ("num_threads", C.c_int32),
    ]


class SolveInfo(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("refinements", C.c_int32), ("status", C.c_int32),
                ("residual", C.c_double), ("setup_ms", C.c_double), ("solve_ms", C.c_double)]


class SurfaceStats(C.Structure):
    _fields_ = [("depth", C.c_int32 * 2), ("num_leaves", C.c_int32 * 2), ("num_cubes", C.c_int32 * 2),
                ("setup_ms", C.c_double * 8), ("device_bytes", C.c_double), ("matvec_bytes_fp32", C.c_double),
                ("matvec_bytes_fp64", C.c_double)]


TUNE_MAX_CANDIDATES = 8


class TuneInfo(C.Structure):
    _fields_ = [("candidates", C.c_int32), ("chosen", C.c_int32 * 2),
                ("max_groups", C.c_int32 * TUNE_MAX_CANDIDATES), ("max_src", C.c_int32 * TUNE_MAX_CANDIDATES),
                ("max_entries", C.c_int32 * TUNE_MAX_CANDIDATES),
                ("matvec_ms", (C.c_double * TUNE_MAX_CANDIDATES) * 2)]


# field name -> (count expression, dtype) used to copy a TreeFlat into numpy arrays
def tree_flat_to_numpy(t: TreeFlat) -> dict:
    """Copy every array of a TreeFlat into owned numpy arrays (dict keyed by field name)."""
    nl, nc, depth = t.num_leaves, t.num_cubes, t.depth

    def arr(ptr, n, dt):
        if n <= 0 or not ptr:
            return np.zeros(0, dtype=dt)
        return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dt, copy=True)

    out = {"num_panels": t.num_panels, "num_points": t.num_points, "depth": depth,
           "grid": np.array(t.grid[:depth], dtype=np.int32), "num_leaves": nl, "num_cubes": nc}
    out["leaf_row_ptr"] = arr(t.leaf_row_ptr, nl + 1, np.int32)
    out["leaf_col_ptr"] = arr(t.leaf_col_ptr, nl + 1, np.int32)
    out["leaf_d_ptr"] = arr(t.leaf_d_ptr, nl + 1, np.int64)
    out["leaf_rows"] = arr(t.leaf_rows, int(out["leaf_row_ptr"][-1]) if nl else 0, np.int32)
    out["leaf_cols"] = arr(t.leaf_cols, int(out["leaf_col_ptr"][-1]) if nl else 0, np.int32)
    nd = int(out["leaf_d_ptr"][-1]) if nl else 0
    out["d_single"] = arr(t.d_single, nd, np.float64)
    out["d_double"] = arr(t.d_double, nd, np.float64)
    out["cube_level"] = arr(t.cube_level, nc, np.int32)
    out["cube_index"] = arr(t.cube_index, 3 * nc, np.int32)
    for name in ("cube_panel_ptr", "cube_point_ptr", "inter_ptr"):
        out[name] = arr(getattr(t, name), nc + 1, np.int32)
    for name in ("cube_vt_ptr", "cube_pv_ptr", "cube_uti_ptr", "cube_u_ptr"):
        out[name] = arr(getattr(t, name), nc + 1, np.int64)
    out["cube_row_rank"] = arr(t.cube_row_rank, nc, np.int32)
    out["cube_col_rank"] = arr(t.cube_col_rank, nc, np.int32)
    out["cube_panels"] = arr(t.cube_panels, int(out["cube_panel_ptr"][-1]) if nc else 0, np.int32)
    out["cube_points"] = arr(t.cube_points, int(out["cube_point_ptr"][-1]) if nc else 0, np.int32)
    out["inter_cubes"] = arr(t.inter_cubes, int(out["inter_ptr"][-1]) if nc else 0, np.int32)
    out["vt"] = arr(t.vt, int(out["cube_vt_ptr"][-1]) if nc else 0, np.float64)
    npv = int(out["cube_pv_ptr"][-1]) if nc else 0
    out["pv_single"] = arr(t.pv_single, npv, np.float64)
    out["pv_double"] = arr(t.pv_double, npv, np.float64)
    out["uti"] = arr(t.uti, int(out["cube_uti_ptr"][-1]) if nc else 0, np.float64)
    out["u"] = arr(t.u, int(out["cube_u_ptr"][-1]) if nc else 0, np.float64)
    out["t_level_ptr"] = arr(t.t_level_ptr, depth + 1, np.int64)
    out["t_ops"] = arr(t.t_ops, 2 * int(out["t_level_ptr"][-1]), np.float64)
    return out


_ARRAY_FIELDS = {
    "leaf_row_ptr": np.int32, "leaf_rows": np.int32, "leaf_col_ptr": np.int32, "leaf_cols": np.int32,
    "leaf_d_ptr": np.int64, "d_single": np.float64, "d_double": np.float64,
    "cube_level": np.int32, "cube_index": np.int32, "cube_panel_ptr": np.int32, "cube_panels": np.int32,
    "cube_point_ptr": np.int32, "cube_points": np.int32, "cube_row_rank": np.int32,
    "cube_col_rank": np.int32, "cube_vt_ptr": np.int64, "vt": np.float64, "cube_pv_ptr": np.int64,
    "pv_single": np.float64, "pv_double": np.float64, "cube_uti_ptr": np.int64, "uti": np.float64,
    "cube_u_ptr": np.int64, "u": np.float64, "inter_ptr": np.int32, "inter_cubes": np.int32,
    "t_level_ptr": np.int64, "t_ops": np.float64,
}


def numpy_to_tree_flat(d: dict):
    """Build a TreeFlat pointing into the numpy arrays of ``d``; returns (struct, keepalive list)."""
    t = TreeFlat()
    keep = []
    t.num_panels = int(d["num_panels"])
    t.num_points = int(d["num_points"])
    t.depth = int(d["depth"])
    for i, g in enumerate(d["grid"]):
        t.grid[i] = int(g)
    t.num_leaves = int(d["num_leaves"])
    t.num_cubes = int(d["num_cubes"])
    for name, dt in _ARRAY_FIELDS.items():
        a = np.ascontiguousarray(d[name], dtype=dt)
        if a.size == 0:
            a = np.zeros(1, dtype=dt)
        keep.append(a)
        ctype = C.c_int32 if dt == np.int32 else (C.c_int64 if dt == np.int64 else C.c_double)
        setattr(t, name, a.ctypes.data_as(C.POINTER(ctype)))
    return t, keep
