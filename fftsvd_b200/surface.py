"""Host-side mirror of the reference PBE operator interface (FFTSVDpbeAPI.h:125-157).

``Surface`` owns one device-resident two-region PBE operator.  The
module-level functions keep the reference names and argument meaning:

    generateSurfaceOperator(panels, charges, ...) -> Surface     (FFTSVDpbeAPI.c:1053)
    generateRHS(surface) -> rhs[2N]                              (FFTSVDpbeAPI.c:1871)
    solveSurfaceOperator(surface, rhs, tol) -> solution[2N]      (FFTSVDpbeAPI.c:1884)
    collectPotentials(surface, solution) -> potentials (kT/e)    (FFTSVDpbeAPI.c:1896)

Where the reference calls exit() on failure (FFTSVDpbeAPI.c:38-50) these raise
FFTSVDError with the library's status code.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _abi
from ._abi import PrecondCSC, Problem, RegionMap, SolveInfo, numpy_to_tree_flat
from .lib import check, f64, i32, load, ptr

KT_CONVERSION = 561.0       # FFTSVDpbeAPI.h:13
DEBYE_CONSTANT = 3.047      # FFTSVDpbeAPI.h:14
COULOMB_KCAL = 332.112      # FFTSVDsalt.c:170

PRECISIONS = {"fp64": _abi.PREC_FP64, "mixed": _abi.PREC_MIXED, "fp32": _abi.PREC_FP32}


def _prec(p) -> int:
    return PRECISIONS[p] if isinstance(p, str) else int(p)


@dataclass
class SolveResult:
    solution: np.ndarray
    iterations: int
    refinements: int
    residual: float
    status: int
    solve_ms: float


def two_region_maps(n: int, eps_in: float, eps_out: float):
    """Region maps of the single-molecule PBE operator (SurfaceOperator.c:51-158).

    Unknowns x = [phi(0..n-1); dphi(0..n-1)].  Tree 0 is the exterior region
    (no own panels, its child's panels enter with phi -> -phi,
    dphi -> eps_in/eps_out dphi, result to the dphi rows, plus the -4 pi phi
    jump); tree 1 is the interior region (phi -> phi, dphi -> -dphi, result to
    the phi rows).
    """
    k = np.arange(n, dtype=np.int32)
    outer = dict(phi_index=k, phi_scale=np.full(n, -1.0), dphi_index=k + n,
                 dphi_scale=np.full(n, eps_in / eps_out), out_index=k + n, jump=np.full(n, -4.0 * np.pi))
    inner = dict(phi_index=k, phi_scale=np.ones(n), dphi_index=k + n, dphi_scale=np.full(n, -1.0),
                 out_index=k, jump=np.zeros(n))
    return [outer, inner]


def two_region_precond(diag_single: np.ndarray, diag_double: np.ndarray, rel_eps: float):
    """Per-panel 2x2 preconditioner blocks (SurfaceOperator.c:170-197) in CSC form.

    Rows/columns (phi_i, dphi_i):  [[Dd, -Ds], [Dd, rel_eps * Ds]] with the
    interior tree's self terms Ds = D_single(i,i), Dd = D_double(i,i).
    """
    n = len(diag_single)
    col_ptr = np.arange(0, 4 * n + 1, 2, dtype=np.int32)
    rows = np.empty(4 * n, dtype=np.int32)
    vals = np.empty(4 * n)
    i = np.arange(n)
    # column phi_i: rows phi_i, dphi_i
    rows[2 * i] = i
    rows[2 * i + 1] = n + i
    vals[2 * i] = diag_double
    vals[2 * i + 1] = diag_double
    # column dphi_i: rows phi_i, dphi_i
    rows[2 * (n + i)] = i
    rows[2 * (n + i) + 1] = n + i
    vals[2 * (n + i)] = -diag_single
    vals[2 * (n + i) + 1] = rel_eps * diag_single
    return dict(n=2 * n, col_ptr=col_ptr, row_index=rows, value=vals)


def leaf_diagonals(tree: dict):
    """Self terms D(i,i) of every panel from a flat tree (Cube.c:2349-2390)."""
    n = tree["num_points"]
    ds = np.zeros(n)
    dd = np.zeros(n)
    rp, cp, dp = tree["leaf_row_ptr"], tree["leaf_col_ptr"], tree["leaf_d_ptr"]
    for l in range(tree["num_leaves"]):
        nr = rp[l + 1] - rp[l]
        nc = cp[l + 1] - cp[l]
        rows = tree["leaf_rows"][rp[l]:rp[l + 1]]
        blk_s = tree["d_single"][dp[l]:dp[l + 1]].reshape(nr, nc)
        blk_d = tree["d_double"][dp[l]:dp[l + 1]].reshape(nr, nc)
        r = np.arange(nr)
        ds[rows] = blk_s[r, r]
        dd[rows] = blk_d[r, r]
    return ds, dd


class Surface:
    """A device-resident PBE surface operator (both FP32 and FP64 copies)."""

    def __init__(self, handle, n_unknowns: int, keep=None, num_charges: int = 0, eps_in: float = 1.0):
        self._h = handle
        self.n = n_unknowns
        self._keep = keep
        self.num_charges = num_charges
        self.eps_in = eps_in

    # ---- construction
    @classmethod
    def from_flat(cls, trees, maps, precond, charge_pos=None, charge=None, eps_in=1.0, vertices=None,
                  geometry_rows=None):
        lib = load()
        n_unknowns = int(precond["n"])
        keep = []
        tf = (_abi.TreeFlat * len(trees))()
        for i, t in enumerate(trees):
            s, k = numpy_to_tree_flat(t)
            tf[i] = s
            keep.append(k)
        rm = (RegionMap * len(maps))()
        for i, m in enumerate(maps):
            arrs = {"phi_index": i32(m["phi_index"]), "phi_scale": f64(m["phi_scale"]),
                    "dphi_index": i32(m["dphi_index"]), "dphi_scale": f64(m["dphi_scale"]),
                    "out_index": i32(m["out_index"]), "jump": f64(m["jump"])}
            keep.append(arrs)
            rm[i] = RegionMap(ptr(arrs["phi_index"], C.c_int32), ptr(arrs["phi_scale"]),
                              ptr(arrs["dphi_index"], C.c_int32), ptr(arrs["dphi_scale"]),
                              ptr(arrs["out_index"], C.c_int32), ptr(arrs["jump"]))
        pc = {"col_ptr": i32(precond["col_ptr"]), "row_index": i32(precond["row_index"]),
              "value": f64(precond["value"])}
        keep.append(pc)
        P = PrecondCSC(n_unknowns, ptr(pc["col_ptr"], C.c_int32), ptr(pc["row_index"], C.c_int32), ptr(pc["value"]))
        nq = 0 if charge is None else len(charge)
        qp = f64(charge_pos if nq else np.zeros((1, 3)))
        qv = f64(charge if nq else np.zeros(1))
        h = C.c_void_p()
        check(lib.fftsvd_b200_surface_create_flat(n_unknowns, len(trees), tf, rm, C.byref(P), nq, ptr(qp), ptr(qv),
                                                  float(eps_in), C.byref(h)))
        s = cls(h, n_unknowns, None, nq, eps_in)
        if vertices is not None:
            vv = f64(vertices)
            npan = len(vv)
            if geometry_rows is None:
                geometry_rows = (np.arange(npan), np.arange(npan) + npan)
            pr, dr = i32(geometry_rows[0]), i32(geometry_rows[1])
            check(lib.fftsvd_b200_set_geometry(h, npan, ptr(vv), ptr(pr, C.c_int32), ptr(dr, C.c_int32)))
        return s

    @classmethod
    def from_problem(cls, vertices, charge_pos, charge, eps_in, eps_out, kappa, svd_tol=1e-5,
                     max_panels_per_leaf=32, grid_points=4, num_threads=0):
        """Own host setup (octree, panel integrals, sampled SVD bases, translation operators)."""
        lib = load()
        vv, qp, qv = f64(vertices), f64(charge_pos), f64(charge)
        p = Problem(len(vv), ptr(vv), len(qv), ptr(qp), ptr(qv), float(eps_in), float(eps_out), float(kappa),
                    float(svd_tol), int(max_panels_per_leaf), int(grid_points), int(num_threads))
        h = C.c_void_p()
        check(lib.fftsvd_b200_surface_create(C.byref(p), C.byref(h)))
        return cls(h, 2 * len(vv), None, len(qv), eps_in)

    def close(self):
        if self._h:
            load().fftsvd_b200_surface_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- operations (host arrays)
    def matvec(self, x, precision="fp32"):
        x = f64(x)
        y = np.empty(self.n)
        check(load().fftsvd_b200_matvec(self._h, _prec(precision), x.ctypes.data, y.ctypes.data))
        return y

    def precond_solve(self, r):
        r = f64(r)
        z = np.empty(self.n)
        check(load().fftsvd_b200_precond_solve(self._h, ptr(r), ptr(z)))
        return z

    def solve(self, rhs, precision="mixed", tol=1e-6, max_iterations=1000, raise_on_error=True) -> SolveResult:
        rhs = f64(rhs)
        sol = np.empty(self.n)
        info = SolveInfo()
        rc = load().fftsvd_b200_solve(self._h, _prec(precision), rhs.ctypes.data, sol.ctypes.data, float(tol),
                                      int(max_iterations), C.byref(info))
        if raise_on_error:
            check(rc)
        return SolveResult(sol, info.iterations, info.refinements, info.residual, rc, info.solve_ms)

    def rhs(self):
        r = np.empty(self.n)
        check(load().fftsvd_b200_rhs(self._h, ptr(r)))
        return r

    def reaction_potentials(self, solution):
        s = f64(solution)
        phi = np.empty(self.num_charges)
        check(load().fftsvd_b200_reaction_potentials(self._h, ptr(s), ptr(phi)))
        return phi

    def energy(self, phi):
        phi = f64(phi)
        e = C.c_double()
        check(load().fftsvd_b200_energy(self._h, ptr(phi), C.byref(e)))
        return e.value

    def matvec_bytes(self, precision="fp32") -> float:
        b = C.c_double()
        check(load().fftsvd_b200_matvec_bytes(self._h, _prec(precision), C.byref(b)))
        return b.value

    def autotune(self) -> dict:
        """Time the matvec of both operator precisions under each candidate translation tile
        shape and keep the fastest (results are unchanged bit for bit).  Returns the
        candidates, their times and the chosen index per precision."""
        info = _abi.TuneInfo()
        check(load().fftsvd_b200_surface_autotune(self._h, C.byref(info)))
        k = info.candidates
        return {
            "candidates": [(info.max_groups[c], info.max_src[c], info.max_entries[c]) for c in range(k)],
            "matvec_ms_fp32": [info.matvec_ms[0][c] for c in range(k)],
            "matvec_ms_fp64": [info.matvec_ms[1][c] for c in range(k)],
            "chosen_fp32": info.chosen[0],
            "chosen_fp64": info.chosen[1],
        }

    def set_tile_limits(self, max_groups=32, max_src=320, max_entries=3072):
        """Rebuild the translation tiles under explicit limits (launch shapes only)."""
        check(load().fftsvd_b200_surface_set_tile_limits(self._h, int(max_groups), int(max_src), int(max_entries)))

    # ---- operations on device pointers (torch tensors or raw ints)
    def matvec_device(self, x_ptr: int, y_ptr: int, precision="fp32"):
        check(load().fftsvd_b200_matvec_device(self._h, _prec(precision), C.c_void_p(x_ptr), C.c_void_p(y_ptr)))

    def solve_device(self, rhs_ptr: int, sol_ptr: int, precision="mixed", tol=1e-6, max_iterations=1000):
        info = SolveInfo()
        rc = load().fftsvd_b200_solve_device(self._h, _prec(precision), C.c_void_p(rhs_ptr), C.c_void_p(sol_ptr),
                                             float(tol), int(max_iterations), C.byref(info))
        check(rc)
        return info

    def rhs_device(self, rhs_ptr: int):
        check(load().fftsvd_b200_rhs_device(self._h, C.c_void_p(rhs_ptr)))

    def reaction_potentials_device(self, sol_ptr: int, phi_ptr: int):
        check(load().fftsvd_b200_reaction_potentials_device(self._h, C.c_void_p(sol_ptr), C.c_void_p(phi_ptr)))

    # ---- adjoint
    def set_charges(self, charge_pos, charge):
        qp, qv = f64(charge_pos), f64(charge)
        check(load().fftsvd_b200_set_charges(self._h, len(qv), ptr(qp), ptr(qv)))
        self.num_charges = len(qv)

    def matvec_transpose(self, x, precision="fp64"):
        x = f64(x)
        y = np.empty(self.n)
        check(load().fftsvd_b200_matvec_transpose(self._h, _prec(precision), ptr(x), ptr(y)))
        return y

    def adjoint(self, precision="fp64", tol=1e-6, max_iterations=1000):
        """Solvation energy and its derivatives: (dG, dG/dq [nq], dG/dx [nq, 3], (forward, adjoint) SolveInfo)."""
        nq = self.num_charges
        e = C.c_double()
        dq = np.empty(max(nq, 1))
        dx = np.empty(max(3 * nq, 1))
        info = (SolveInfo * 2)()
        check(load().fftsvd_b200_adjoint(self._h, _prec(precision), float(tol), int(max_iterations), C.byref(e),
                                         ptr(dq), ptr(dx), info))
        return e.value, dq[:nq].copy(), dx[:3 * nq].reshape(nq, 3).copy(), (info[0], info[1])

    # ---- many right-hand sides (blocks of k vectors, one after the other)
    def matvec_batch_device(self, x_ptr: int, y_ptr: int, nrhs: int, precision="fp32"):
        check(load().fftsvd_b200_matvec_batch_device(self._h, _prec(precision), int(nrhs), C.c_void_p(x_ptr),
                                                     C.c_void_p(y_ptr)))

    def solve_batch_device(self, rhs_ptr: int, sol_ptr: int, nrhs: int, precision="mixed", tol=1e-6,
                           max_iterations=1000, raise_on_error=True):
        """Returns the per-column SolveInfo array."""
        info = (SolveInfo * int(nrhs))()
        rc = load().fftsvd_b200_solve_batch_device(self._h, int(nrhs), _prec(precision), C.c_void_p(rhs_ptr),
                                                   C.c_void_p(sol_ptr), float(tol), int(max_iterations), info)
        if raise_on_error:
            check(rc)
        return info

    def solve_batch(self, rhs, precision="mixed", tol=1e-6, max_iterations=1000, raise_on_error=True):
        """rhs: (k, n) host array.  Returns (solutions (k, n), per-column SolveInfo array)."""
        rhs = np.ascontiguousarray(rhs, dtype=np.float64)
        k = rhs.shape[0]
        sol = np.empty_like(rhs)
        info = (SolveInfo * k)()
        rc = load().fftsvd_b200_solve_batch(self._h, k, _prec(precision), rhs.ctypes.data, sol.ctypes.data,
                                            float(tol), int(max_iterations), info)
        if raise_on_error:
            check(rc)
        return sol, info

    def solve_block_device(self, rhs_ptr: int, sol_ptr: int, nrhs: int, precision="mixed", tol=1e-6,
                           max_iterations=1000, raise_on_error=True):
        """Block GMRES over one shared Krylov space; returns the per-column SolveInfo array."""
        info = (SolveInfo * int(nrhs))()
        rc = load().fftsvd_b200_solve_block_device(self._h, int(nrhs), _prec(precision), C.c_void_p(rhs_ptr),
                                                   C.c_void_p(sol_ptr), float(tol), int(max_iterations), info)
        if raise_on_error:
            check(rc)
        return info

    def solve_block(self, rhs, precision="mixed", tol=1e-6, max_iterations=1000, raise_on_error=True):
        """Block GMRES; rhs: (k, n) host array.  Returns (solutions (k, n), per-column SolveInfo array)."""
        rhs = np.ascontiguousarray(rhs, dtype=np.float64)
        k = rhs.shape[0]
        sol = np.empty_like(rhs)
        info = (SolveInfo * k)()
        rc = load().fftsvd_b200_solve_block(self._h, k, _prec(precision), rhs.ctypes.data, sol.ctypes.data,
                                            float(tol), int(max_iterations), info)
        if raise_on_error:
            check(rc)
        return sol, info

    def rhs_groups_device(self, group_ptr, rhs_ptr: int):
        gp = i32(group_ptr)
        check(load().fftsvd_b200_rhs_groups_device(self._h, len(gp) - 1, ptr(gp, C.c_int32), C.c_void_p(rhs_ptr)))

    def group_energies_device(self, group_ptr, sol_ptr: int):
        gp = i32(group_ptr)
        e = np.empty(len(gp) - 1)
        check(load().fftsvd_b200_group_energies_device(self._h, len(gp) - 1, ptr(gp, C.c_int32), C.c_void_p(sol_ptr),
                                                       ptr(e)))
        return e


def solve_many(surfaces, rhs_ptrs, sol_ptrs, precision="mixed", tol=1e-6, max_iterations=1000, raise_on_error=True):
    """Solve several surfaces concurrently (device vectors per surface).  Returns the SolveInfo array."""
    k = len(surfaces)
    hs = (C.c_void_p * k)(*[s._h for s in surfaces])
    rp = (C.c_void_p * k)(*[C.c_void_p(int(p)) for p in rhs_ptrs])
    xp = (C.c_void_p * k)(*[C.c_void_p(int(p)) for p in sol_ptrs])
    info = (SolveInfo * k)()
    rc = load().fftsvd_b200_solve_many(k, hs, rp, xp, _prec(precision), float(tol), int(max_iterations), info)
    if raise_on_error:
        check(rc)
    return info


def host_operator(vertices, eps_in, eps_out, kappa, svd_tol=1e-5, max_panels_per_leaf=32, grid_points=4,
                  num_threads=0, integrals="host", timings=None):
    """Run only the setup: returns ([exterior tree, interior tree], preconditioner) as numpy.
    integrals: "host" (fftsvd_b200_host_setup), "device" (the panel integrals in batches
    on the current CUDA device, fftsvd_b200_device_setup) or "batched" (the device path's
    batches evaluated on the host, fftsvd_b200_host_setup_batched).  A dict passed as
    timings receives the wall milliseconds of the setup stages."""
    lib = load()
    vv = f64(vertices)
    zero3, zero1 = np.zeros(3), np.zeros(1)
    p = Problem(len(vv), ptr(vv), 0, ptr(zero3), ptr(zero1), float(eps_in), float(eps_out), float(kappa),
                float(svd_tol), int(max_panels_per_leaf), int(grid_points), int(num_threads))
    h = C.c_void_p()
    setup = {"host": lib.fftsvd_b200_host_setup, "device": lib.fftsvd_b200_device_setup,
             "batched": lib.fftsvd_b200_host_setup_batched}[integrals]
    check(setup(C.byref(p), C.byref(h)))
    try:
        if timings is not None:
            ms = np.zeros(6)
            check(lib.fftsvd_b200_host_operator_timings(h, ptr(ms)))
            timings.update(zip(["partition", "near", "pinv_t", "bases", "flatten", "integrals"], ms.tolist()))
        trees = []
        for t in range(2):
            tf = _abi.TreeFlat()
            check(lib.fftsvd_b200_host_operator_tree(h, t, C.byref(tf)))
            trees.append(_abi.tree_flat_to_numpy(tf))
        pc = PrecondCSC()
        check(lib.fftsvd_b200_host_operator_precond(h, C.byref(pc)))
        n = pc.n
        col_ptr = np.ctypeslib.as_array(pc.col_ptr, shape=(n + 1,)).copy()
        nnz = int(col_ptr[-1])
        pre = dict(n=n, col_ptr=col_ptr, row_index=np.ctypeslib.as_array(pc.row_index, shape=(nnz,)).copy(),
                   value=np.ctypeslib.as_array(pc.value, shape=(nnz,)).copy())
    finally:
        lib.fftsvd_b200_host_operator_free(h)
    return trees, pre


# ---- reference-named entry points

def generateSurfaceOperator(vertices, charge_pos, charge, innerdielectric, outerdielectric, ionicstrength=0.0,
                            svd_tol=1e-5, max_panels_per_leaf=32, grid_points=4) -> Surface:
    """Two-region PBE operator; kappa = sqrt(I)/3.047 as in FFTSVDpbeAPI.c:1060."""
    kappa = np.sqrt(ionicstrength) / DEBYE_CONSTANT if ionicstrength > 0 else 0.0
    return Surface.from_problem(vertices, charge_pos, charge, innerdielectric, outerdielectric, kappa, svd_tol,
                                max_panels_per_leaf, grid_points)


def generateRHS(surface: Surface) -> np.ndarray:
    return surface.rhs()


def solveSurfaceOperator(surface: Surface, rhs, errortolerance=1e-6, precision="mixed") -> np.ndarray:
    return surface.solve(rhs, precision=precision, tol=errortolerance).solution


def collectPotentials(surface: Surface, solution) -> np.ndarray:
    """Reaction potentials at the charges in kT/e (KT_CONVERSION * phi / eps_in)."""
    return KT_CONVERSION * surface.reaction_potentials(solution) / surface.eps_in


def solvation_energy(surface: Surface, solution) -> float:
    """0.5 * sum q phi_reac * 332.112 / eps_in in kcal/mol."""
    return surface.energy(surface.reaction_potentials(solution))
