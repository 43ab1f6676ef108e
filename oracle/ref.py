"""ORACLE — test infrastructure only (never imported by the product path).

ctypes access to the reference FFTSVD C code compiled by oracle/Makefile into
oracle/_ref/ (libfftsvd_ref.so: as shipped, FP32 operator storage;
libfftsvd_ref64.so: FP64 operator storage).  See oracle/ref_driver.c for the
reference functions behind each call.

The reference prints progress and every GMRES residual to stdout
(GMRES.c:505-507); calls are wrapped so that this output goes to stderr and a
caller's stdout stays clean.
"""
from __future__ import annotations

import contextlib
import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
# the reference source tree (read-only; only the oracle build and the CPU tests that
# compile against its headers read it): FFTSVD_REFERENCE, else the Makefile's default
REFERENCE_TREE = os.environ.get("FFTSVD_REFERENCE") or "/root/reference"
sys.path.insert(0, os.path.dirname(HERE))
from fftsvd_b200._abi import TreeFlat, tree_flat_to_numpy  # noqa: E402

_f64p = C.POINTER(C.c_double)
_libs = {}


def library_path(fp64: bool) -> str:
    """The compiled reference; FFTSVD_REF_LIB names another build of it (the CPU baseline
    table times the as-shipped build through it)."""
    if not fp64 and os.environ.get("FFTSVD_REF_LIB"):
        return os.environ["FFTSVD_REF_LIB"]
    return os.path.join(REF_DIR, "libfftsvd_ref64.so" if fp64 else "libfftsvd_ref.so")


def available(fp64: bool = False) -> bool:
    return os.path.exists(library_path(fp64))


def _lib(fp64: bool):
    key = bool(fp64)
    if key not in _libs:
        lib = C.CDLL(library_path(fp64))
        lib.oref_create.restype = C.c_void_p
        lib.oref_create.argtypes = [C.c_uint, _f64p, C.c_uint, _f64p, _f64p, C.c_double, C.c_double, C.c_double,
                                    C.c_double, C.c_uint, C.c_uint]
        lib.oref_create_api.restype = C.c_void_p
        lib.oref_create_api.argtypes = [C.c_uint, _f64p, C.c_uint, _f64p, _f64p, C.c_double, C.c_double,
                                        C.c_double, C.c_double]
        lib.oref_free.argtypes = [C.c_void_p]
        lib.oref_surface_operator.restype = C.c_void_p
        lib.oref_surface_operator.argtypes = [C.c_void_p]
        lib.oref_preconditioner.restype = C.c_void_p
        lib.oref_preconditioner.argtypes = [C.c_void_p]
        lib.oref_num_panels.restype = C.c_uint
        lib.oref_num_panels.argtypes = [C.c_void_p]
        lib.oref_depth.restype = C.c_uint
        lib.oref_depth.argtypes = [C.c_void_p, C.c_int]
        lib.oref_matvec.argtypes = [C.c_void_p, _f64p, _f64p]
        lib.oref_tree_multiplyboth.argtypes = [C.c_void_p, C.c_int, _f64p, _f64p, _f64p]
        lib.oref_precond_solve.argtypes = [C.c_void_p, _f64p, _f64p]
        lib.oref_rhs.argtypes = [C.c_void_p, _f64p]
        lib.oref_gmres.restype = C.c_int
        lib.oref_gmres.argtypes = [C.c_void_p, _f64p, _f64p, C.c_double]
        lib.oref_reaction.argtypes = [C.c_void_p, _f64p, _f64p]
        lib.oref_energy.restype = C.c_double
        lib.oref_energy.argtypes = [C.c_void_p, _f64p]
        lib.oref_panel_integrals.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_uint, _f64p,
                                             C.POINTER(C.c_uint), _f64p, _f64p]
        lib.oref_export_tree.restype = C.c_int
        lib.oref_export_tree.argtypes = [C.c_void_p, C.c_int, C.POINTER(TreeFlat)]
        lib.oref_export_free.argtypes = [C.POINTER(TreeFlat)]
        _libs[key] = lib
    return _libs[key]


@contextlib.contextmanager
def stdout_to_stderr():
    """Route fd 1 to fd 2 while the reference prints."""
    sys.stdout.flush()
    saved = os.dup(1)
    try:
        os.dup2(2, 1)
        yield
    finally:
        C.CDLL(None).fflush(None)
        os.dup2(saved, 1)
        os.close(saved)


def _p(a):
    return a.ctypes.data_as(_f64p)


class PDBentry(C.Structure):
    """FFTSVDpbeAPI.h:23-42, the atom record collectPotentials reads and writes."""
    _fields_ = [("record", C.c_char * 7), ("atomnumber", C.c_uint), ("atomname", C.c_char * 5),
                ("alternatelocation", C.c_char), ("residuename", C.c_char * 4), ("chain", C.c_char),
                ("residuenumber", C.c_uint), ("residueinsertion", C.c_char), ("x", C.c_double),
                ("y", C.c_double), ("z", C.c_double), ("occupancy", C.c_double), ("temperature", C.c_double),
                ("footnotenumber", C.c_uint), ("radius", C.c_double), ("charge", C.c_double),
                ("potential", C.c_double)]


def pdb_entries(pos, charge=None, chain=b"A", potential=0.0):
    """A PDBentry array with the given positions, charges and chain letters."""
    pos = np.asarray(pos, dtype=np.float64).reshape(-1, 3)
    arr = (PDBentry * len(pos))()
    for i, p in enumerate(pos):
        e = arr[i]
        e.x, e.y, e.z = float(p[0]), float(p[1]), float(p[2])
        e.charge = 0.0 if charge is None else float(charge[i])
        e.chain = chain[i] if isinstance(chain, (list, tuple)) else chain
        e.potential = potential
    return arr


def export_api_globals(fp64: bool = False) -> None:
    """Put the compiled reference's symbols, among them the API's process globals
    (innerdielectric, addcoulombic; FFTSVDpbeAPI.c:18-34), into the process-wide
    symbol scope, as a program linked with the reference objects has them."""
    _lib(fp64)
    C.CDLL(library_path(fp64), mode=os.RTLD_GLOBAL | os.RTLD_NOLOAD)


def set_threads(n: int) -> None:
    """OpenMP threads used by the reference's parallel regions (Tree.c:630-656)."""
    os.environ["OMP_NUM_THREADS"] = str(n)
    try:
        C.CDLL("libgomp.so.1").omp_set_num_threads(int(n))
    except OSError:
        pass


class RefSystem:
    """The reference two-region PBE operator (outer region: tree 0, inner: tree 1)."""

    def __init__(self, tri, qpos, q, eps_in, eps_out, kappa, svd_tol=1e-5, max_panels=32, grid=4,
                 fp64=False, via_api=False, gmres_tol=1e-6):
        self.fp64 = fp64
        self.lib = _lib(fp64)
        self.tri = np.ascontiguousarray(tri, dtype=np.float64)
        self.qpos = np.ascontiguousarray(qpos, dtype=np.float64)
        self.q = np.ascontiguousarray(q, dtype=np.float64)
        self.n = len(self.tri)
        self.nq = len(self.q)
        with stdout_to_stderr():
            if via_api:
                ionic = (kappa * 3.047) ** 2
                self.h = self.lib.oref_create_api(self.n, _p(self.tri), self.nq, _p(self.qpos), _p(self.q),
                                                  eps_in, eps_out, ionic, gmres_tol)
            else:
                self.h = self.lib.oref_create(self.n, _p(self.tri), self.nq, _p(self.qpos), _p(self.q),
                                              eps_in, eps_out, kappa, svd_tol, max_panels, grid)

    def close(self):
        if self.h:
            self.lib.oref_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def surface_operator(self):
        return self.lib.oref_surface_operator(self.h)

    @property
    def preconditioner(self):
        return self.lib.oref_preconditioner(self.h)

    def depth(self, which):
        return int(self.lib.oref_depth(self.h, which))

    def matvec(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.zeros(2 * self.n)
        self.lib.oref_matvec(self.h, _p(x), _p(y))
        return y

    def tree_multiplyboth(self, which, xs, xd):
        xs = np.ascontiguousarray(xs, dtype=np.float64)
        xd = np.ascontiguousarray(xd, dtype=np.float64)
        b = np.zeros(self.n)
        self.lib.oref_tree_multiplyboth(self.h, which, _p(xs), _p(xd), _p(b))
        return b

    def precond_solve(self, b):
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros(2 * self.n)
        self.lib.oref_precond_solve(self.h, _p(b), _p(x))
        return x

    def rhs(self):
        r = np.zeros(2 * self.n)
        self.lib.oref_rhs(self.h, _p(r))
        return r

    def solve(self, rhs, tol=1e-6):
        rhs = np.ascontiguousarray(rhs, dtype=np.float64)
        sol = np.zeros(2 * self.n)
        with stdout_to_stderr():
            it = self.lib.oref_gmres(self.h, _p(rhs), _p(sol), tol)
        return sol, it

    def reaction(self, sol):
        sol = np.ascontiguousarray(sol, dtype=np.float64)
        phi = np.zeros(self.nq)
        self.lib.oref_reaction(self.h, _p(sol), _p(phi))
        return phi

    def energy(self, phi):
        phi = np.ascontiguousarray(phi, dtype=np.float64)
        return float(self.lib.oref_energy(self.h, _p(phi)))

    def collect_potentials(self, collect, inputs, sol, addcoulombic=0):
        """The reference's own collectPotentials (FFTSVDpbeAPI.c:1896-1922) on this
        API-built operator; writes collect[a].potential.  innerdielectric is the
        eps_in the operator was built with (set by oref_create_api)."""
        sol = np.ascontiguousarray(sol, dtype=np.float64)
        C.c_uint.in_dll(self.lib, "addcoulombic").value = int(addcoulombic)
        try:
            self.lib.collectPotentials(collect, C.c_uint(len(collect)), inputs, C.c_uint(len(inputs)),
                                       C.c_void_p(self.surface_operator), _p(sol))
        finally:
            C.c_uint.in_dll(self.lib, "addcoulombic").value = 0

    def panel_integrals(self, kernel, kappa, pts, panel_of_point):
        pts = np.ascontiguousarray(pts, dtype=np.float64)
        idx = np.ascontiguousarray(panel_of_point, dtype=np.uint32)
        s = np.zeros(len(pts))
        d = np.zeros(len(pts))
        self.lib.oref_panel_integrals(self.h, int(kernel), float(kappa), len(pts), _p(pts),
                                      idx.ctypes.data_as(C.POINTER(C.c_uint)), _p(s), _p(d))
        return s, d

    def export_tree(self, which) -> dict:
        t = TreeFlat()
        self.lib.oref_export_tree(self.h, which, C.byref(t))
        try:
            return tree_flat_to_numpy(t)
        finally:
            self.lib.oref_export_free(C.byref(t))
