"""End-to-end on the GPU: surfaces built by the library's own host setup, and
the drop-in entry points called on operators built by the reference API."""
import ctypes as C

import numpy as np
import pytest

import fftsvd_b200 as F
import ref
from fftsvd_b200.surface import Surface
from helpers import make_case, ref_system, rel

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=["born3", "blob3", "blob4"])
def own_and_ref(request, gpu):
    name = request.param
    rs, tri, c = ref_system(name, fp64=True)
    s = Surface.from_problem(tri, rs.qpos, rs.q, c["eps_in"], c["eps_out"], c["kappa"], svd_tol=1e-4)
    return name, rs, s, c


def test_own_setup_matvec_matches_reference64(own_and_ref):
    _, rs, s, _ = own_and_ref
    x = np.random.default_rng(8).standard_normal(s.n)
    assert rel(s.matvec(x, "fp64"), rs.matvec(x)) < 1e-10
    assert rel(s.matvec(x, "fp32"), rs.matvec(x)) < 2e-5


def test_own_setup_energy_matches_reference64(own_and_ref):
    """FP64 reference solve vs this library's solves on its own operator.

    Tolerance: both solves stop at a GMRES relative residual of 1e-6, so the
    energies agree to the solve tolerance; the FP64 and mixed solves of the
    library converge to the same FP64-operator solution."""
    name, rs, s, c = own_and_ref
    rhs = s.rhs()
    assert rel(rhs, rs.rhs()) < 1e-13
    sol_ref, _ = rs.solve(rhs, 1e-6)
    e_ref = rs.energy(rs.reaction(sol_ref))
    e = {}
    for prec in ("fp64", "mixed", "fp32"):
        r = s.solve(rhs, precision=prec, tol=1e-6)
        e[prec] = s.energy(s.reaction_potentials(r.solution))
        assert abs(e[prec] - e_ref) < 2e-6 * abs(e_ref), (prec, e[prec], e_ref)
    assert abs(e["mixed"] - e["fp64"]) < 1e-6 * abs(e["fp64"])
    if name == "born3":
        born = -332.112 / (2 * 10.0) * (1 - 1 / 80.0)
        assert abs(e["fp64"] - born) < 5e-3 * abs(born)


def test_solver_fault_paths(own_and_ref):
    _, _, s, _ = own_and_ref
    rhs = s.rhs()
    bad = rhs.copy()
    bad[3] = np.nan
    with pytest.raises(F.FFTSVDError) as ei:
        s.solve(bad, precision="fp64", tol=1e-6)
    assert ei.value.code == F._abi.FFTSVD_ERR_NONFINITE
    r = s.solve(rhs, precision="fp64", tol=1e-12, max_iterations=3, raise_on_error=False)
    assert r.status == F._abi.FFTSVD_ERR_NOT_CONVERGED and r.iterations == 3
    zero = s.solve(np.zeros(s.n), precision="mixed", tol=1e-6)
    assert not np.any(zero.solution)


def test_dropin_solve_and_rhs_on_reference_api_operator(gpu):
    """solveSurfaceOperator / generateRHS of this library on a SurfaceOperator and
    Preconditioner built by the reference's generateSurfaceOperator."""
    tri, qpos, q, c = make_case("blob3")
    rs = ref.RefSystem(tri, qpos, q, c["eps_in"], c["eps_out"], c["kappa"], via_api=True, gmres_tol=1e-6)
    lib = F.load()
    so, pre = C.c_void_p(rs.surface_operator), C.c_void_p(rs.preconditioner)
    n = len(tri)
    out = C.POINTER(C.c_double)()
    lib.generateRHS.argtypes = [C.POINTER(C.POINTER(C.c_double)), C.c_void_p, C.c_uint]
    lib.generateRHS(C.byref(out), so, n)
    assert out
    rhs = np.ctypeslib.as_array(out, shape=(2 * n,)).copy()
    C.CDLL(None).free(out)
    assert rel(rhs, rs.rhs()) < 1e-13
    lib.solveSurfaceOperator.argtypes = [C.POINTER(C.POINTER(C.c_double)), C.c_void_p, C.c_void_p,
                                         C.POINTER(C.c_double), C.c_uint]
    rhs_c = np.ascontiguousarray(rhs)
    sol = C.POINTER(C.c_double)()
    lib.solveSurfaceOperator(C.byref(sol), so, pre, rhs_c.ctypes.data_as(C.POINTER(C.c_double)), n)
    assert sol
    x = np.ctypeslib.as_array(sol, shape=(2 * n,)).copy()
    C.CDLL(None).free(sol)
    x_ref, _ = rs.solve(rhs, 1e-6)
    e, e_ref = rs.energy(rs.reaction(x)), rs.energy(rs.reaction(x_ref))
    assert abs(e - e_ref) < 2e-6 * abs(e_ref)
    assert rel(x, x_ref) < 1e-4
