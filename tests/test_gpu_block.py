"""Block GMRES (one Krylov space shared by many right-hand sides) against the
single solves.

The block solve searches each column's solution in a different (larger) Krylov
space than the single solve, so the columns are not bit-identical to it.  What
is exact is the stopping test: each column's preconditioned residual
||P^-1 (b - A x)|| / ||P^-1 b||, recomputed here with the FP64 matvec, is below
the tolerance.  Solutions of two solves that both meet it differ by at most the
tolerance times the preconditioned operator's condition number; the bounds below
(1e-4 in the solution, 1e-5 in the energy at tol 1e-6) allow for that."""
import numpy as np
import pytest

import fftsvd_b200 as F
from fftsvd_b200.surface import Surface
from helpers import make_case, rel

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def blob3(gpu):
    tri, qpos, q, c = make_case("blob3")
    s = Surface.from_problem(tri, qpos, q, c["eps_in"], c["eps_out"], c["kappa"], svd_tol=1e-4)
    return s, tri, qpos, q, c


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _presid(s, b, x, prec="fp64"):
    """||P^-1 (b - A x)|| / ||P^-1 b||: the quantity the solver's stopping test bounds."""
    return float(np.linalg.norm(s.precond_solve(b - s.matvec(x, prec))) / np.linalg.norm(s.precond_solve(b)))


def _groups(s, nq, g):
    import torch
    gptr = np.linspace(0, nq, g + 1).astype(np.int32)
    rd = torch.empty((g, s.n), dtype=torch.float64, device="cuda")
    s.rhs_groups_device(gptr, rd.data_ptr())
    return gptr, rd


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_solve_block_meets_the_tolerance_and_matches_single_solves(blob3, prec):
    s = blob3[0]
    rng = np.random.default_rng(3)
    base = s.rhs()
    k = 6
    R = np.stack([base * (1.0 + 0.3 * c) + 0.05 * rng.standard_normal(s.n) * np.abs(base).max()
                  for c in range(k)])
    sol, info = s.solve_block(R, precision=prec, tol=1e-6)
    for c in range(k):
        assert info[c].status == 0, c
        assert info[c].residual < 1e-6
        assert _presid(s, R[c], sol[c]) < 1e-6 * 1.001, c
        one = s.solve(R[c], precision=prec, tol=1e-6)
        assert rel(sol[c], one.solution) < 1e-4, c
    # the block Krylov space holds each column's own: no column takes more steps than
    # it alone (one spare for a refinement pass started by rounding at the threshold)
    assert max(i.iterations for i in info) <= 1 + max(s.solve(R[c], precision=prec, tol=1e-6).iterations
                                                       for c in range(k))


def test_charge_group_energies_match_single_solves(blob3):
    """The batched-energy workload: every charge group's solvation energy from the block
    solve (mixed precision) against its FP64 single solve."""
    s, tri, qpos, q, c = blob3
    g = 12
    gptr, rd = _groups(s, len(q), g)
    import torch
    sd = torch.empty_like(rd)
    info = s.solve_block_device(rd.data_ptr(), sd.data_ptr(), g, "mixed", tol=1e-6)
    e_block = s.group_energies_device(gptr, sd.data_ptr())
    R = rd.cpu().numpy()
    steps = []
    for gi in range(g):
        assert info[gi].status == 0
        one = s.solve(R[gi], precision="fp64", tol=1e-10)
        steps.append(s.solve(R[gi], precision="mixed", tol=1e-6).iterations)
        phi = s.reaction_potentials(one.solution)
        lo, hi = gptr[gi], gptr[gi + 1]
        expect = 0.5 * np.sum(q[lo:hi] * phi[lo:hi]) * 332.112 / c["eps_in"]
        assert abs(e_block[gi] - expect) < 1e-5 * abs(expect), (gi, e_block[gi], expect)
    assert max(i.iterations for i in info) <= 1 + max(steps)


def test_zero_and_nonfinite_columns(blob3):
    s = blob3[0]
    base = s.rhs()
    rng = np.random.default_rng(5)
    R = np.stack([base, np.zeros(s.n), base * 3.0, 2.0 * base + 0.1 * rng.standard_normal(s.n) * np.abs(base).max()])
    R[2, 11] = np.inf
    sol, info = s.solve_block(R, precision="mixed", tol=1e-6, raise_on_error=False)
    assert info[2].status == F._abi.FFTSVD_ERR_NONFINITE
    assert not np.any(sol[2])
    assert info[1].status == 0 and info[1].iterations == 0 and not np.any(sol[1])
    for c in (0, 3):
        assert info[c].status == 0
        assert _presid(s, R[c], sol[c]) < 1e-6 * 1.001, c


@pytest.mark.parametrize("k", [11, 24])
def test_widths_not_a_multiple_of_eight(blob3, k):
    s = blob3[0]
    R = np.random.default_rng(k).standard_normal((k, s.n))
    sol, info = s.solve_block(R, precision="fp64", tol=1e-6)
    for c in range(k):
        assert info[c].status == 0
        assert _presid(s, R[c], sol[c]) < 1e-6 * 1.001, c


def test_fp32_operator_mode(blob3):
    s = blob3[0]
    R = np.random.default_rng(2).standard_normal((8, s.n))
    sol, info = s.solve_block(R, precision="fp32", tol=1e-5)
    for c in range(8):
        assert info[c].status == 0
        assert _presid(s, R[c], sol[c], "fp32") < 1e-5 * 1.001, c


def test_dependent_columns_still_solve(blob3):
    """Repeated and proportional right-hand sides make the first block rank deficient;
    the solve either carries the dependent directions or hands the block to the lockstep
    batch, and every column meets the tolerance either way."""
    s = blob3[0]
    base = s.rhs()
    R = np.stack([base, base, -2.0 * base])
    sol, info = s.solve_block(R, precision="fp64", tol=1e-6)
    one = s.solve(base, precision="fp64", tol=1e-6).solution
    for c in range(3):
        assert info[c].status == 0
        assert _presid(s, R[c], sol[c]) < 1e-6 * 1.001, c
    assert rel(sol[0], one) < 1e-4 and rel(sol[2], -2.0 * one) < 1e-4


def test_iteration_cap_reports_not_converged(blob3):
    s = blob3[0]
    R = np.random.default_rng(9).standard_normal((8, s.n))
    sol, info = s.solve_block(R, precision="fp64", tol=1e-12, max_iterations=2, raise_on_error=False)
    for c in range(8):
        assert info[c].status == F._abi.FFTSVD_ERR_NOT_CONVERGED
        assert info[c].iterations <= 2
        # the residual reported is the true one of the returned iterate
        assert abs(_presid(s, R[c], sol[c]) - info[c].residual) < 1e-6 * info[c].residual


def test_krylov_space_exhausted_by_a_wide_block(blob3):
    """256 random columns on a surface of 2 560 unknowns fill the whole space in ten block
    steps, before a 1e-8 solve would converge from its rate: the tenth block is what remains
    after projecting against every direction, rounding noise, and its factor in the block
    Hessenberg matrix is at rounding level.  The least-squares update on the device then
    reports residuals at rounding level (a lucky breakdown) and the recomputed FP64
    residuals meet the tolerance, with no more block steps than the space has blocks."""
    s = blob3[0]
    R = np.random.default_rng(21).standard_normal((256, s.n))
    sol, info = s.solve_block(R, precision="fp64", tol=1e-8)
    for c in range(0, 256, 17):
        assert info[c].status == 0, c
        assert _presid(s, R[c], sol[c]) < 1e-8 * 1.001, c
    assert max(i.iterations for i in info) <= s.n // 256
