"""Many right-hand sides on one surface: the multi-vector matvec and the
lockstep batched GMRES against the single-vector path, column by column.

Each column of a batch goes through the same arithmetic as the same vector on
its own (the translation reads each table entry once for 8 right-hand sides
but multiplies and accumulates in the same order), so columns agree with the
single path to rounding of the reduction order only; the tolerances below are
far tighter than the solver tolerance."""
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


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
@pytest.mark.parametrize("k", [5, 16])
def test_matvec_batch_matches_single(blob3, prec, k):
    import torch
    s = blob3[0]
    X = np.random.default_rng(k).standard_normal((k, s.n))
    xd = _dev(X)
    yd = torch.empty_like(xd)
    s.matvec_batch_device(xd.data_ptr(), yd.data_ptr(), k, prec)
    torch.cuda.synchronize()  # the matvec is issued on the library's stream
    Y = yd.cpu().numpy()
    for c in range(k):
        assert rel(Y[c], s.matvec(X[c], prec)) < 1e-12, c


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_solve_batch_matches_single_solves(blob3, prec):
    s = blob3[0]
    rng = np.random.default_rng(3)
    base = s.rhs()
    k = 6
    R = np.stack([base * (1.0 + 0.3 * c) + 0.05 * rng.standard_normal(s.n) * np.abs(base).max()
                  for c in range(k)])
    sol, info = s.solve_batch(R, precision=prec, tol=1e-6)
    for c in range(k):
        one = s.solve(R[c], precision=prec, tol=1e-6)
        assert info[c].status == 0
        assert info[c].iterations == one.iterations, (c, info[c].iterations, one.iterations)
        assert rel(sol[c], one.solution) < 1e-9, c


def test_charge_groups_rhs_and_energies(blob3):
    import torch
    s, tri, qpos, q, c = blob3
    nq = len(q)
    gptr = np.array([0, nq // 3, nq // 3, nq], dtype=np.int32)  # includes an empty group
    g = len(gptr) - 1
    rd = torch.empty((g, s.n), dtype=torch.float64, device="cuda")
    s.rhs_groups_device(gptr, rd.data_ptr())
    R = rd.cpu().numpy()
    assert not np.any(R[1])
    assert rel(R.sum(axis=0), s.rhs()) < 1e-13  # the right-hand side is linear in the charges
    # one group holding every charge: the energy of the single solve
    sol = s.solve(s.rhs(), precision="fp64", tol=1e-8).solution
    e_all = s.energy(s.reaction_potentials(sol))
    e1 = s.group_energies_device(np.array([0, nq], dtype=np.int32), _dev(sol[None, :]).data_ptr())
    assert abs(e1[0] - e_all) < 1e-12 * abs(e_all)
    # per-group energies from per-group solutions
    sd = torch.empty_like(rd)
    info = s.solve_batch_device(rd.data_ptr(), sd.data_ptr(), g, "fp64", tol=1e-8, raise_on_error=False)
    assert info[1].status == 0 and info[1].iterations == 0
    e = s.group_energies_device(gptr, sd.data_ptr())
    for gi in (0, 2):
        sg = s.solve(R[gi], precision="fp64", tol=1e-8).solution
        phi = s.reaction_potentials(sg)
        lo, hi = gptr[gi], gptr[gi + 1]
        expect = 0.5 * np.sum(q[lo:hi] * phi[lo:hi]) * 332.112 / c["eps_in"]
        assert abs(e[gi] - expect) < 1e-9 * abs(expect), gi
    assert e[1] == 0.0


def test_solve_batch_fault_isolated_to_its_column(blob3):
    s = blob3[0]
    base = s.rhs()
    R = np.stack([base, base * 2.0, base * 3.0])
    R[1, 7] = np.nan
    sol, info = s.solve_batch(R, precision="fp64", tol=1e-6, raise_on_error=False)
    assert info[1].status == F._abi.FFTSVD_ERR_NONFINITE
    assert info[0].status == 0 and info[2].status == 0
    one = s.solve(base, precision="fp64", tol=1e-6)
    assert rel(sol[0], one.solution) < 1e-9
    assert rel(sol[2], 3.0 * one.solution) < 1e-6


def test_solve_many_matches_individual_solves(gpu):
    import torch
    from fftsvd_b200.surface import solve_many
    surfs, rhs, sols = [], [], []
    for name in ("born3", "blob3", "blob4"):
        tri, qpos, q, c = make_case(name)
        s = Surface.from_problem(tri, qpos, q, c["eps_in"], c["eps_out"], c["kappa"], svd_tol=1e-4)
        surfs.append(s)
        rhs.append(_dev(s.rhs()))
        sols.append(torch.empty_like(rhs[-1]))
    info = solve_many(surfs, [r.data_ptr() for r in rhs], [x.data_ptr() for x in sols], "mixed", tol=1e-6)
    torch.cuda.synchronize()
    for i, s in enumerate(surfs):
        one = s.solve(rhs[i].cpu().numpy(), precision="mixed", tol=1e-6)
        assert info[i].status == 0 and info[i].iterations == one.iterations
        assert rel(sols[i].cpu().numpy(), one.solution) < 1e-12, i
