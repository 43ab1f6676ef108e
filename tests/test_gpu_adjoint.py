"""Transposed operator and adjoint derivatives of the solvation energy.

The transposed operator is checked through the identity <A x, y> = <x, A^T y>; the
adjoint derivatives against central finite differences of the energy itself (FP64
solves to 1e-12, step 1e-4 A in position and 1e-4 e in charge), which is the
gradient of the same discrete energy the adjoint differentiates."""
import numpy as np
import pytest

from fftsvd_b200.surface import Surface
from helpers import make_case

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=["born3", "blob3"])
def case(request, gpu):
    tri, qpos, q, c = make_case(request.param)
    s = Surface.from_problem(tri, qpos, q, c["eps_in"], c["eps_out"], c["kappa"], svd_tol=1e-4)
    return request.param, s, qpos.copy(), q.copy(), c


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-12), ("fp32", 2e-6)])
def test_transpose_identity(case, prec, tol):
    _, s, _, _, _ = case
    rng = np.random.default_rng(21)
    for _ in range(2):
        x, y = rng.standard_normal(s.n), rng.standard_normal(s.n)
        ax, aty = s.matvec(x, prec), s.matvec_transpose(y, prec)
        lhs, rhs = float(ax @ y), float(x @ aty)
        assert abs(lhs - rhs) <= tol * np.linalg.norm(ax) * np.linalg.norm(y), (lhs, rhs)


def _energy(s, qpos, q):
    s.set_charges(qpos, q)
    e, _, _, _ = s.adjoint(precision="fp64", tol=1e-12)
    return e


def test_adjoint_matches_finite_differences(case):
    name, s, qpos, q, c = case
    s.set_charges(qpos, q)
    e, dq, dx, info = s.adjoint(precision="fp64", tol=1e-12)
    assert info[0].status == 0 and info[1].status == 0
    picks = [0] if len(q) == 1 else [0, 7, 23, 41]
    h = 1e-4
    scale = max(np.abs(dx).max(), 1e-12)
    for j in picks:
        for a in range(3):
            p, m = qpos.copy(), qpos.copy()
            p[j, a] += h
            m[j, a] -= h
            fd = (_energy(s, p, q) - _energy(s, m, q)) / (2 * h)
            assert abs(dx[j, a] - fd) <= 1e-4 * max(abs(fd), 1e-2 * scale), (name, j, a, dx[j, a], fd)
        qp, qm = q.copy(), q.copy()
        qp[j] += h
        qm[j] -= h
        fdq = (_energy(s, qpos, qp) - _energy(s, qpos, qm)) / (2 * h)
        assert abs(dq[j] - fdq) <= 1e-4 * abs(fdq), (name, j, dq[j], fdq)
    s.set_charges(qpos, q)
    if name == "born3":  # a central charge: no net force, and dG is quadratic in q
        assert np.abs(dx).max() < 1e-6 * abs(e)
        assert abs(dq[0] - 2 * e / q[0]) < 1e-8 * abs(dq[0])


def test_mixed_adjoint_close_to_fp64(case):
    _, s, qpos, q, _ = case
    s.set_charges(qpos, q)
    e64, dq64, dx64, _ = s.adjoint(precision="fp64", tol=1e-8)
    em, dqm, dxm, _ = s.adjoint(precision="mixed", tol=1e-8)
    assert abs(em - e64) < 1e-6 * abs(e64)
    assert np.abs(dqm - dq64).max() < 1e-5 * np.abs(dq64).max()
    # force scale: the largest force, or (where every force vanishes, Born) the energy over 10 A
    assert np.abs(dxm - dx64).max() < 1e-4 * max(np.abs(dx64).max(), 0.1 * abs(e64))


def test_autograd_function(case):
    import torch
    from fftsvd_b200.autograd import SolvationEnergy
    _, s, qpos, q, _ = case
    pos = torch.tensor(qpos, dtype=torch.float64, requires_grad=True)
    chg = torch.tensor(q, dtype=torch.float64, requires_grad=True)
    energy = SolvationEnergy.apply(s, pos, chg)
    (2.0 * energy).backward()
    s.set_charges(qpos, q)
    e, dq, dx, _ = s.adjoint(precision="fp64", tol=1e-8)
    assert abs(float(energy) - e) < 1e-9 * abs(e)
    assert np.allclose(pos.grad.numpy(), 2.0 * dx, rtol=1e-6, atol=1e-9 * np.abs(dx).max() + 1e-15)
    assert np.allclose(chg.grad.numpy(), 2.0 * dq, rtol=1e-6, atol=1e-12)


@pytest.fixture(scope="module")
def warp_pair(gpu, monkeypatch_module):
    """The blob3 surface twice: once with the default kernels and once with every small
    grid on the one-cube-per-warp kernels (the 4^3 transposed transforms on their
    register DFTs), which large surfaces select by cube count."""
    tri, qpos, q, c = make_case("blob3")
    make = lambda: Surface.from_problem(tri, qpos, q, c["eps_in"], c["eps_out"], c["kappa"], svd_tol=1e-4)
    s_block = make()
    monkeypatch_module.setenv("FFTSVD_B200_WARP_MIN_CUBES", "0")
    s_warp = make()
    monkeypatch_module.delenv("FFTSVD_B200_WARP_MIN_CUBES")
    return s_block, s_warp


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-12), ("fp32", 2e-6)])
def test_warp_transpose_kernels(warp_pair, prec, tol):
    from helpers import rel
    s_block, s_warp = warp_pair
    rng = np.random.default_rng(33)
    for _ in range(2):
        x, y = rng.standard_normal(s_warp.n), rng.standard_normal(s_warp.n)
        aty = s_warp.matvec_transpose(y, prec)
        assert rel(aty, s_block.matvec_transpose(y, prec)) < tol
        ax = s_warp.matvec(x, prec)
        assert abs(float(ax @ y) - float(x @ aty)) <= tol * np.linalg.norm(ax) * np.linalg.norm(y)
