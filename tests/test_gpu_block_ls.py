"""Least-squares update of block GMRES on the device (fftsvd_b200/csrc/block_ls.cu) against numpy.

The block Hessenberg problem min ||E1 S0 - Hbar Y|| is updated one block column at a time by
block Householder reflections, the block form of the Givens update in GMRES.c:485-503.  After
each step the residual norm of every right-hand side must equal the least-squares residual of
the problem truncated to the blocks so far (numpy lstsq), and R^-1 g_top must be the
least-squares solution.  The problems are seeded: S0 upper triangular with 5 added to its
diagonal, Gaussian projection blocks, upper-triangular subdiagonal blocks with 2 added to
their diagonal (or zero: an invariant Krylov space, whose last reflector of each panel has
nothing below its pivot)."""
import ctypes as C

import numpy as np
import pytest

import fftsvd_b200 as F

pytestmark = pytest.mark.gpu


def _problem(K, M, seed, zero_sub=False):
    rng = np.random.default_rng(seed)
    S0 = np.triu(rng.standard_normal((K, K))) + 5.0 * np.eye(K)
    H = np.zeros(((M + 1) * K, M * K))
    for j in range(M):
        H[:(j + 1) * K, j * K:(j + 1) * K] = rng.standard_normal(((j + 1) * K, K))
        sub = np.triu(rng.standard_normal((K, K))) + 2.0 * np.eye(K)
        H[(j + 1) * K:(j + 2) * K, j * K:(j + 1) * K] = 0.0 if zero_sub else sub
    return S0, H


def _run(S0, H, K, M):
    import torch

    lib = F.load()

    def dev(a):
        return torch.tensor(np.asfortranarray(a).ravel(order="F"), dtype=torch.float64, device="cuda")

    dS, dH = dev(S0), dev(H)
    res = torch.zeros(M * K, dtype=torch.float64, device="cuda")
    R = torch.zeros((M * K) ** 2, dtype=torch.float64, device="cuda")
    gt = torch.zeros(M * K * K, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    rc = lib.fftsvd_b200_block_ls_device(K, M, C.c_void_p(dS.data_ptr()), C.c_void_p(dH.data_ptr()),
                                         C.c_void_p(res.data_ptr()), C.c_void_p(R.data_ptr()),
                                         C.c_void_p(gt.data_ptr()))
    assert rc == 0, lib.fftsvd_b200_last_error()
    return (res.cpu().numpy().reshape(M, K), R.cpu().numpy().reshape((M * K, M * K), order="F"),
            gt.cpu().numpy().reshape((M * K, K), order="F"))


@pytest.mark.parametrize("K,M,seed,zero_sub", [(8, 6, 3, False), (16, 4, 11, False), (24, 9, 5, False),
                                               (1, 5, 2, False), (40, 5, 7, False), (256, 3, 13, False),
                                               (16, 3, 17, True)])
def test_block_least_squares_matches_numpy(gpu, K, M, seed, zero_sub):
    S0, H = _problem(K, M, seed, zero_sub)
    res, R, gt = _run(S0, H, K, M)
    rows = (M + 1) * K
    rhs = np.zeros((rows, K))
    rhs[:K] = S0
    scale = np.abs(S0).max()
    for j in range(M):
        Hj = H[:(j + 2) * K, :(j + 1) * K]
        Y, *_ = np.linalg.lstsq(Hj, rhs[:(j + 2) * K], rcond=None)
        r = np.linalg.norm(rhs[:(j + 2) * K] - Hj @ Y, axis=0)
        assert np.allclose(res[j], r, rtol=1e-10, atol=1e-11 * scale), j
    assert np.allclose(np.tril(R, -1), 0.0)
    Y = np.linalg.solve(R, gt)
    Yref, *_ = np.linalg.lstsq(H, rhs, rcond=None)
    assert np.linalg.norm(Y - Yref) <= 1e-10 * np.linalg.norm(Yref)


def test_block_least_squares_rejects_oversized_block(gpu):
    lib = F.load()
    assert lib.fftsvd_b200_block_ls_device(257, 1, C.c_void_p(8), C.c_void_p(8), C.c_void_p(8), C.c_void_p(8),
                                           C.c_void_p(8)) != 0
