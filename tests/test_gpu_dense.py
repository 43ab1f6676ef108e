"""The block solve's dense FP64 kernels (FP64 tensor-core MMA GEMMs, the triangular
inverse and the blocked left triangular solve) against numpy on seeded matrices.

Each GEMM entry is held to 1e-13 of sum_k |a_ik| |b_kj| (the rounding bound of a
length-K FP64 dot product, with room for K up to about 1e5; measured values are near
1e-16), so the bar does not depend on cancellation.  The triangular solve is held to
1e-12 relative to the solution's norm on a well-conditioned upper triangle."""
import ctypes as C

import numpy as np
import pytest

import fftsvd_b200 as F

pytestmark = pytest.mark.gpu

BAR = 1e-13


def _dev(a):
    import torch

    return torch.tensor(np.asfortranarray(a).ravel(order="F"), dtype=torch.float64, device="cuda")


def _host(t, shape):
    return t.cpu().numpy().reshape(shape, order="F")


def _gemm(trans_a, A, B, Cin, alpha, beta):
    import torch

    lib = F.load()
    m = A.shape[1] if trans_a else A.shape[0]
    k = A.shape[0] if trans_a else A.shape[1]
    n = B.shape[1]
    dA, dB, dC = _dev(A), _dev(B), _dev(Cin)
    torch.cuda.synchronize()
    rc = lib.fftsvd_b200_dense_gemm_device(trans_a, m, n, k, alpha, C.c_void_p(dA.data_ptr()), A.shape[0],
                                           C.c_void_p(dB.data_ptr()), B.shape[0], beta, C.c_void_p(dC.data_ptr()),
                                           m)
    assert rc == 0, lib.fftsvd_b200_last_error()
    return _host(dC, (m, n))


@pytest.mark.parametrize("m,n,k", [(2, 1, 2), (130, 70, 36), (20000, 256, 512), (163840, 64, 256)])
def test_gemm_nn(gpu, m, n, k):
    rng = np.random.default_rng(m + n + k)
    A, B, Cin = rng.standard_normal((m, k)), rng.standard_normal((k, n)), rng.standard_normal((m, n))
    got = _gemm(0, A, B, Cin, -0.75, 0.5)
    ref = -0.75 * (A @ B) + 0.5 * Cin
    scale = 0.75 * (np.abs(A) @ np.abs(B)) + 0.5 * np.abs(Cin)
    assert np.max(np.abs(got - ref) / scale) < BAR


@pytest.mark.parametrize("m,n,k", [(8, 8, 10), (256, 256, 163840), (520, 256, 40000), (3584, 256, 20480)])
def test_gemm_tn(gpu, m, n, k):
    rng = np.random.default_rng(m * 7 + n + k)
    A, B, Cin = rng.standard_normal((k, m)), rng.standard_normal((k, n)), rng.standard_normal((m, n))
    got = _gemm(1, A, B, Cin, 1.0, 0.0)
    ref = A.T @ B
    scale = np.abs(A).T @ np.abs(B)
    assert np.max(np.abs(got - ref) / scale) < BAR
    got2 = _gemm(1, A, B, Cin, 2.0, -1.0)  # beta path: C is read back
    ref2 = 2.0 * ref - Cin
    assert np.max(np.abs(got2 - ref2) / (2.0 * scale + np.abs(Cin))) < BAR


def test_gemm_rejects_odd_inner_dimension(gpu):
    import torch

    lib = F.load()
    a = torch.zeros(9 * 4 + 16, dtype=torch.float64, device="cuda")
    assert lib.fftsvd_b200_dense_gemm_device(1, 4, 4, 9, 1.0, C.c_void_p(a.data_ptr()), 9, C.c_void_p(a.data_ptr()),
                                             9, 0.0, C.c_void_p(a.data_ptr() + 8 * 36), 4) != 0


@pytest.mark.parametrize("rows,n,bs", [(256, 64, 256), (768, 256, 256), (3584, 256, 256), (96, 8, 16)])
def test_block_triangular_solve(gpu, rows, n, bs):
    import torch

    lib = F.load()
    rng = np.random.default_rng(rows + n)
    R = np.triu(rng.standard_normal((rows, rows))) / np.sqrt(rows)
    R[np.diag_indices(rows)] = 1.0 + rng.random(rows)
    R_stored = R + np.tril(rng.standard_normal((rows, rows)), -1)  # below the diagonal is never read
    Y = rng.standard_normal((rows, n))
    dR, dY = _dev(R_stored), _dev(Y)
    out = torch.empty(rows * n, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    rc = lib.fftsvd_b200_dense_trsm_device(rows, n, bs, C.c_void_p(dR.data_ptr()), rows, C.c_void_p(dY.data_ptr()),
                                           C.c_void_p(out.data_ptr()))
    assert rc == 0, lib.fftsvd_b200_last_error()
    got = _host(out, (rows, n))
    ref = np.linalg.solve(R, Y)
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-12
