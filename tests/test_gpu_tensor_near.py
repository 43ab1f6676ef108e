"""The multi-vector FP32 matvec with its near field on the tensor cores
(fftsvd_b200_matvec_batch_tensor_device: kind::tf32 MMAs with three-product
splitting and one TMEM accumulator per K-chunk of 32, 128 right-hand sides per CTA)
against the CUDA-core multi-vector matvec and the FP64 matvec.  Three TF32 products
accumulated over short chunks give FP32-level results: measured on a 20 480-panel
blob, 3.5e-7 against the CUDA-core FP32 matvec and 3.3e-7 against FP64 (the FP32
operator's own error is 1.3e-7), where one accumulator over the whole K gave 1.7e-6.
Bars: 2e-6 per column (relative 2-norm) against both."""
import ctypes as C

import numpy as np
import pytest

import fftsvd_b200 as F
from fftsvd_b200.surface import Surface
from helpers import make_case

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=["blob3", "blob4"])
def surface(request, gpu):
    tri, qpos, q, c = make_case(request.param)
    s = Surface.from_problem(tri, qpos, q, c["eps_in"], c["eps_out"], c["kappa"], svd_tol=1e-4)
    yield s
    s.close()


@pytest.mark.parametrize("nrhs", [8, 136, 256])
def test_tensor_near_field_matches_cuda_core_matvec(surface, nrhs):
    import torch

    s = surface
    lib = F.load()
    rng = np.random.default_rng(nrhs)
    X = torch.tensor(rng.standard_normal((nrhs, s.n)), dtype=torch.float64, device="cuda")
    Yt = torch.empty_like(X)
    Yc = torch.empty_like(X)
    torch.cuda.synchronize()
    assert lib.fftsvd_b200_matvec_batch_tensor_device(s._h, nrhs, C.c_void_p(X.data_ptr()),
                                                       C.c_void_p(Yt.data_ptr())) == 0, lib.fftsvd_b200_last_error()
    s.matvec_batch_device(X.data_ptr(), Yc.data_ptr(), nrhs, "fp32")
    torch.cuda.synchronize()
    yt, yc, x = Yt.cpu().numpy(), Yc.cpu().numpy(), X.cpu().numpy()
    for c in range(nrhs):
        e = np.linalg.norm(yt[c] - yc[c]) / np.linalg.norm(yc[c])
        assert e < 2e-6, (c, e)
    for c in (0, nrhs // 2, nrhs - 1):
        y64 = s.matvec(x[c], "fp64")
        assert np.linalg.norm(yt[c] - y64) / np.linalg.norm(y64) < 2e-6
