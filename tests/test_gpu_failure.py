"""Failure detection without a GPU fault: a bounded device wait that nothing satisfies
(an mbarrier with no arrival, polled as the tensor-core kernels poll theirs) gives up,
the library reports FFTSVD_ERR_TIMEOUT, and the context stays usable: a matvec right
after it matches one taken before."""
import numpy as np
import pytest

import fftsvd_b200 as F
from fftsvd_b200 import _abi
from fftsvd_b200.surface import Surface
from helpers import make_case

pytestmark = pytest.mark.gpu


def test_bounded_wait_gives_up_and_context_survives(gpu):
    lib = F.load()
    tri, qpos, q, c = make_case("blob3")
    s = Surface.from_problem(tri, qpos, q, c["eps_in"], c["eps_out"], c["kappa"], svd_tol=1e-4)
    x = np.random.default_rng(4).standard_normal(s.n)
    before = s.matvec(x, "fp32")
    assert lib.fftsvd_b200_bounded_wait_selftest(2000) == _abi.FFTSVD_ERR_TIMEOUT
    assert b"gave up" in lib.fftsvd_b200_last_error()
    after = s.matvec(x, "fp32")
    assert np.array_equal(before, after)
    s.close()
