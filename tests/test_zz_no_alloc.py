"""The allocation-free reaction-potential entry point.

Some callers cannot call cudaMalloc: their device memory belongs to another
allocator (a framework's caching allocator or a pool reserved up front), or
they cannot accept the device-wide synchronisation that cudaMalloc/cudaFree
imply.  fftsvd_b200_reaction_potentials_noalloc serves them with a fixed
4 MiB scratch array that lives in the library.  These tests call it through the
C-ABI twice in a row, on device buffers the test allocates itself, check both
results against the regular (allocating) entry point, and check with the
library's own counter that the two calls made no device allocation.  They live
in a file of their own that pytest collects last, and they build their own
surface, so they run the same alone in a fresh process or after every other
test.
"""
import ctypes as C

import numpy as np
import pytest

import fftsvd_b200 as F
from fftsvd_b200 import _abi
from fftsvd_b200.surface import Surface
from helpers import make_case

pytestmark = pytest.mark.gpu

# Up to 8192 charges both paths sum the same 64 panel-chunk partials in the same order:
# rounding only.  Above that the scratch array holds fewer chunks, so the panel sums are
# grouped differently: a few ulps of the largest terms.
TOL_SAME_ORDER = 1e-12
TOL_REGROUPED = 1e-11
SCRATCH_CHARGES = 524288  # doubles in the library's scratch array


@pytest.fixture(scope="module")
def blob3_surface(gpu):
    tri, qpos, q, c = make_case("blob3")
    s = Surface.from_problem(tri, qpos, q, c["eps_in"], c["eps_out"], c["kappa"], svd_tol=1e-4)
    yield s, c
    s.close()


def _noalloc_twice(s, tol, seed):
    import torch

    lib = F.load()
    rng = np.random.default_rng(seed)
    for _ in range(2):  # two calls in a row share the scratch array
        sol = rng.standard_normal(s.n)
        expected = s.reaction_potentials(sol)
        sol_d = torch.tensor(sol, dtype=torch.float64, device="cuda")
        phi_d = torch.full((s.num_charges,), np.nan, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()  # every write to sol is finished before the call
        allocs = lib.fftsvd_b200_device_alloc_count()
        rc = lib.fftsvd_b200_reaction_potentials_noalloc(s._h, C.c_void_p(sol_d.data_ptr()),
                                                          C.c_void_p(phi_d.data_ptr()))
        assert rc == 0, lib.fftsvd_b200_last_error()
        assert lib.fftsvd_b200_device_alloc_count() == allocs, "the call allocated device memory"
        got = phi_d.cpu().numpy()
        assert np.all(np.isfinite(got))
        err = np.linalg.norm(got - expected) / np.linalg.norm(expected)
        assert err < tol, err


def test_noalloc_reaction_potentials_match_allocating_path(blob3_surface):
    s, _ = blob3_surface
    _noalloc_twice(s, TOL_SAME_ORDER, seed=21)


def test_noalloc_many_charges_take_fewer_chunks(blob3_surface):
    """20 000 charges: 524288 / 20000 = 26 panel chunks instead of 64."""
    s, c = blob3_surface
    rng = np.random.default_rng(33)
    nq = 20000
    d = rng.standard_normal((nq, 3))
    pos = 0.6 * c["radius"] * d / np.linalg.norm(d, axis=1, keepdims=True) * rng.uniform(0, 1, (nq, 1)) ** (1 / 3)
    s.set_charges(pos, rng.uniform(-0.6, 0.6, nq))
    _noalloc_twice(s, TOL_REGROUPED, seed=22)


def test_noalloc_rejects_more_charges_than_scratch_before_any_launch(blob3_surface):
    import torch

    s, _ = blob3_surface
    lib = F.load()
    nq = SCRATCH_CHARGES + 1
    rng = np.random.default_rng(34)
    s.set_charges(rng.uniform(-5, 5, (nq, 3)), rng.uniform(-0.6, 0.6, nq))
    sol_d = torch.zeros(s.n, dtype=torch.float64, device="cuda")
    phi_d = torch.zeros(nq, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    launches, allocs = lib.fftsvd_b200_launch_count(), lib.fftsvd_b200_device_alloc_count()
    rc = lib.fftsvd_b200_reaction_potentials_noalloc(s._h, C.c_void_p(sol_d.data_ptr()), C.c_void_p(phi_d.data_ptr()))
    assert rc == _abi.FFTSVD_ERR_ARGUMENT
    assert b"scratch" in lib.fftsvd_b200_last_error()
    assert lib.fftsvd_b200_launch_count() == launches
    assert lib.fftsvd_b200_device_alloc_count() == allocs
