"""The allocation-free reaction-potential entry point.

Some callers cannot call cudaMalloc: their device memory belongs to another
allocator (a framework's caching allocator or a pool reserved up front), or
they cannot accept the device-wide synchronisation that cudaMalloc/cudaFree
imply.  fftsvd_b200_reaction_potentials_noalloc serves them with a fixed
4 MiB scratch array that lives in the library.  This test calls it through the
C-ABI twice in a row, on device buffers the test allocates itself, and checks
both results against the regular (allocating) entry point.  It lives in a file
of its own that pytest collects last, and it builds its own surface, so it
runs the same alone in a fresh process or after every other test.
"""
import ctypes as C

import numpy as np
import pytest

import fftsvd_b200 as F
from fftsvd_b200.surface import Surface
from helpers import make_case

pytestmark = pytest.mark.gpu

# both paths sum the same panel-chunk partials in the same order; allow rounding only
TOL = 1e-12


def test_noalloc_reaction_potentials_match_allocating_path(gpu):
    import torch

    tri, qpos, q, c = make_case("blob3")
    s = Surface.from_problem(tri, qpos, q, c["eps_in"], c["eps_out"], c["kappa"], svd_tol=1e-4)
    lib = F.load()
    rng = np.random.default_rng(21)
    for _ in range(2):  # two calls in a row share the scratch array
        sol = rng.standard_normal(s.n)
        expected = s.reaction_potentials(sol)
        sol_d = torch.tensor(sol, dtype=torch.float64, device="cuda")
        phi_d = torch.full((s.num_charges,), np.nan, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        rc = lib.fftsvd_b200_reaction_potentials_noalloc(s._h, C.c_void_p(sol_d.data_ptr()),
                                                          C.c_void_p(phi_d.data_ptr()))
        assert rc == 0, lib.fftsvd_b200_last_error()
        got = phi_d.cpu().numpy()
        assert np.all(np.isfinite(got))
        err = np.linalg.norm(got - expected) / np.linalg.norm(expected)
        assert err < TOL, err
    s.close()
