"""Device kernels on the reference's own compressed operator (exported from the
reference C compiled in oracle/_ref/) against the reference's CPU results."""
import numpy as np
import pytest

import ref
from helpers import ref_system, rel, surface_from_reference

pytestmark = pytest.mark.gpu

# FP32 operator storage: device and reference both accumulate leaf and grid
# products in FP32 but in different orders; FP64: only rounding differences.
TOL_FP32 = 2e-5
TOL_FP64 = 1e-11


@pytest.fixture(scope="module", params=["born3", "blob3", "blob4"])
def case32(request, gpu):
    rs, tri, c = ref_system(request.param, fp64=False)
    return rs, surface_from_reference(rs, tri, c), c


@pytest.fixture(scope="module", params=["blob3", "blob4"])
def case64(request, gpu):
    if not ref.available(fp64=True):
        pytest.fail("oracle/_ref/libfftsvd_ref64.so missing")
    rs, tri, c = ref_system(request.param, fp64=True)
    return rs, surface_from_reference(rs, tri, c), c


def test_matvec_fp32_matches_reference(case32):
    rs, s, _ = case32
    rng = np.random.default_rng(3)
    for _ in range(3):
        x = rng.standard_normal(s.n)
        assert rel(s.matvec(x, "fp32"), rs.matvec(x)) < TOL_FP32


def test_matvec_fp64_matches_reference64(case64):
    rs, s, _ = case64
    x = np.random.default_rng(4).standard_normal(s.n)
    assert rel(s.matvec(x, "fp64"), rs.matvec(x)) < TOL_FP64


def test_preconditioner_matches_reference(case32):
    rs, s, _ = case32
    b = np.random.default_rng(5).standard_normal(s.n)
    assert rel(s.precond_solve(b), rs.precond_solve(b)) < 1e-6


def test_rhs_matches_reference(case32):
    rs, s, _ = case32
    assert rel(s.rhs(), rs.rhs()) < 1e-13


def test_solve_and_energy_match_reference(case32):
    rs, s, c = case32
    rhs = rs.rhs()
    sol_ref, it_ref = rs.solve(rhs, 1e-6)
    e_ref = rs.energy(rs.reaction(sol_ref))
    for prec in ("fp32", "fp64", "mixed"):
        r = s.solve(rhs, precision=prec, tol=1e-6)
        phi = s.reaction_potentials(r.solution)
        e = s.energy(phi)
        assert abs(e - e_ref) < 2e-5 * abs(e_ref), (prec, e, e_ref)
        if prec == "fp32":
            assert abs(r.iterations - it_ref) <= 1
            assert rel(r.solution, sol_ref) < 1e-4


def test_reaction_potentials_match_reference(case32):
    rs, s, _ = case32
    sol = np.random.default_rng(6).standard_normal(s.n)
    assert rel(s.reaction_potentials(sol), rs.reaction(sol)) < 1e-11


@pytest.fixture(scope="module", params=["blob3", "blob4"])
def case_warp(request, gpu, monkeypatch_module):
    """The reference operator with every small grid (n <= 5) on the one-cube-per-warp
    kernels (the 4^3 grid on its register DFT), which large surfaces select by cube
    count: the threshold is lowered to zero for this surface."""
    if not ref.available(fp64=True):
        pytest.fail("oracle/_ref/libfftsvd_ref64.so missing")
    monkeypatch_module.setenv("FFTSVD_B200_WARP_MIN_CUBES", "0")
    rs64, tri, c = ref_system(request.param, fp64=True)
    s64 = surface_from_reference(rs64, tri, c)
    rs32, _, _ = ref_system(request.param, fp64=False)
    s32 = surface_from_reference(rs32, tri, c)
    monkeypatch_module.delenv("FFTSVD_B200_WARP_MIN_CUBES")
    return rs64, s64, rs32, s32


def test_warp_kernels_match_reference(case_warp):
    rs64, s64, rs32, s32 = case_warp
    rng = np.random.default_rng(12)
    for _ in range(2):
        x = rng.standard_normal(s64.n)
        assert rel(s64.matvec(x, "fp64"), rs64.matvec(x)) < TOL_FP64
        assert rel(s32.matvec(x, "fp32"), rs32.matvec(x)) < TOL_FP32
