"""The library's own host setup against the reference's operator construction
(CPU only): octree, lists, near-field integrals, translation operators and
the compressed far field, compared through the full matvec (oracle port over
the flat layout, FP64) with the reference's FP64 build."""
import numpy as np
import pytest

import port
import ref
from fftsvd_b200.surface import host_operator, leaf_diagonals, two_region_maps, two_region_precond
from helpers import ref_system, rel

pytestmark = pytest.mark.skipif(not ref.available(fp64=True), reason="oracle/_ref not built")


def _canon(tree):
    """Leaf blocks keyed by their first row (order-independent comparison)."""
    out = {}
    rp, cp, dp = tree["leaf_row_ptr"], tree["leaf_col_ptr"], tree["leaf_d_ptr"]
    for l in range(tree["num_leaves"]):
        rows = tuple(tree["leaf_rows"][rp[l]:rp[l + 1]])
        out[rows] = (tuple(tree["leaf_cols"][cp[l]:cp[l + 1]]), tree["d_single"][dp[l]:dp[l + 1]],
                     tree["d_double"][dp[l]:dp[l + 1]])
    return out


@pytest.mark.parametrize("name", ["born3", "blob3"])
def test_host_setup_matches_reference_operator(name):
    rs, tri, c = ref_system(name, fp64=True)
    n = len(tri)
    mine, pre = host_operator(tri, c["eps_in"], c["eps_out"], c["kappa"], svd_tol=1e-4)
    theirs = [rs.export_tree(0), rs.export_tree(1)]
    for t in range(2):
        a, b = mine[t], theirs[t]
        assert a["depth"] == b["depth"] and list(a["grid"]) == list(b["grid"])
        assert a["num_leaves"] == b["num_leaves"] and a["num_cubes"] == b["num_cubes"]
        assert sorted(a["cube_row_rank"]) == sorted(b["cube_row_rank"])
        assert sorted(a["cube_col_rank"]) == sorted(b["cube_col_rank"])
        ca, cb = _canon(a), _canon(b)
        assert ca.keys() == cb.keys()
        for k in ca:
            assert ca[k][0] == cb[k][0]  # same near-field columns, same order
            assert rel(ca[k][1], cb[k][1]) < 1e-12 and rel(ca[k][2], cb[k][2]) < 1e-12
        assert rel(a["t_ops"], b["t_ops"]) < 1e-12
    maps = two_region_maps(n, c["eps_in"], c["eps_out"])
    x = np.random.default_rng(1).standard_normal(2 * n)
    assert rel(port.matvec(mine, maps, x, 2 * n), rs.matvec(x)) < 1e-10
    # preconditioner from the interior self terms
    ds, dd = leaf_diagonals(theirs[1])
    ref_pre = two_region_precond(ds, dd, c["eps_in"] / c["eps_out"])
    assert np.array_equal(pre["col_ptr"], ref_pre["col_ptr"])
    assert rel(pre["value"], ref_pre["value"]) < 1e-12


def test_host_setup_rejects_bad_input():
    from fftsvd_b200 import FFTSVDError
    tri = np.zeros((4, 9))
    with pytest.raises(FFTSVDError):
        host_operator(tri, 1.0, 80.0, 0.0)  # degenerate panels
    with pytest.raises(FFTSVDError):
        host_operator(np.full((4, 9), np.nan), 1.0, 80.0, 0.0)


_FLAT_ARRAYS = ["leaf_row_ptr", "leaf_rows", "leaf_col_ptr", "leaf_cols", "leaf_d_ptr", "d_single", "d_double",
                "cube_level", "cube_index", "cube_panel_ptr", "cube_panels", "cube_point_ptr", "cube_points",
                "cube_row_rank", "cube_col_rank", "cube_vt_ptr", "vt", "cube_pv_ptr", "pv_single", "pv_double",
                "cube_uti_ptr", "uti", "cube_u_ptr", "u", "inter_ptr", "inter_cubes", "t_level_ptr", "t_ops"]


@pytest.mark.parametrize("name", ["born3", "blob3"])
def test_batched_integrals_reproduce_host_setup_bit_for_bit(name):
    """The device setup's batch layout (near-field blocks, first-pass samples, sphere fits),
    evaluated on the host: the same operator as the per-cube host setup, bit for bit."""
    from helpers import make_case
    tri, _, _, c = make_case(name)
    a, pa = host_operator(tri, c["eps_in"], c["eps_out"], c["kappa"], svd_tol=1e-4)
    b, pb = host_operator(tri, c["eps_in"], c["eps_out"], c["kappa"], svd_tol=1e-4, integrals="batched")
    for t in range(2):
        for key in _FLAT_ARRAYS:
            assert np.array_equal(a[t][key], b[t][key]), (t, key)
    assert np.array_equal(pa["value"], pb["value"])
