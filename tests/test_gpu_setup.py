"""Setup with the panel integrals on the GPU (fftsvd_b200_device_setup, the path
fftsvd_b200_surface_create takes) against the all-host setup: the same octree,
lists and ranks, near-field blocks and bases equal to rounding (the device's FP64
sqrt, log, exp and atan2 against the host's), and the same FP64 matvec; and the
surface it builds against the reference's own operator."""
import numpy as np
import pytest

import port  # oracle
from fftsvd_b200.surface import host_operator, two_region_maps
from helpers import make_case, ref_system, rel

pytestmark = pytest.mark.gpu

_INDEX_ARRAYS = ["leaf_row_ptr", "leaf_rows", "leaf_col_ptr", "leaf_cols", "leaf_d_ptr", "cube_level", "cube_index",
                 "cube_panel_ptr", "cube_panels", "cube_point_ptr", "cube_points", "cube_row_rank", "cube_col_rank",
                 "cube_vt_ptr", "cube_pv_ptr", "cube_uti_ptr", "cube_u_ptr", "inter_ptr", "inter_cubes",
                 "t_level_ptr"]


@pytest.mark.parametrize("name", ["born3", "blob3", "blob4"])
def test_device_integrals_match_host_setup(gpu, name):
    tri, _, _, c = make_case(name)
    h, ph = host_operator(tri, c["eps_in"], c["eps_out"], c["kappa"], svd_tol=1e-4)
    d, pd = host_operator(tri, c["eps_in"], c["eps_out"], c["kappa"], svd_tol=1e-4, integrals="device")
    for t in range(2):
        for key in _INDEX_ARRAYS:  # same partition, lists and ranks
            assert np.array_equal(h[t][key], d[t][key]), (t, key)
        # near-field integrals: rounding of the device's transcendental functions only
        for key in ("d_single", "d_double"):
            assert rel(d[t][key], h[t][key]) < 1e-14, (t, key, rel(d[t][key], h[t][key]))
        for key in ("vt", "pv_single", "pv_double", "uti", "u"):
            assert rel(d[t][key], h[t][key]) < 1e-10, (t, key, rel(d[t][key], h[t][key]))
        assert np.array_equal(h[t]["t_ops"], d[t]["t_ops"])
    assert rel(pd["value"], ph["value"]) < 1e-14
    n = len(tri)
    maps = two_region_maps(n, c["eps_in"], c["eps_out"])
    x = np.random.default_rng(3).standard_normal(2 * n)
    yh = port.matvec(h, maps, x, 2 * n)
    yd = port.matvec(d, maps, x, 2 * n)
    assert rel(yd, yh) < 1e-12, rel(yd, yh)
    # and against the reference's own FP64 operator, as the host setup is held to
    rs, _, _ = ref_system(name, fp64=True)
    assert rel(yd, rs.matvec(x)) < 1e-10
    rs.close()
