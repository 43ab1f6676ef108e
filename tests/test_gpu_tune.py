"""Translation tile shapes: explicit limits and the autotuner.

Tile limits decide how the member groups of one tree and level are packed into
thread blocks; the groups themselves and the order of every sum are fixed before
tiling.  Every matvec (FP32, FP64, transposed, many right-hand sides) must therefore
give the same bits under any limits, and the autotuner, which only picks among such
limits, must leave results unchanged."""
import numpy as np
import pytest

from fftsvd_b200.surface import Surface
from helpers import make_case, rel

pytestmark = pytest.mark.gpu

LIMITS = [(32, 320, 3072), (16, 192, 1536), (8, 128, 768), (1, 16, 4)]


@pytest.fixture(scope="module")
def blob3(gpu):
    tri, qpos, q, c = make_case("blob3")
    return Surface.from_problem(tri, qpos, q, c["eps_in"], c["eps_out"], c["kappa"], svd_tol=1e-4)


def _results(s, x, X):
    import torch
    out = {p: s.matvec(x, p) for p in ("fp32", "fp64")}
    out["transpose"] = s.matvec_transpose(x, "fp64")
    xd = torch.from_numpy(np.ascontiguousarray(X)).cuda()
    yd = torch.empty_like(xd)
    s.matvec_batch_device(xd.data_ptr(), yd.data_ptr(), X.shape[0], "fp32")
    torch.cuda.synchronize()  # the batched matvec is issued on the library's stream
    out["batch"] = yd.cpu().numpy()
    return out


def test_tile_limits_leave_results_unchanged(blob3):
    s = blob3
    rng = np.random.default_rng(5)
    x = rng.standard_normal(s.n)
    X = rng.standard_normal((8, s.n))
    s.set_tile_limits(*LIMITS[0])
    ref = _results(s, x, X)
    for lim in LIMITS[1:]:
        s.set_tile_limits(*lim)
        got = _results(s, x, X)
        for k in ("fp32", "fp64", "batch"):
            assert np.array_equal(got[k], ref[k]), (lim, k)
        # the transposed near field sums columns with atomics: equal to rounding only
        assert rel(got["transpose"], ref["transpose"]) < 1e-13, lim
    s.set_tile_limits(*LIMITS[0])


def test_tile_limits_rejected_out_of_range(blob3):
    import fftsvd_b200 as F
    for lim in [(0, 320, 3072), (33, 320, 3072), (32, 321, 3072), (32, 320, 3073)]:
        with pytest.raises(F.FFTSVDError):
            blob3.set_tile_limits(*lim)


def test_autotune_keeps_results(blob3):
    s = blob3
    s.set_tile_limits(*LIMITS[0])
    x = np.random.default_rng(9).standard_normal(s.n)
    before = {p: s.matvec(x, p) for p in ("fp32", "fp64")}
    sol_before = s.solve(s.rhs(), precision="mixed", tol=1e-6)
    info = s.autotune()
    k = len(info["candidates"])
    assert k >= 2 and info["candidates"][0] == LIMITS[0]
    assert 0 <= info["chosen_fp32"] < k and 0 <= info["chosen_fp64"] < k
    assert all(t > 0 for t in info["matvec_ms_fp32"] + info["matvec_ms_fp64"])
    for p in ("fp32", "fp64"):
        assert np.array_equal(s.matvec(x, p), before[p]), p
    sol = s.solve(s.rhs(), precision="mixed", tol=1e-6)
    assert sol.iterations == sol_before.iterations
    assert np.array_equal(sol.solution, sol_before.solution)
