"""Host least-squares update of block GMRES (fftsvd_b200/csrc/block_ls.cpp) against numpy.

The block Hessenberg problem min ||E1 S0 - Hbar Y|| is updated one block column at a time by
block Householder reflections, the block form of the Givens update in GMRES.c:485-503.  After
each step the residual norm of every right-hand side must equal the least-squares residual of
the problem truncated to the blocks so far, and R^-1 g_top must be the least-squares solution."""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.fail("g++ is needed to build the least-squares test driver")
    exe = str(tmp_path_factory.mktemp("block_ls") / "block_ls_driver")
    subprocess.run([cxx, "-O2", "-std=c++17", "-fopenmp", os.path.join(ROOT, "tests", "block_ls_driver.cpp"),
                    os.path.join(ROOT, "fftsvd_b200", "csrc", "block_ls.cpp"), "-o", exe], check=True)
    return exe


@pytest.mark.parametrize("K,M,seed", [(8, 6, 3), (16, 4, 11), (24, 9, 5), (1, 5, 2)])
def test_block_least_squares_matches_numpy(driver, tmp_path, K, M, seed):
    out = str(tmp_path / "ls.bin")
    subprocess.run([driver, str(K), str(M), str(seed), out], check=True)
    rows, cols = (M + 1) * K, M * K
    d = np.fromfile(out)
    sizes = [M * K, rows * cols, K * K, cols * cols, cols * K]
    parts, o = [], 0
    for sz in sizes:
        parts.append(d[o:o + sz])
        o += sz
    assert o == d.size
    res = parts[0].reshape(M, K)
    H = parts[1].reshape(cols, rows).T
    S0 = parts[2].reshape(K, K).T
    R = parts[3].reshape(cols, cols).T
    gt = parts[4].reshape(K, cols).T
    rhs = np.zeros((rows, K))
    rhs[:K] = S0
    for j in range(M):
        Hj = H[:(j + 2) * K, :(j + 1) * K]
        Y, *_ = np.linalg.lstsq(Hj, rhs[:(j + 2) * K], rcond=None)
        r = np.linalg.norm(rhs[:(j + 2) * K] - Hj @ Y, axis=0)
        assert np.allclose(res[j], r, rtol=1e-10, atol=1e-12 * np.abs(S0).max()), j
    assert np.allclose(np.tril(R, -1), 0.0)
    Y = np.linalg.solve(R, gt)
    Yref, *_ = np.linalg.lstsq(H, rhs, rcond=None)
    assert np.linalg.norm(Y - Yref) <= 1e-10 * np.linalg.norm(Yref)
