"""Host side of surface creation (fftsvd_b200/csrc/setup.cpp, operator.cu build_layout) does
not depend on the number of host threads.

The octree, the near-field and basis sample batches, the flat trees, the operator layout and
the translation tiles are built in parallel at offsets fixed before each parallel step, so
every array must come out bit-identical with one thread and with several.  The driver
(tests/layout_driver.cpp) runs the host setup with its integrals in batches on the host (the
same batches the device evaluator receives) and prints a hash of every array."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from helpers import make_case

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "fftsvd_b200")


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.fail("g++ is needed to build the layout test driver")
    if not os.path.exists(os.path.join(PKG, "libfftsvd_b200.so")):
        pytest.fail("the library is not built (python -m fftsvd_b200.build)")
    exe = str(tmp_path_factory.mktemp("layout") / "layout_driver")
    subprocess.run([cxx, "-O2", "-std=c++17", "-fopenmp", "-I", os.path.join(ROOT, "include"), "-I",
                    "/usr/local/cuda/include", os.path.join(ROOT, "tests", "layout_driver.cpp"), "-o", exe, "-L", PKG,
                    "-lfftsvd_b200", "-Wl,-rpath," + PKG], check=True)
    return exe


@pytest.mark.parametrize("case", ["blob3", "blob4"])
def test_layout_does_not_depend_on_thread_count(driver, tmp_path, case):
    tri, qpos, q, c = make_case(case)
    path = str(tmp_path / "problem.bin")
    with open(path, "wb") as f:
        np.array([len(tri), len(q)], dtype=np.int64).tofile(f)
        np.array([c["eps_in"], c["eps_out"], c["kappa"]], dtype=np.float64).tofile(f)
        np.ascontiguousarray(np.asarray(tri, dtype=np.float64).reshape(-1, 9)).tofile(f)
        np.ascontiguousarray(np.asarray(qpos, dtype=np.float64).reshape(-1, 3)).tofile(f)
        np.ascontiguousarray(np.asarray(q, dtype=np.float64)).tofile(f)
    outs = []
    for threads in (1, 4):
        env = dict(os.environ, OMP_NUM_THREADS=str(threads))
        r = subprocess.run([driver, path], env=env, capture_output=True, text=True, check=True, timeout=600)
        outs.append(r.stdout)
    assert outs[0].count("\n") > 50
    assert outs[0] == outs[1]
