"""ORACLE — test infrastructure only: CPU baselines of the reference's own C1 solve.

Times the compiled reference (oracle/_ref) on the C1 blob (81 920 panels, 2 500 charges,
eps 4/80, kappa 0.125, FFTSVD tolerance 1e-4, GMRES 1e-6) for each build and thread count:

  O3       oracle/_ref/libfftsvd_ref.so          -O3 -march=x86-64-v3, OpenMP (-DOMP)
  shipped  oracle/_ref/libfftsvd_ref_shipped.so  -g as in make-gcc.inc: no optimisation, no OpenMP

Setup (generateSurfaceOperator's tree fill), one matvec (SurfaceOperator_topmultiply),
the solve (GMRES_SurfaceOperator) and the reaction-potential collection
(SurfaceOperator_calculateReactionPotentials) are timed separately, each configuration in
a fresh process. Build the shipped variant first with
`make -C oracle shipped`.

    python oracle/cpu_baselines.py [--runs O3:1,O3:8,shipped:1] [--timeout SECONDS] > table.json
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
BUILDS = {"O3": os.path.join(HERE, "_ref", "libfftsvd_ref.so"),
          "shipped": os.path.join(HERE, "_ref", "libfftsvd_ref_shipped.so")}

_CHILD = r"""
import json, sys, time
sys.path.insert(0, {root!r}); sys.path.insert(0, {here!r})
import ref
from fftsvd_b200 import meshes
ref.set_threads({threads})
tri = meshes.blob(6, 22.0, seed=1)
qpos, q = meshes.blob_charges(tri, 22.0, 2500, seed=2, surface_seed=1)
t0 = time.perf_counter()
rs = ref.RefSystem(tri, qpos, q, 4.0, 80.0, 0.125, svd_tol=1e-4)
t1 = time.perf_counter()
rhs = rs.rhs()
tm0 = time.perf_counter()
rs.matvec(rhs)
tm1 = time.perf_counter()
with ref.stdout_to_stderr():
    sol, it = rs.solve(rhs, 1e-6)
t2 = time.perf_counter()
phi = rs.reaction(sol)
t3 = time.perf_counter()
e = rs.energy(phi)
print(json.dumps(dict(setup_s=t1 - t0, matvec_s=tm1 - tm0, solve_s=t2 - tm1, iterations=it,
                      collect_s=t3 - t2, dG=e)))
"""


def run(build: str, threads: int, timeout: float) -> dict:
    env = dict(os.environ, FFTSVD_REF_LIB=BUILDS[build], OMP_NUM_THREADS=str(threads))
    code = _CHILD.format(root=ROOT, here=HERE, threads=threads)
    try:
        out = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=timeout)
    except subprocess.TimeoutExpired:
        return {"build": build, "threads": threads, "unfinished_after_s": timeout}
    if out.returncode != 0:
        return {"build": build, "threads": threads, "error": out.stderr.strip().splitlines()[-1:]}
    res = json.loads(out.stdout.strip().splitlines()[-1])
    res.update(build=build, threads=threads)
    return res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--runs", default="O3:8,O3:1,shipped:1")
    ap.add_argument("--timeout", type=float, default=3600.0)
    args = ap.parse_args()
    rows = []
    for item in args.runs.split(","):
        build, threads = item.split(":")
        rows.append(run(build, int(threads), args.timeout))
        print(json.dumps(rows[-1]), file=sys.stderr, flush=True)
    print(json.dumps({"cores": os.cpu_count(), "runs": rows}))


if __name__ == "__main__":
    main()
