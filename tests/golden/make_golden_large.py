"""Writes the benchmark-size golden fixtures from the compiled reference's FP64
build (oracle/_ref/libfftsvd_ref64.so, built by `make -C oracle REF=<reference tree>`).

The benchmark systems are far too large for the reference to run inside a test,
so its results are computed once here and committed:

    python tests/golden/make_golden_large.py blob6      # 81 920 panels, 2 500 charges
    python tests/golden/make_golden_large.py blob7      # 327 680 panels, 30 000 charges

Per case (<name>_ref64.npz):
  inputs_sha256  hash of the seeded inputs (tri, qpos, q as float64 bytes), so a
                 test can confirm that the generators still produce them
  dG, it         reaction energy (kcal/mol) of GMRES_SurfaceOperator at relative
                 residual 1e-6 and its iteration count
  dG_tight, it_tight   the same solve at relative residual 1e-10
  phi            reaction potential of every charge (tol 1e-6 solution)
  sol_stride, sol_sample, sol_norm   every sol_stride-th entry of the tol 1e-6
                 surface solution [phi; dphi/dn] and the norm of the whole vector
  setup_s, solve_s, threads   wall times of the reference on this machine
"""
from __future__ import annotations

import hashlib
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import ref  # noqa: E402  (oracle)
from fftsvd_b200 import meshes  # noqa: E402

# the benchmark systems: level, radius, charges and seeds as the benchmark builds them
LARGE = {
    "blob6": dict(level=6, radius=22.0, nq=2500, seed=1, eps_in=4.0, eps_out=80.0, kappa=0.125, stride=8),
    "blob7": dict(level=7, radius=60.0, nq=30000, seed=3, eps_in=4.0, eps_out=80.0, kappa=0.125, stride=32),
}
SVD_TOL = 1e-4
GMRES_TOL = 1e-6
TIGHT_TOL = 1e-10


def make_inputs(name: str):
    c = LARGE[name]
    tri = meshes.blob(c["level"], c["radius"], seed=c["seed"])
    qpos, q = meshes.blob_charges(tri, c["radius"], c["nq"], seed=c["seed"] + 1, surface_seed=c["seed"])
    return tri, qpos, q, c


def inputs_hash(tri, qpos, q) -> str:
    h = hashlib.sha256()
    for a in (tri, qpos, q):
        h.update(np.ascontiguousarray(a, dtype=np.float64).tobytes())
    return h.hexdigest()


def make(name: str) -> str:
    tri, qpos, q, c = make_inputs(name)
    threads = os.cpu_count() or 1
    ref.set_threads(threads)
    t0 = time.time()
    r64 = ref.RefSystem(tri, qpos, q, c["eps_in"], c["eps_out"], c["kappa"], svd_tol=SVD_TOL, fp64=True)
    setup_s = time.time() - t0
    rhs = r64.rhs()
    t0 = time.time()
    sol, it = r64.solve(rhs, GMRES_TOL)
    solve_s = time.time() - t0
    phi = r64.reaction(sol)
    dG = r64.energy(phi)
    sol_t, it_t = r64.solve(rhs, TIGHT_TOL)
    dG_t = r64.energy(r64.reaction(sol_t))
    r64.close()
    out = os.path.join(HERE, name + "_ref64.npz")
    np.savez_compressed(
        out, inputs_sha256=inputs_hash(tri, qpos, q), level=c["level"], radius=c["radius"], nq=c["nq"],
        seed=c["seed"], eps_in=c["eps_in"], eps_out=c["eps_out"], kappa=c["kappa"], svd_tol=SVD_TOL,
        gmres_tol=GMRES_TOL, tight_tol=TIGHT_TOL, dG=dG, it=it, dG_tight=dG_t, it_tight=it_t, phi=phi,
        sol_stride=c["stride"], sol_sample=sol[::c["stride"]].copy(), sol_norm=float(np.linalg.norm(sol)),
        setup_s=setup_s, solve_s=solve_s, threads=threads)
    return out


if __name__ == "__main__":
    for name in sys.argv[1:] or ["blob6"]:
        path = make(name)
        print(path, os.path.getsize(path), flush=True)
