"""Writes the golden fixtures of this directory from the compiled reference
(oracle/_ref, built by `make -C oracle REF=<reference tree>`): the reference's own
FP64 and as-shipped FP32 results on two small seeded systems, with the inputs
they were computed from.  The fixtures pin the oracle's numpy restatement, the
library's host setup and the GPU path without the compiled reference.

    python tests/golden/make_golden.py

Per case (<name>.npz): tri (n x 9 vertices), qpos, q, the parameters, and
  x        seeded vector (default_rng(5), 2n)
  y64/y32  SurfaceOperator_topmultiply(x), FP64 build / as-shipped FP32 build
  rhs      SurfaceOperator_makeRHS
  z        Preconditioner_solve(rhs)
  sol, it  GMRES_SurfaceOperator(rhs) at relative residual 1e-6, iterations
  phi, dG  reaction potentials of sol, 0.5 sum q phi * 332.112 / eps_in
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

import ref  # noqa: E402  (oracle)
from helpers import make_case  # noqa: E402

CASES = ["born3", "blob3"]
SVD_TOL = 1e-4
GMRES_TOL = 1e-6


def make(name: str) -> str:
    tri, qpos, q, c = make_case(name)
    n = len(tri)
    with ref.stdout_to_stderr():
        r64 = ref.RefSystem(tri, qpos, q, c["eps_in"], c["eps_out"], c["kappa"], svd_tol=SVD_TOL, fp64=True)
        r32 = ref.RefSystem(tri, qpos, q, c["eps_in"], c["eps_out"], c["kappa"], svd_tol=SVD_TOL, fp64=False)
    x = np.random.default_rng(5).standard_normal(2 * n)
    rhs = r64.rhs()
    sol, it = r64.solve(rhs, GMRES_TOL)
    phi = r64.reaction(sol)
    out = os.path.join(HERE, name + ".npz")
    np.savez_compressed(
        out, tri=np.asarray(tri, dtype=np.float64), qpos=np.asarray(qpos, dtype=np.float64),
        q=np.asarray(q, dtype=np.float64), eps_in=c["eps_in"], eps_out=c["eps_out"], kappa=c["kappa"],
        svd_tol=SVD_TOL, gmres_tol=GMRES_TOL, x=x, y64=r64.matvec(x), y32=r32.matvec(x), rhs=rhs,
        z=r64.precond_solve(rhs), sol=sol, it=it, phi=phi, dG=r64.energy(phi))
    r64.close()
    r32.close()
    return out


if __name__ == "__main__":
    for name in CASES:
        path = make(name)
        print(path, os.path.getsize(path))
