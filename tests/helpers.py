"""Shared test helpers: reference systems from the oracle and the matching
device surfaces built from the reference's own exported operator."""
from __future__ import annotations

import os

import numpy as np

from fftsvd_b200 import meshes
from fftsvd_b200.surface import Surface, leaf_diagonals, two_region_maps, two_region_precond

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")

# small cases the CPU reference finishes in seconds
CASES = {
    "born3": dict(kind="born", level=3, radius=10.0, eps_in=1.0, eps_out=80.0, kappa=0.0),
    "blob3": dict(kind="blob", level=3, radius=12.0, eps_in=4.0, eps_out=80.0, kappa=0.125, nq=60, seed=7),
    "blob4": dict(kind="blob", level=4, radius=16.0, eps_in=4.0, eps_out=80.0, kappa=0.125, nq=200, seed=11),
}


def make_case(name: str):
    c = CASES[name]
    if c["kind"] == "born":
        tri, qpos, q = meshes.born_ion(c["level"], c["radius"])
    else:
        tri = meshes.blob(c["level"], c["radius"], seed=c["seed"])
        qpos, q = meshes.blob_charges(tri, c["radius"], c["nq"], seed=c["seed"] + 1, surface_seed=c["seed"])
    return tri, qpos, q, c


def ref_system(name: str, fp64: bool = False, svd_tol: float = 1e-4):
    import ref  # oracle

    tri, qpos, q, c = make_case(name)
    return ref.RefSystem(tri, qpos, q, c["eps_in"], c["eps_out"], c["kappa"], svd_tol=svd_tol, fp64=fp64), tri, c


def surface_from_reference(rs, tri, c) -> Surface:
    """Device surface built from the reference's own compressed operator."""
    n = len(tri)
    trees = [rs.export_tree(0), rs.export_tree(1)]
    maps = two_region_maps(n, c["eps_in"], c["eps_out"])
    ds, dd = leaf_diagonals(trees[1])
    pre = two_region_precond(ds, dd, c["eps_in"] / c["eps_out"])
    return Surface.from_flat(trees, maps, pre, rs.qpos, rs.q, eps_in=c["eps_in"], vertices=tri)


def rel(a, b) -> float:
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
