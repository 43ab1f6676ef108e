"""Seeded synthetic surfaces and charge sets for the PBE workloads.

No molecular mesher runs here (the reference shells out to MSMS,
FFTSVDpbeAPI.c:1034-1049), so every workload is generated:

* ``icosphere(level, radius)`` — a level-L subdivided icosahedron,
  20 * 4**L flat triangles (level 5: 20 480, level 6: 81 920, level 7: 327 680).
* ``blob(level, radius, seed)`` — the icosphere displaced radially by a seeded
  sum of real spherical harmonics of degree 1..8, scaled so that the largest
  displacement is 15 % of the radius.
* ``blob_charges(...)`` — charges uniform inside the surface, at least
  ``margin`` from every panel centroid, values uniform in [-qmax, qmax] and
  shifted to zero net charge.

Triangles are returned as ``(N, 9)`` float64 arrays ``v1, v2, v3`` ordered so
that ``(v3 - v1) x (v2 - v1)`` points outward, which is the orientation the
reference reads from MSMS faces (VertFace.c:78-101 swaps the second and third
vertex, FlatPanel.c:41-49 forms the normal).
"""
from __future__ import annotations

import numpy as np

__all__ = ["icosphere", "blob", "blob_charges", "born_ion", "panel_centroids", "panel_normals"]


def _icosahedron():
    t = (1.0 + 5.0 ** 0.5) / 2.0
    v = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0],
                  [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
                  [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], dtype=np.float64)
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11],
                  [1, 5, 9], [5, 11, 4], [11, 10, 2], [10, 7, 6], [7, 1, 8],
                  [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9],
                  [4, 9, 5], [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], dtype=np.int64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    return v, f


def _subdivide(v, f):
    edge_mid = {}
    verts = [row for row in v]

    def mid(a, b):
        key = (a, b) if a < b else (b, a)
        idx = edge_mid.get(key)
        if idx is None:
            m = verts[a] + verts[b]
            m = m / np.linalg.norm(m)
            idx = len(verts)
            verts.append(m)
            edge_mid[key] = idx
        return idx

    out = np.empty((4 * len(f), 3), dtype=np.int64)
    for i, (a, b, c) in enumerate(f):
        ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
        out[4 * i + 0] = (a, ab, ca)
        out[4 * i + 1] = (b, bc, ab)
        out[4 * i + 2] = (c, ca, bc)
        out[4 * i + 3] = (ab, bc, ca)
    return np.array(verts), out


def _unit_icosphere(level: int):
    v, f = _icosahedron()
    for _ in range(level):
        v, f = _subdivide(v, f)
    return v, f


def _triangles(v, f):
    # f is counter-clockwise seen from outside: (b - a) x (c - a) points out.
    # Emit (a, c, b) so that (v3 - v1) x (v2 - v1) points out.
    a, b, c = v[f[:, 0]], v[f[:, 1]], v[f[:, 2]]
    return np.ascontiguousarray(np.concatenate([a, c, b], axis=1))


def icosphere(level: int, radius: float = 1.0, center=(0.0, 0.0, 0.0)) -> np.ndarray:
    v, f = _unit_icosphere(level)
    return _triangles(v * radius + np.asarray(center, dtype=np.float64), f)


def icosphere_mesh(level: int, radius: float = 1.0, center=(0.0, 0.0, 0.0)):
    """The icosphere as shared vertices (nv, 3) and faces (nf, 3) of vertex indices, in the
    corner order of icosphere()."""
    v, f = _unit_icosphere(level)
    f = np.asarray(f, dtype=np.int64)[:, [0, 2, 1]]  # the corner order _triangles emits
    return v * radius + np.asarray(center, dtype=np.float64), np.ascontiguousarray(f)


def _real_sph_harm_table(lmax: int, theta: np.ndarray, phi: np.ndarray):
    """Real spherical harmonics up to degree lmax (orthonormal), as a dict (l, m) -> values."""
    x = np.cos(theta)
    s = np.sqrt(np.maximum(0.0, 1.0 - x * x))
    # associated Legendre P_l^m(x) without Condon-Shortley phase, by the standard recurrences
    P = {(0, 0): np.ones_like(x)}
    for m in range(1, lmax + 1):
        P[(m, m)] = P[(m - 1, m - 1)] * (2 * m - 1) * s
    for m in range(0, lmax):
        P[(m + 1, m)] = (2 * m + 1) * x * P[(m, m)]
    for m in range(0, lmax + 1):
        for l in range(m + 2, lmax + 1):
            P[(l, m)] = ((2 * l - 1) * x * P[(l - 1, m)] - (l + m - 1) * P[(l - 2, m)]) / (l - m)
    Y = {}
    from math import factorial, pi, sqrt
    for l in range(lmax + 1):
        for m in range(0, l + 1):
            norm = sqrt((2 * l + 1) / (4 * pi) * factorial(l - m) / factorial(l + m))
            if m == 0:
                Y[(l, 0)] = norm * P[(l, 0)]
            else:
                Y[(l, m)] = sqrt(2.0) * norm * P[(l, m)] * np.cos(m * phi)
                Y[(l, -m)] = sqrt(2.0) * norm * P[(l, m)] * np.sin(m * phi)
    return Y


def _blob_radius_function(seed: int, lmax: int = 8, amplitude: float = 0.15):
    rng = np.random.default_rng(seed)
    coeffs = {}
    for l in range(1, lmax + 1):
        for m in range(-l, l + 1):
            coeffs[(l, m)] = rng.standard_normal() / (1.0 + l)

    def raw(dirs):
        theta = np.arccos(np.clip(dirs[:, 2], -1.0, 1.0))
        phi = np.arctan2(dirs[:, 1], dirs[:, 0])
        Y = _real_sph_harm_table(lmax, theta, phi)
        out = np.zeros(len(dirs))
        for key, c in coeffs.items():
            out += c * Y[key]
        return out

    # scale on a dense reference set of directions so the scale does not depend on the mesh level
    vref, _ = _unit_icosphere(5)
    peak = np.max(np.abs(raw(vref)))
    scale = amplitude / peak

    def radius_factor(dirs):
        return 1.0 + scale * raw(dirs)

    return radius_factor


def blob(level: int, radius: float, seed: int, amplitude: float = 0.15, lmax: int = 8) -> np.ndarray:
    v, f = _unit_icosphere(level)
    rf = _blob_radius_function(seed, lmax, amplitude)
    v = v * (radius * rf(v))[:, None]
    return _triangles(v, f)


def panel_centroids(tri: np.ndarray) -> np.ndarray:
    return (tri[:, 0:3] + tri[:, 3:6] + tri[:, 6:9]) / 3.0


def panel_normals(tri: np.ndarray) -> np.ndarray:
    n = np.cross(tri[:, 6:9] - tri[:, 0:3], tri[:, 3:6] - tri[:, 0:3])
    return n / np.linalg.norm(n, axis=1, keepdims=True)


def blob_charges(tri: np.ndarray, radius: float, count: int, seed: int, margin: float = 1.5,
                 qmax: float = 0.6, surface_seed: int | None = None, amplitude: float = 0.15,
                 lmax: int = 8):
    """Charges uniformly inside a blob (or sphere when surface_seed is None)."""
    from scipy.spatial import cKDTree

    rng = np.random.default_rng(seed)
    cent = panel_centroids(tri)
    kd = cKDTree(cent)
    rf = _blob_radius_function(surface_seed, lmax, amplitude) if surface_seed is not None else None
    rmax = radius * (1.0 + amplitude)
    pts = []
    need = count
    while need > 0:
        cand = rng.uniform(-rmax, rmax, size=(max(4 * need, 64), 3))
        r = np.linalg.norm(cand, axis=1)
        dirs = cand / np.maximum(r, 1e-300)[:, None]
        rs = radius * (rf(dirs) if rf is not None else np.ones(len(cand)))
        ok = r < rs
        cand = cand[ok]
        if len(cand):
            d, _ = kd.query(cand)
            cand = cand[d >= margin]
        take = cand[:need]
        pts.append(take)
        need -= len(take)
    pos = np.concatenate(pts, axis=0)[:count]
    q = rng.uniform(-qmax, qmax, size=count)
    q -= q.mean()
    return np.ascontiguousarray(pos), q


def born_ion(level: int = 5, radius: float = 10.0, charge: float = 1.0):
    tri = icosphere(level, radius)
    return tri, np.zeros((1, 3)), np.array([charge], dtype=np.float64)
