"""ORACLE — test infrastructure only (never imported by the product path).

CPU restatement (numpy, FP64) of the FFTSVD PBE hot path over the flat
operator layout declared in include/fftsvd_b200.h.  Each function cites the
reference code it restates.  It is checked against the reference itself
(oracle/_ref/, tests/test_oracle.py) and then used as the checker for the
device kernels where the compiled reference is not available.
"""
from __future__ import annotations

import numpy as np


def tree_multiplyboth(t: dict, xs: np.ndarray, xd: np.ndarray) -> np.ndarray:
    """b = S xs + D xd for one tree (Tree.c:597-683).

    near field   Cube_multiply_D                 Cube.c:1730-1798
    far field    Cube_multiplyboth_FFT_PV_VT     Cube.c:1986-2060
                 FFT_forwardGridTransform        FFT.c:66-108 (pad n^3 into (2n-1)^3 at n/2, r2c)
                 Cube_multiply_T                 Cube.c:2062-2111
                 Cube_multiply_U_UTI_IFFT        Cube.c:2156-2225
                 FFT_backwardGridTransform       FFT.c:112-150 (c2r, crop, 1/(2n-1)^3)
    """
    b = np.zeros(t["num_points"])
    rp, cp, dp = t["leaf_row_ptr"], t["leaf_col_ptr"], t["leaf_d_ptr"]
    for l in range(t["num_leaves"]):
        rows = t["leaf_rows"][rp[l]:rp[l + 1]]
        cols = t["leaf_cols"][cp[l]:cp[l + 1]]
        nr, nc = len(rows), len(cols)
        Ds = t["d_single"][dp[l]:dp[l + 1]].reshape(nr, nc)
        Dd = t["d_double"][dp[l]:dp[l + 1]].reshape(nr, nc)
        b[rows] += Ds @ xs[cols] + Dd @ xd[cols]

    nc = t["num_cubes"]
    spectra = {}
    for c in range(nc):
        lvl = int(t["cube_level"][c])
        n = int(t["grid"][lvl])
        Np, off = 2 * n - 1, n // 2
        panels = t["cube_panels"][t["cube_panel_ptr"][c]:t["cube_panel_ptr"][c + 1]]
        r = int(t["cube_row_rank"][c])
        if len(panels) == 0 or r == 0 or t["inter_ptr"][c + 1] == t["inter_ptr"][c]:
            continue
        VT = t["vt"][t["cube_vt_ptr"][c]:t["cube_vt_ptr"][c + 1]].reshape(r, len(panels))
        PVs = t["pv_single"][t["cube_pv_ptr"][c]:t["cube_pv_ptr"][c + 1]].reshape(n ** 3, r)
        PVd = t["pv_double"][t["cube_pv_ptr"][c]:t["cube_pv_ptr"][c + 1]].reshape(n ** 3, r)
        g = PVs @ (VT @ xs[panels]) + PVd @ (VT @ xd[panels])
        pad = np.zeros((Np, Np, Np))
        pad[off:off + n, off:off + n, off:off + n] = g.reshape(n, n, n)
        spectra[c] = np.fft.rfftn(pad)
    for d in range(nc):
        lvl = int(t["cube_level"][d])
        n = int(t["grid"][lvl])
        Np, off = 2 * n - 1, n // 2
        points = t["cube_points"][t["cube_point_ptr"][d]:t["cube_point_ptr"][d + 1]]
        r = int(t["cube_col_rank"][d])
        if len(points) == 0 or r == 0:
            continue
        pg = Np * Np * n
        S = np.zeros((Np, Np, n), dtype=np.complex128)
        any_src = False
        for s in t["inter_cubes"][t["inter_ptr"][d]:t["inter_ptr"][d + 1]]:
            if s not in spectra:
                continue
            dx, dy, dz = (t["cube_index"][3 * d:3 * d + 3] - t["cube_index"][3 * s:3 * s + 3])
            slot = ((dx + 3) * 7 + (dy + 3)) * 7 + (dz + 3)
            base = 2 * (int(t["t_level_ptr"][lvl]) + slot * pg)
            T = t["t_ops"][base:base + 2 * pg].view(np.complex128).reshape(Np, Np, n)
            S += T * spectra[s]
            any_src = True
        if not any_src:
            continue
        gp = np.fft.irfftn(S, s=(Np, Np, Np), axes=(0, 1, 2))[off:off + n, off:off + n, off:off + n].ravel()
        UTI = t["uti"][t["cube_uti_ptr"][d]:t["cube_uti_ptr"][d + 1]].reshape(r, n ** 3)
        U = t["u"][t["cube_u_ptr"][d]:t["cube_u_ptr"][d + 1]].reshape(len(points), r)
        b[points] += U @ (UTI @ gp)
    return b


def matvec(trees, maps, x: np.ndarray, n_unknowns: int) -> np.ndarray:
    """y = A x: join, per-tree multiply, jump, split/join (SurfaceOperator.c:51-158)."""
    y = np.zeros(n_unknowns)
    for t, m in zip(trees, maps):
        xs = m["dphi_scale"] * x[m["dphi_index"]]
        xd = m["phi_scale"] * x[m["phi_index"]]
        b = tree_multiplyboth(t, xs, xd)
        npts = t["num_points"]
        y[m["out_index"][:npts]] = b + m["jump"][:npts] * xd[:npts]
    return y


def precond_solve(pre: dict, r: np.ndarray) -> np.ndarray:
    """z = P^-1 r for the assembled sparse preconditioner (Preconditioner.c:201-294), dense."""
    n = pre["n"]
    P = np.zeros((n, n))
    for c in range(n):
        for k in range(pre["col_ptr"][c], pre["col_ptr"][c + 1]):
            P[pre["row_index"][k], c] += pre["value"][k]
    return np.linalg.solve(P, r)


def precond_operator(pre: dict):
    """precond_solve with the dense LU factored once, for repeated solves."""
    import scipy.linalg as sl

    n = pre["n"]
    P = np.zeros((n, n))
    for c in range(n):
        for k in range(pre["col_ptr"][c], pre["col_ptr"][c + 1]):
            P[pre["row_index"][k], c] += pre["value"][k]
    lu = sl.lu_factor(P)
    return lambda r: sl.lu_solve(lu, r)


def gmres(apply, psolve, rhs: np.ndarray, tol: float, maxit: int = 1000):
    """Left-preconditioned full GMRES with MGS and Givens rotations (GMRES.c:3-22, 446-539)."""
    r = psolve(rhs)
    normr = np.linalg.norm(r)
    n = len(rhs)
    if normr < tol:
        return np.zeros(n), 0
    V = [r / normr]
    H = np.zeros((maxit + 1, maxit + 1))
    c = np.zeros(maxit + 1)
    s = np.zeros(maxit + 1)
    g = np.zeros(maxit + 1)
    g[0] = normr

    def rot(cc, ss, a, b):
        return a * cc - b * ss, cc * b + ss * a

    i = 0
    for i in range(maxit):
        P = psolve(apply(V[i]))
        for j in range(i + 1):
            H[i, j] = P @ V[j]
            P = P - H[i, j] * V[j]
        H[i, i + 1] = np.linalg.norm(P)
        V.append(P / H[i, i + 1])
        for k in range(i):
            H[i, k], H[i, k + 1] = rot(c[k], s[k], H[i, k], H[i, k + 1])
        a, bb = H[i, i], H[i, i + 1]
        if bb == 0.0:
            c[i], s[i] = 1.0, 0.0
        else:
            ln = np.hypot(abs(a), abs(bb))
            c[i], s[i] = a / ln, -bb / ln
        H[i, i], H[i, i + 1] = rot(c[i], s[i], H[i, i], H[i, i + 1])
        g[i + 1] = 0.0
        g[i], g[i + 1] = rot(c[i], s[i], g[i], g[i + 1])
        if abs(g[i + 1]) / normr < tol:
            break
    k = i + 1
    y = g[:k].copy()
    for q in range(k - 1, -1, -1):
        y[q] /= H[q, q]
        y[:q] -= H[q, :q] * y[q]
    x = np.zeros(n)
    for j in range(k):
        x += y[j] * V[j]
    return x, k


def rhs(centroids: np.ndarray, qpos: np.ndarray, q: np.ndarray, n_unknowns: int) -> np.ndarray:
    """rhs[i] = sum_j q_j / |x_j - c_i| on the phi rows (SurfaceOperator.c:291-321)."""
    out = np.zeros(n_unknowns)
    d = np.linalg.norm(qpos[None, :, :] - centroids[:, None, :], axis=2)
    out[:len(centroids)] = (q[None, :] / d).sum(axis=1)
    return out
