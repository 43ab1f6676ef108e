"""ORACLE — test infrastructure only (never imported by the product path).

CPU restatement (numpy, FP64) of the FFTSVD PBE hot path over the flat
operator layout declared in include/fftsvd_b200.h: the matvec, preconditioner,
GMRES and right-hand side, and from the panel geometry the Laplace and Yukawa
panel integrals, the reaction potentials and the energy.  Each function cites the
reference code it restates.  It is checked against the compiled reference
(oracle/_ref/) and its golden fixtures (tests/golden/, tests/test_golden.py,
tests/test_setup.py) and serves as the checker where the compiled reference is
not available.
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


# ---- Laplace panel integrals and reaction potentials ---------------------------------------------
# The truncated constants of FlatIntegration.c:3-9 and the moment coefficients of FlatPanel.c:218-219,
# kept as the reference has them: the far-field moment expansion depends on these exact values.
_ONE3, _FIVE3, _ONE6, _SEVEN3 = 0.3333333333333, 1.666666666667, 0.16666666666667, 2.3333333333333
_LIMITFOURTH, _LIMITSECOND = 9.0, 36.0
_CS = (0.0, 1.0, 1.0, 1.5, 1.5, 3.75, 1.0, 3.0, 1.5, 7.5, 1.5, 1.5, 3.75, 1.5, 7.5, 3.75)


def _unit(v):
    return v / np.sqrt(v @ v)


def flat_panel(v1, v2, v3) -> dict:
    """The fields of a flat triangle the Laplace integral reads (FlatPanel.c:5-150): centroid, panel
    frame (axis 0 along v3-v1, axis 2 the normal (v3-v1)x(v2-v1)), vertices in that frame relative to
    the centroid, edge lengths and direction cosines, largest edge, area and moments."""
    v = [np.asarray(x, dtype=np.float64) for x in (v1, v2, v3)]
    centroid = ((v[0] + v[1]) + v[2]) * (1.0 / 3.0)
    edge = [np.sqrt((v[1] - v[0]) @ (v[1] - v[0])), np.sqrt((v[2] - v[1]) @ (v[2] - v[1])),
            np.sqrt((v[0] - v[2]) @ (v[0] - v[2]))]
    a0 = v[2] - v[0]
    a2 = np.cross(a0, v[1] - v[0])
    area = 0.5 * np.sqrt(a2 @ a2)
    a2 = _unit(a2)
    a0 = _unit(a0)
    a1 = np.cross(a2, a0)
    axis = np.array([a0, a1, a2])
    pv = np.array([axis @ (x - centroid) for x in v])
    cC = [(pv[(i + 1) % 3, 0] - pv[i, 0]) / edge[i] for i in range(3)]
    cS = [(pv[(i + 1) % 3, 1] - pv[i, 1]) / edge[i] for i in range(3)]
    # the second, edge-aligned frame the Yukawa edge integrals use, and the edge lines in it (FlatPanel.c:53-128)
    e = [(v[1] - v[0]) * (1.0 / np.sqrt((v[1] - v[0]) @ (v[1] - v[0]))),
         (v[2] - v[1]) * (1.0 / np.sqrt((v[2] - v[1]) @ (v[2] - v[1]))),
         (v[0] - v[2]) * (1.0 / np.sqrt((v[0] - v[2]) @ (v[0] - v[2])))]
    n0, n1 = e[0].copy(), e[1].copy()
    if abs(e[2] @ n0) < abs(n1 @ n0):
        n1 = -e[2]
    alpha = n1 @ n0
    n1 = n1 + e[0] * (-alpha)
    n1 = n1 * (1.0 / np.sqrt(n1 @ n1))
    axisnum = np.array([n0, n1, np.cross(n0, n1)])
    pvnum = np.array([axisnum @ (x - centroid) for x in v])
    lines, rhs, ov = [], [], []
    for i in range(3):
        d = pvnum[(i + 1) % 3] - pvnum[i]
        line = np.array([-d[1], d[0], d[2]])
        lines.append(line)
        rhs.append(pvnum[i] @ line)
        ov.append(pvnum[(i + 2) % 3] @ line - rhs[-1])
    return dict(centroid=centroid, axis=axis, pv=pv, edge=edge, cC=cC, cS=cS, max_diag=max(edge), area=area,
                moments=panel_moments(pv, area), axisnum=axisnum, pvnum=pvnum, edgeline=lines, edgeRHS=rhs,
                edgeOV=ov)


def panel_moments(pv, area) -> list:
    """FastCap's Euclidean moments up to order 4 by edge recurrences, scaled into the S vector
    (FlatPanel.c:214-318); S[1..15], S[0] unused."""
    order = 4
    IM = np.zeros((order + 1, order + 1))
    XP = [[pv[i, 0] ** j if j else 0.0 for j in range(order + 3)] for i in range(3)]
    YP = [[pv[i, 1] ** j if j else 0.0 for j in range(order + 3)] for i in range(3)]
    for i in range(3):  # repeated products, as the reference forms the powers
        for j in range(2, order + 3):
            XP[i][j] = XP[i][j - 1] * XP[i][1]
            YP[i][j] = YP[i][j - 1] * YP[i][1]
    IM[0, 0] = area
    for side in range(3):
        xp, yp = XP[side], YP[side]
        xpn, ypn = XP[(side + 1) % 3], YP[(side + 1) % 3]
        dx, dy = xpn[1] - xp[1], ypn[1] - yp[1]
        if abs(dx) >= abs(dy):
            dydx = dy / dx
            for M in range(2, order + 1):
                M1, M2 = M + 1, M + 2
                SI = (xpn[M1] * ypn[1] - xp[M1] * yp[1]) / M1 + dydx * (xp[M2] - xpn[M2]) / (M1 * M2)
                IM[M, 0] += SI
                for N in range(1, M + 1):
                    N1, MN1 = N + 1, M - N + 1
                    SI = (xpn[MN1] * ypn[N1] - xp[MN1] * yp[N1]) / (MN1 * N1) - (dydx * N * SI) / MN1
                    IM[M - N, N] += SI
        else:
            dxdy = dx / dy
            for M in range(2, order + 1):
                M1, M2 = M + 1, M + 2
                SI = (dxdy / (M1 * M2)) * (ypn[M2] - yp[M2])
                IM[0, M] += SI
                for N in range(1, M + 1):
                    MN1 = M - N + 1
                    MN2 = MN1 + 1
                    SI = dxdy * ((xpn[N] * ypn[MN2] - xp[N] * yp[MN2]) / (MN1 * MN2) - (N * SI / MN1))
                    IM[N, M - N] += SI
    S = [0.0] * 16
    i = 0
    for M in range(5):
        for N in range(5 - M):
            i += 1
            S[i] = IM[M, N] * _CS[i]
    return S


def laplace_panel(point, P) -> tuple:
    """Single- and double-layer integrals of 1/r over a flat panel at a point (FlatIntegration.c:295-429):
    the moment expansion when r^2 > 9 diag^2 (third and fourth moments below 36 diag^2), else the analytic
    edge formula; the double layer of the panel's own centroid is 2 pi."""
    point = np.asarray(point, dtype=np.float64)
    pmc = point - P["centroid"]
    xn, yn, zn = (float(P["axis"][k] @ pmc) for k in range(3))
    xsq, ysq, zsq = xn * xn, yn * yn, zn * zn
    rsq = xsq + ysq + zsq
    diagsq = P["max_diag"] * P["max_diag"]
    s = P["moments"]
    if rsq > _LIMITFOURTH * diagsq:
        r2Inv = 1.0 / rsq
        rInv = np.sqrt(r2Inv)
        r3Inv = r2Inv * rInv
        r5Inv = r3Inv * r2Inv
        zr2Inv = zn * r2Inv
        ss1 = s[1] * rInv
        ss3 = -(s[3] + s[10]) * r3Inv
        ss5 = (xsq * s[10] + (xn * yn * s[7]) + ysq * s[3]) * r5Inv
        fs = ss1 + _ONE3 * ss3 + ss5
        fd = zr2Inv * (ss1 + ss3 + 5.0 * ss5)
        if rsq < _LIMITSECOND * diagsq:
            s914, s813, s411 = s[9] + s[14], s[8] + s[13], s[4] + s[11]
            s512, s1215 = s[5] + s[12], s[12] + s[15]
            r7Inv = r5Inv * r2Inv
            r9Inv = r7Inv * r2Inv
            t5 = (-xn * s813 - yn * s411 + 0.1 * (s512 + s1215)) * r5Inv
            t7 = (_FIVE3 * ((xn * xsq * s[13] + yn * ysq * s[4]) + 3.0 * xn * yn * (xn * s[11] + yn * s[8]))
                  - xsq * s1215 - ysq * s512 - xn * yn * s914) * r7Inv
            t9 = (7.0 * (_ONE6 * (xsq * xsq * s[15] + ysq * ysq * s[5]) + xsq * ysq * s[12])
                  + _SEVEN3 * xn * yn * (xsq * s[14] + ysq * s[9])) * r9Inv
            fs += t5 + t7 + t9
            fd += zr2Inv * (5.0 * t5 + 7.0 * t7 + 9.0 * t9)
        return fs, fd
    znabs = abs(zn)
    pv = P["pv"]
    xm = [xn - pv[i, 0] for i in range(3)]
    ym = [yn - pv[i, 1] for i in range(3)]
    fe = [xm[i] * xm[i] + (zn - pv[i, 2]) ** 2 for i in range(3)]
    r = [np.sqrt(ym[i] * ym[i] + fe[i]) for i in range(3)]
    ok = all(r[i] >= 1.005 * znabs for i in range(3))
    fs = fd = 0.0
    for i in range(3):
        nx = (i + 1) % 3
        cC, cS = P["cC"][i], P["cS"][i]
        v = xm[i] * cS - ym[i] * cC
        arg = (r[i] + r[nx] - P["edge"][i]) / (r[i] + r[nx] + P["edge"][i])
        if arg > 0.0:
            fs -= v * np.log(arg)
        if ok:
            s1, c1 = v * r[i], znabs * (xm[i] * cC + ym[i] * cS)
            s2, c2 = v * r[nx], znabs * (xm[nx] * cC + ym[nx] * cS)
        else:
            s1, c1 = fe[i] * cS - xm[i] * ym[i] * cC, znabs * r[i] * cC
            s2, c2 = fe[nx] * cS - xm[nx] * ym[nx] * cC, znabs * r[nx] * cC
        fd += np.arctan2(s1 * c2 - s2 * c1, c1 * c2 + s1 * s2)
    if fd < 0.0:
        fd += 2.0 * np.pi
    if zn < 0.0:
        fd = -fd
    fs -= zn * fd
    if np.array_equal(P["centroid"], point):
        fd = 2.0 * np.pi
    return fs, fd


_DBL_EPS, _FLT_EPS = 2.220446049250313e-16, 1.1920928955078125e-07


def _gauss4():
    """The 4-point Gauss-Legendre rule on [0, 1] (QuadratureRule_allocate(4), QuadratureRule.c:3-125)."""
    t, w = np.polynomial.legendre.leggauss(4)
    return (t + 1.0) / 2.0, w / 2.0


def _yukawa_line(z, x, y1, y2, kappa):
    """Angular integral over one edge strip, single and double layer (FlatIntegration.c:473-635, Helmholtz):
    the angle range is split geometrically (factors of 10) and each piece takes the 4-point rule."""
    X, W = _gauss4()
    absZ = abs(z)
    x = abs(x)
    startY = y1
    if x < y1:
        endY = 10.0 * y1 if y2 > 10.0 * y1 else y2
    else:
        endY = y2 if x > y2 else x
    signZ = 1.0 if z > 0.0 else (-1.0 if z < 0.0 else 0.0)
    ls = ld = 0.0
    pieces = 0
    while startY < y2:
        pieces += 1
        if pieces > 1000:
            raise RuntimeError("line integral subdivision did not end")
        phi1, phi2 = np.arctan2(startY, x), np.arctan2(endY, x)
        dPhi = phi2 - phi1
        for i in range(4):
            theta = phi1 + (phi2 - phi1) * X[i]
            RT = np.sqrt((x * (1.0 / np.cos(theta))) ** 2 + z * z)
            ls -= W[i] * dPhi * (np.exp(-kappa * RT) - np.exp(-kappa * absZ)) / kappa
            ld -= W[i] * dPhi * (signZ * np.exp(-kappa * absZ) - (z / RT) * np.exp(-kappa * RT))
        startY = endY
        if endY == y2:
            endY = 10.0 * y2
        elif endY * 10.0 > y2:
            endY = y2
        else:
            endY = 10.0 * endY
    return ls, ld


def _rot(m, v):
    return np.array([m[0] * v[0] + m[1] * v[1] + m[2] * v[2], m[3] * v[0] + m[4] * v[1] + m[5] * v[2],
                     m[6] * v[0] + m[7] * v[1] + m[8] * v[2]])


def _yukawa_edge(v1, v2, p, kappa):
    """One edge (FlatIntegration.c:431-471, 637-799): rotate the plane through the edge and the point
    level, translate the point onto the z axis, turn the edge parallel to y, integrate both sides."""
    v1, v2, p = (np.array(a, dtype=np.float64) for a in (v1, v2, p))
    n = np.cross(v1, v2)
    if np.sqrt(n[0] ** 2 + n[1] ** 2) > 10 * _DBL_EPS:
        th = -np.arctan2(n[1], n[0])
        c, s = np.cos(th), np.sin(th)
        Z = (c, -s, 0.0, s, c, 0.0, 0.0, 0.0, 1.0)
        v1, v2, p = _rot(Z, v1), _rot(Z, v2), _rot(Z, p)
        Np = np.cross(v1, v2)
        th = np.pi / 2 - np.arctan2(Np[2], Np[0])
        c, s = np.cos(th), np.sin(th)
        Y = (c, 0.0, -s, 0.0, 1.0, 0.0, s, 0.0, c)
        v1, v2, p = _rot(Y, v1), _rot(Y, v2), _rot(Y, p)
    t = np.array([-p[0], -p[1], -v1[2]])
    v1, v2, p = v1 + t, v2 + t, p + t
    if abs(v1[2] - v2[2]) > 1e-6:
        raise RuntimeError("edge did not rotate onto the plane")
    dv = np.array([v1[0] - v2[0], v1[1] - v2[1], 0.0])
    dv = dv * (1.0 / np.sqrt(dv @ dv))
    c, s = dv[0], dv[1]
    v1x, v1y = s * v1[0] - c * v1[1], c * v1[0] + s * v1[1]
    v2y = c * v2[0] + s * v2[1]
    if abs(v1x) < 10 * _DBL_EPS:
        return 0.0, 0.0
    z, x1, y1, y2 = p[2], v1x, v2y, v1y
    if y2 < 0 and y1 < 0:
        y1, y2 = -y1, -y2
    if y2 < y1:
        y1, y2 = y2, y1
    s0, d0 = _yukawa_line(z, x1, y1 if y1 >= 0 else 0.0, y2, kappa)
    if y1 < 0.0:
        s1, d1 = _yukawa_line(z, x1, 0.0, -y1, kappa)
        s0, d0 = s0 + s1, d0 + d1
    return s0, d0


def yukawa_panel(point, P, kappa) -> tuple:
    """Single- and double-layer integrals of exp(-kappa r)/r over a flat panel (FlatIntegration.c:882-949,
    1035-1049): signed edge integrals in the panel's edge-aligned frame; the double layer in the panel's
    plane is 2 pi inside and 0 outside; kappa < 1e-6 takes the Laplace formula."""
    if kappa < 1e-6:
        return laplace_panel(point, P)
    pnt = P["axisnum"] @ (np.asarray(point, dtype=np.float64) - P["centroid"])
    fs = fd = 0.0
    left = 0
    for j in range(3):
        d = pnt @ P["edgeline"][j] - P["edgeRHS"][j]
        if (d > 0.0 and P["edgeOV"][j] > 0.0) or (d < 0.0 and P["edgeOV"][j] < 0.0):
            left += 1
            sign = 1.0
        else:
            sign = -1.0
        s, dd = _yukawa_edge(P["pvnum"][j], P["pvnum"][(j + 1) % 3], pnt, kappa)
        fs += sign * s
        fd += sign * dd
    if abs(pnt[2]) < 10 * _FLT_EPS:
        fd = 2.0 * np.pi if left == 3 else 0.0
    return fs, fd


def reaction(tri, phi, dphi, qpos) -> np.ndarray:
    """Reaction potentials at the charges of the region that owns the panels, direct branch
    (SurfaceOperator.c:364-396): phi_j = sum_i dphi_i SLP(x_j, i) - phi_i DLP(x_j, i), minus 4 pi phi_i
    where x_j is panel i's centroid.  tri: n x 9 vertices; phi, dphi: the region's slices of the solution."""
    tri = np.asarray(tri, dtype=np.float64).reshape(-1, 3, 3)
    panels = [flat_panel(*t) for t in tri]
    out = np.zeros(len(qpos))
    for j, x in enumerate(np.asarray(qpos, dtype=np.float64)):
        acc = 0.0
        for i, P in enumerate(panels):
            slp, dlp = laplace_panel(x, P)
            acc += dphi[i] * slp - phi[i] * dlp
            if np.array_equal(x, P["centroid"]):
                acc -= 4.0 * np.pi * phi[i]
        out[j] = acc
    return out


def energy(q, phi, eps_in) -> float:
    """0.5 sum q phi * 332.112 / eps_in in kcal/mol (FFTSVDsalt.c:167-170)."""
    return 0.5 * float(np.dot(q, phi)) * 332.112 / eps_in
