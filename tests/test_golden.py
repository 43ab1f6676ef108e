"""Golden fixtures (tests/golden/*.npz, written by tests/golden/make_golden.py from
the compiled reference) against: the input generators that made them, the
compiled reference itself, and the oracle's numpy restatement run on this
library's own host setup.  CPU only.

Tolerances: the compiled reference is deterministic, so it reproduces its own
fixtures to rounding (1e-13).  The restatement over the library's host setup is
an FP64 operator built independently of the reference's, equal to it to
~1e-13 (matvec 1e-10 allowed, as in the setup test); right-hand side and
preconditioner are the same arithmetic (1e-13, 1e-12); GMRES at 1e-6 takes the
same iterations and lands on the same solution to 1e-8."""
import os

import numpy as np
import pytest

import port
import ref
from fftsvd_b200.surface import host_operator, two_region_maps
from helpers import GOLDEN, make_case, rel

CASES = ["born3", "blob3"]


def load(name):
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    return {k: g[k] for k in g.files}


@pytest.mark.parametrize("name", CASES)
def test_generators_reproduce_golden_inputs(name):
    g = load(name)
    tri, qpos, q, c = make_case(name)
    assert np.array_equal(np.asarray(tri, dtype=np.float64), g["tri"])
    assert np.array_equal(qpos, g["qpos"]) and np.array_equal(q, g["q"])
    assert (c["eps_in"], c["eps_out"], c["kappa"]) == (g["eps_in"], g["eps_out"], g["kappa"])


@pytest.mark.skipif(not (ref.available(fp64=True) and ref.available()), reason="oracle/_ref not built")
@pytest.mark.parametrize("name", CASES)
def test_compiled_reference_reproduces_golden(name):
    g = load(name)
    args = (g["tri"], g["qpos"], g["q"], float(g["eps_in"]), float(g["eps_out"]), float(g["kappa"]))
    with ref.stdout_to_stderr():
        r64 = ref.RefSystem(*args, svd_tol=float(g["svd_tol"]), fp64=True)
        r32 = ref.RefSystem(*args, svd_tol=float(g["svd_tol"]))
    assert rel(r64.matvec(g["x"]), g["y64"]) < 1e-13
    assert rel(r32.matvec(g["x"]), g["y32"]) < 1e-13
    assert rel(r64.rhs(), g["rhs"]) < 1e-15
    assert rel(r64.precond_solve(g["rhs"]), g["z"]) < 1e-13
    sol, it = r64.solve(g["rhs"], float(g["gmres_tol"]))
    assert it == int(g["it"]) and rel(sol, g["sol"]) < 1e-12
    phi = r64.reaction(g["sol"])
    assert rel(phi, g["phi"]) < 1e-13 and abs(r64.energy(phi) - float(g["dG"])) < 1e-12 * abs(float(g["dG"]))


@pytest.mark.parametrize("name", CASES)
def test_restatement_on_own_setup_matches_golden(name):
    g = load(name)
    tri = g["tri"]
    n = len(tri)
    eps_in, eps_out = float(g["eps_in"]), float(g["eps_out"])
    trees, pre = host_operator(tri, eps_in, eps_out, float(g["kappa"]), svd_tol=float(g["svd_tol"]))
    maps = two_region_maps(n, eps_in, eps_out)
    y = port.matvec(trees, maps, g["x"], 2 * n)
    assert rel(y, g["y64"]) < 1e-10
    assert rel(g["y32"], g["y64"]) < 2e-5  # the as-shipped FP32 operator storage
    cent = tri.reshape(n, 3, 3).mean(axis=1)
    assert rel(port.rhs(cent, g["qpos"], g["q"], 2 * n), g["rhs"]) < 1e-13
    assert rel(port.precond_solve(pre, g["rhs"]), g["z"]) < 1e-12
    psolve = port.precond_operator(pre)
    sol, it = port.gmres(lambda v: port.matvec(trees, maps, v, 2 * n), psolve, g["rhs"], float(g["gmres_tol"]))
    assert abs(it - int(g["it"])) <= 1 and rel(sol, g["sol"]) < 1e-8


@pytest.mark.parametrize("name", CASES)
def test_restated_reaction_potentials_match_golden(name):
    """The numpy restatement of the Laplace panel integrals and the direct
    reaction-potential sum (SurfaceOperator.c:364-396) reproduces the compiled
    reference's potentials and energy to rounding."""
    g = load(name)
    n = len(g["tri"])
    phi = port.reaction(g["tri"], g["sol"][:n], g["sol"][n:], g["qpos"])
    assert rel(phi, g["phi"]) < 1e-13
    assert abs(port.energy(g["q"], phi, float(g["eps_in"])) - float(g["dG"])) < 1e-13 * abs(float(g["dG"]))


@pytest.mark.skipif(not ref.available(fp64=True), reason="oracle/_ref not built")
def test_restated_panel_integrals_match_compiled_reference():
    """Point by point against the reference's Integration (FlatIntegration.c:295-429) on every branch:
    the panel's own centroid, points just off the plane above the centroid and above a vertex (the
    r < 1.005|z| switch), in-plane points outside the panel, the analytic near zone, and both
    moment-expansion zones.  Points on the panel's edges and vertices are left out: there the double
    layer jumps and both codes return either side of the jump depending on the rounding of z."""
    g = load("blob3")
    with ref.stdout_to_stderr():
        rs = ref.RefSystem(g["tri"], g["qpos"], g["q"], float(g["eps_in"]), float(g["eps_out"]),
                           float(g["kappa"]), svd_tol=float(g["svd_tol"]), fp64=True)
    tri = g["tri"].reshape(-1, 3, 3)
    rng = np.random.default_rng(3)
    pts, owner = [], []
    for i in rng.choice(len(tri), 12, replace=False):
        P = port.flat_panel(*tri[i])
        c, nrm, d = P["centroid"], P["axis"][2], P["max_diag"]
        cand = [c]
        for h in (1e-9, 1e-3, 0.05, 0.4, 1.5, 2.9, 3.1, 5.0, 6.1, 9.0):
            cand += [c + h * d * nrm, c - h * d * nrm]
            if h >= 1e-3:  # closer above a vertex the formula loses digits to cancellation in both codes
                cand.append(tri[i][1] + h * d * nrm)
        cand += [c + 2.0 * d * P["axis"][0], c + 4.0 * d * (P["axis"][0] + P["axis"][1])]
        for p in cand:
            pts.append(p)
            owner.append(i)
    pts = np.array(pts)
    s_ref, d_ref = rs.panel_integrals(0, 0.0, pts, np.array(owner))
    for k, (p, i) in enumerate(zip(pts, owner)):
        s, d = port.laplace_panel(p, port.flat_panel(*tri[i]))
        assert abs(s - s_ref[k]) <= 1e-12 * max(1.0, abs(s_ref[k])), (k, s, s_ref[k])
        assert abs(d - d_ref[k]) <= 1e-12 * max(1.0, abs(d_ref[k])), (k, d, d_ref[k])


@pytest.mark.skipif(not ref.available(fp64=True), reason="oracle/_ref not built")
@pytest.mark.parametrize("kappa", [0.125, 1.0])
def test_restated_yukawa_integrals_match_compiled_reference(kappa):
    """The Yukawa panel integrals (edge line integrals, FlatIntegration.c:431-949, 1035-1049) point by
    point against the reference's Integration: points on the panel's plane (inside and outside), just
    off it, above a vertex, and at several distances along the normal."""
    g = load("blob3")
    with ref.stdout_to_stderr():
        rs = ref.RefSystem(g["tri"], g["qpos"], g["q"], float(g["eps_in"]), float(g["eps_out"]),
                           float(g["kappa"]), svd_tol=float(g["svd_tol"]), fp64=True)
    tri = g["tri"].reshape(-1, 3, 3)
    pts, owner = [], []
    for i in np.random.default_rng(4).choice(len(tri), 8, replace=False):
        P = port.flat_panel(*tri[i])
        c, nrm, d = P["centroid"], P["axis"][2], P["max_diag"]
        for h in (0.0, 1e-9, 1e-3, 0.05, 0.4, 1.5, 3.0, 7.0, 20.0):
            for p in (c + h * d * nrm, c - h * d * nrm, tri[i][1] + max(h, 1e-3) * d * nrm,
                      c + (h + 0.5) * d * P["axis"][0]):
                pts.append(p)
                owner.append(i)
    pts = np.array(pts)
    s_ref, d_ref = rs.panel_integrals(1, kappa, pts, np.array(owner))
    for k, (p, i) in enumerate(zip(pts, owner)):
        s, d = port.yukawa_panel(p, port.flat_panel(*tri[i]), kappa)
        assert abs(s - s_ref[k]) <= 1e-12 * max(1.0, abs(s_ref[k])), (k, s, s_ref[k])
        assert abs(d - d_ref[k]) <= 1e-12 * max(1.0, abs(d_ref[k])), (k, d, d_ref[k])
