"""The GPU solve against the analytic Kirkwood energy of four off-centre charges in a
sphere with salt outside (kappa 0.125 1/A), on a level-4 icosphere (5 120 panels).  The
discretisation error of the boundary-element method is the reference's own: the GPU
energy equals the compiled reference's on the same mesh to the solver tolerance, and
both lie within 2.5e-3 of the exact energy (measured 1.7e-3)."""
import numpy as np
import pytest

import analytic  # oracle
import ref  # oracle
from fftsvd_b200 import meshes
from fftsvd_b200.surface import Surface

pytestmark = pytest.mark.gpu

RADIUS = 10.0
POS = np.array([[0.0, 0.0, 0.0], [3.0, 1.0, -2.0], [-2.5, 4.0, 1.5], [0.5, -5.0, 3.0]])
Q = np.array([0.7, -0.4, 0.5, -0.3])


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_kirkwood_sphere_with_salt(gpu, precision):
    kappa, eps_in, eps_out = 0.125, 4.0, 80.0
    tri = meshes.icosphere(4, RADIUS)
    s = Surface.from_problem(tri, POS, Q, eps_in, eps_out, kappa, svd_tol=1e-5)
    r = s.solve(s.rhs(), precision=precision, tol=1e-8)
    e = s.energy(s.reaction_potentials(r.solution))
    s.close()
    exact = analytic.kirkwood_energy(RADIUS, POS, Q, eps_in, eps_out, kappa)
    assert abs(e - exact) < 2.5e-3 * abs(exact), (e, exact)
    if ref.available(True):
        rs = ref.RefSystem(tri, POS, Q, eps_in, eps_out, kappa, svd_tol=1e-5, fp64=True)
        sol, _ = rs.solve(rs.rhs(), 1e-8)
        e_ref = rs.energy(rs.reaction(sol))
        rs.close()
        assert abs(e - e_ref) < 1e-6 * abs(e_ref), (e, e_ref)
