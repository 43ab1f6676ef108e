"""The analytic sphere energies of the oracle (Born, Kirkwood with salt) against the
compiled reference's own boundary-element solve: the reference converges to them at
second order in the mesh size, so a level-3 icosphere (1 280 panels) is within 1 %.
CPU only; needs the compiled reference (oracle/_ref)."""
import numpy as np
import pytest

import analytic  # oracle
import ref  # oracle
from fftsvd_b200 import meshes

# four charges off the centre of a 10 A sphere
RADIUS = 10.0
POS = np.array([[0.0, 0.0, 0.0], [3.0, 1.0, -2.0], [-2.5, 4.0, 1.5], [0.5, -5.0, 3.0]])
Q = np.array([0.7, -0.4, 0.5, -0.3])


def test_kirkwood_reduces_to_born():
    for kappa in (0.0, 0.125):
        assert analytic.kirkwood_energy(RADIUS, [[0, 0, 0]], [1.0], 4.0, 80.0, kappa) == pytest.approx(
            analytic.born_energy(RADIUS, 1.0, 4.0, 80.0, kappa), rel=1e-14)
    assert analytic.born_energy(10.0, 1.0, 1.0, 80.0) == pytest.approx(-332.112 / 20.0 * (1 - 1 / 80.0), rel=1e-15)


def test_kirkwood_series_converged():
    e60 = analytic.kirkwood_energy(RADIUS, POS, Q, 4.0, 80.0, 0.125, nmax=60)
    e80 = analytic.kirkwood_energy(RADIUS, POS, Q, 4.0, 80.0, 0.125, nmax=80)
    assert abs(e60 - e80) < 1e-13 * abs(e60)


@pytest.mark.skipif(not ref.available(True), reason="compiled reference (oracle/_ref) not built")
@pytest.mark.parametrize("kappa", [0.0, 0.125])
def test_reference_solve_approaches_kirkwood(kappa):
    tri = meshes.icosphere(3, RADIUS)
    r = ref.RefSystem(tri, POS, Q, 4.0, 80.0, kappa, svd_tol=1e-5, fp64=True)
    sol, _ = r.solve(r.rhs(), 1e-8)
    e = r.energy(r.reaction(sol))
    r.close()
    exact = analytic.kirkwood_energy(RADIUS, POS, Q, 4.0, 80.0, kappa)
    # measured 7.1e-3 (kappa 0) and 7.0e-3 (kappa 0.125) at level 3, 1.8e-3 and 1.7e-3 at level 4
    assert abs(e - exact) < 1e-2 * abs(exact), (e, exact)
