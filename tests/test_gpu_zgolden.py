"""The GPU path against the committed golden fixtures (tests/golden/*.npz, the
compiled reference's FP64 results), with no compiled reference needed at run
time.  The surface is built by the library's own host setup from the fixture's
inputs.  Tolerances as in the live-reference tests: FP64 matvec 1e-10, FP32
matvec 2e-5, right-hand side 1e-13, preconditioner 1e-6, reaction potentials
1e-11, and energies within 2e-6 of the reference's, both solves stopping at a
relative residual of 1e-6."""
import os

import numpy as np
import pytest

from fftsvd_b200.surface import Surface
from helpers import GOLDEN, rel

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=["born3", "blob3"])
def golden_surface(request, gpu):
    g = np.load(os.path.join(GOLDEN, request.param + ".npz"))
    g = {k: g[k] for k in g.files}
    s = Surface.from_problem(g["tri"], g["qpos"], g["q"], float(g["eps_in"]), float(g["eps_out"]),
                             float(g["kappa"]), svd_tol=float(g["svd_tol"]))
    yield g, s
    s.close()


def test_operator_pieces_match_golden(golden_surface):
    g, s = golden_surface
    assert rel(s.matvec(g["x"], "fp64"), g["y64"]) < 1e-10
    assert rel(s.matvec(g["x"], "fp32"), g["y64"]) < 2e-5
    assert rel(s.rhs(), g["rhs"]) < 1e-13
    assert rel(s.precond_solve(g["rhs"]), g["z"]) < 1e-6
    assert rel(s.reaction_potentials(g["sol"]), g["phi"]) < 1e-11


def test_solve_energy_matches_golden(golden_surface):
    g, s = golden_surface
    dG = float(g["dG"])
    for prec in ("fp64", "mixed"):
        r = s.solve(g["rhs"], precision=prec, tol=float(g["gmres_tol"]))
        e = s.energy(s.reaction_potentials(r.solution))
        assert abs(e - dG) < 2e-6 * abs(dG), (prec, e, dG)
