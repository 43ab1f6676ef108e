"""ORACLE — test infrastructure only (never imported by the product path).

Analytic reaction energies of point charges inside a dielectric sphere, the
exact solutions the boundary-element solve converges to as the sphere's mesh is
refined:

* Born (one charge at the centre, no salt):
  dG = 1/2 q^2 / a (1/eps_out - 1/eps_in)
* Kirkwood (1934, J. Chem. Phys. 2, 351): charges anywhere inside a sphere of
  radius a (dielectric eps_in), outside it a linearised Poisson-Boltzmann
  medium (eps_out, inverse Debye length kappa).  Inside, the reaction potential
  of a charge q at r_j is sum_n A_n r^n P_n(cos gamma) with

      A_n = q b^n / a^(2n+1) * ((n+1) + eps_out x_n / eps_in) / (eps_in n - eps_out x_n),

  b = |r_j|, x_n = z k_n'(z) / k_n(z) at z = kappa a (k_n the modified spherical
  Bessel function of the second kind; x_n = -(n+1) for kappa = 0).  It follows
  from continuity of phi and eps dphi/dr at r = a term by term in Legendre
  polynomials.

Energies in kcal/mol with the reference's constant 332.112 (FFTSVDsalt.c:167-170),
lengths in A, charges in e.  Both reduce to the reference's single-charge checks:
n = 0 with b = 0 gives the Born energy with the Debye-Hueckel factor 1/(1 + kappa a).
"""
from __future__ import annotations

import numpy as np

COULOMB = 332.112


def born_energy(a: float, q: float, eps_in: float, eps_out: float, kappa: float = 0.0) -> float:
    return 0.5 * COULOMB * q * q / a * (1.0 / (eps_out * (1.0 + kappa * a)) - 1.0 / eps_in)


def _log_derivative(n: int, z: float) -> float:
    """z k_n'(z) / k_n(z) for the modified spherical Bessel function of the second kind."""
    if z == 0.0:
        return -(n + 1.0)
    from scipy.special import spherical_kn
    return z * spherical_kn(n, z, derivative=True) / spherical_kn(n, z)


def kirkwood_energy(a: float, pos, q, eps_in: float, eps_out: float, kappa: float = 0.0,
                    nmax: int = 60) -> float:
    """0.5 * sum_i q_i phi_reac(r_i) * 332.112 for charges q at pos (n x 3, inside the sphere
    of radius a centred at the origin)."""
    from scipy.special import eval_legendre

    pos = np.asarray(pos, dtype=np.float64).reshape(-1, 3)
    q = np.asarray(q, dtype=np.float64).reshape(-1)
    r = np.linalg.norm(pos, axis=1)
    assert np.all(r < a), "charges must lie inside the sphere"
    # cos of the angle between every pair of position vectors (1 where one is the centre)
    with np.errstate(invalid="ignore", divide="ignore"):
        cosg = (pos @ pos.T) / np.outer(r, r)
    cosg = np.where(np.isfinite(cosg), np.clip(cosg, -1.0, 1.0), 1.0)
    z = kappa * a
    phi = np.zeros(len(q))
    for n in range(nmax + 1):
        x = _log_derivative(n, z)
        c = ((n + 1.0) + eps_out * x / eps_in) / (eps_in * n - eps_out * x) / a ** (2 * n + 1)
        # phi_i += sum_j q_j c (r_j r_i)^n P_n(cos gamma_ij)
        rr = np.outer(r, r) ** n
        phi += (rr * eval_legendre(n, cosg)) @ q * c
    return 0.5 * COULOMB * float(np.dot(q, phi))
