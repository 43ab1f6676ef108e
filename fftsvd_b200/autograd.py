"""A thin torch.autograd.Function over the adjoint C entry point, for testing the
derivatives through autograd (gradcheck-style comparisons with finite differences).

    energy = SolvationEnergy.apply(surface, positions, charges)
    energy.backward()   # positions.grad = d dG / d x, charges.grad = d dG / d q

`positions` (nq x 3, A) and `charges` (nq, e) are CPU float64 tensors; the surface's
charges are replaced by them on every forward call.  The energy is in kcal/mol.
"""
import numpy as np
import torch


class SolvationEnergy(torch.autograd.Function):
    @staticmethod
    def forward(ctx, surface, positions, charges, precision="fp64", tol=1e-8):
        pos = positions.detach().cpu().numpy().astype(np.float64)
        q = charges.detach().cpu().numpy().astype(np.float64)
        surface.set_charges(pos, q)
        energy, dq, dx, _ = surface.adjoint(precision=precision, tol=tol)
        ctx.save_for_backward(torch.from_numpy(dx), torch.from_numpy(dq))
        return torch.tensor(energy, dtype=torch.float64)

    @staticmethod
    def backward(ctx, grad):
        dx, dq = ctx.saved_tensors
        return None, grad * dx, grad * dq, None, None
