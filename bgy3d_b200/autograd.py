"""The solvation free energy as a differentiable torch function.

``solvation_free_energy(q, sigma, epsilon, x, solvent, settings, chi)``
returns mu (kcal/mol, a 0-d FP64 tensor) of the solute whose sites carry
charges q [n], LJ sigma [n] and epsilon [n] and positions x [n][3]; its
backward pass uses the adjoint gradient of rism3d_solute_grad, so
``mu.backward()`` fills q.grad, sigma.grad, epsilon.grad and x.grad (x.grad
is minus the solvation force on each site).  The forward solve and the
gradient run on the current CUDA device through librism3d.so; the tensors
themselves may live anywhere (they are read and written on the host).
"""
import numpy as np
import torch

from .solver import hnc3d_solute_grad


class SoluteFreeEnergy(torch.autograd.Function):
    """mu(q, sigma, epsilon, x) with the adjoint gradient in backward."""

    @staticmethod
    def forward(ctx, q, sigma, epsilon, x, solvent, settings, chi, names=None):
        n = q.shape[0]
        qh, sh, eh = (a.detach().to("cpu", torch.float64).numpy() for a in (q, sigma, epsilon))
        xh = x.detach().to("cpu", torch.float64).numpy().reshape(n, 3)
        solute = [dict(name=(names[i] if names else f"S{i}"), x=tuple(float(v) for v in xh[i]),
                       sigma=float(sh[i]), epsilon=float(eh[i]), charge=float(qh[i])) for i in range(n)]
        out = hnc3d_solute_grad(solute, solvent, settings, chi)
        g = out["gradient"]
        ctx.xshape = x.shape
        ctx.save_for_backward(*(torch.from_numpy(np.array(g[k])).to(ref.device)
                                for k, ref in (("charge", q), ("sigma", sigma), ("epsilon", epsilon), ("x", x))))
        return torch.tensor(out["free-energy"], dtype=torch.float64, device=q.device)

    @staticmethod
    def backward(ctx, gmu):
        dq, ds, de, dx = ctx.saved_tensors
        return (gmu * dq, gmu * ds, gmu * de, gmu * dx.reshape(ctx.xshape), None, None, None, None)


def solvation_free_energy(q, sigma, epsilon, x, solvent, settings, chi, names=None):
    """mu of the solute (q, sigma, epsilon [n]; x [n][3]) in ``solvent``,
    differentiable in all four (see the module docstring)."""
    return SoluteFreeEnergy.apply(q, sigma, epsilon, x, solvent, settings, chi, names)
