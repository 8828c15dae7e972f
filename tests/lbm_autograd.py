"""Gradient-check harness only: a thin torch.autograd.Function over the
engine's checkpointed adjoint (lbm_ke_gradient_async). Not part of the engine.

KineticEnergy.apply(u0, tau) returns J = sum 0.5 rho |u|^2 after `steps`
collide-stream steps started from f_eq(rho0 = 1, u0); its backward returns
dJ/du0 and dJ/dtau from the adjoint.
"""
import torch

import lbcube as E


def run_gradient(u0, tau, steps, interval, collision="BGK", lattice="D3Q19"):
    """(J, dJ/dtau, dJ/du0) from one call of the engine's gradient driver."""
    nz, ny, nx = u0.shape[1:]
    real = "double" if u0.dtype == torch.float64 else "float"
    rho0 = torch.ones(u0.shape[1:], dtype=u0.dtype, device=u0.device)
    nbytes = E.ke_gradient_workspace_bytes(lattice, real, nx, ny, nz, steps, interval)
    ws = torch.empty(nbytes, dtype=torch.uint8, device=u0.device)
    out = torch.zeros(2, dtype=torch.float64, device=u0.device)
    grad = torch.empty_like(u0)
    E.check(E.ke_gradient_async(lattice, real, collision, rho0, u0.contiguous(), nx, ny, nz, float(tau),
                                steps, interval, ws, nbytes, out, grad))
    torch.cuda.synchronize()
    return float(out[0]), float(out[1]), grad


class KineticEnergy(torch.autograd.Function):
    @staticmethod
    def forward(ctx, u0, tau, steps, interval, collision):
        J, dtau, grad = run_gradient(u0.detach(), float(tau), steps, interval, collision)
        ctx.save_for_backward(grad, torch.tensor(dtau, dtype=torch.float64))
        return torch.tensor(J, dtype=torch.float64, device=u0.device)

    @staticmethod
    def backward(ctx, g):
        grad, dtau = ctx.saved_tensors
        return g.to(grad.dtype) * grad, g.cpu() * dtau, None, None, None
