"""torch.autograd wrapper of the adjoint solve (tt_solve_faddeev_adjoint).

U(theta) is the on-shell U of one channel for the potential
V = V0 + sum_k theta_k dV_k with the wave-packet basis and the resolvent held
fixed (the arguments of solve_faddeev_equations); backward returns
Re(sum conj(grad_U) dU/dtheta_k), PyTorch's convention for real parameters and
complex outputs.  torch is needed only by this module."""
import numpy as np
import torch

from . import PRECISION_MIXED, solve_faddeev_adjoint


class FaddeevU(torch.autograd.Function):
    @staticmethod
    def forward(ctx, theta, problem):
        th = theta.detach().cpu().numpy().astype(np.float64)
        p = problem
        Vu = p["V_unco"] + np.tensordot(th, p["dV_unco"], axes=1)
        Vc = p["V_coup"] + np.tensordot(th, p["dV_coup"], axes=1) if np.size(p["V_coup"]) else p["V_coup"]
        U, dU, _ = solve_faddeev_adjoint(p["G"], p["P_val"], p["P_row"], p["P_colptr"], Vu, Vc, p["swp"], p["q_idx"],
                                         p["deut"], p["pw"], p["dV_unco"], p["dV_coup"],
                                         precision=p.get("precision", PRECISION_MIXED), **p.get("rp", {}))
        ctx.save_for_backward(torch.from_numpy(dU))
        return torch.from_numpy(U)

    @staticmethod
    def backward(ctx, grad_U):
        (J,) = ctx.saved_tensors
        g = (grad_U.conj().unsqueeze(0) * J).sum(dim=1).real
        return g.to(torch.float64), None


def u_of_theta(theta, problem):
    """U for parameters theta (float64 tensor [n_theta]); differentiable."""
    return FaddeevU.apply(theta, problem)
