"""torch.autograd wrappers of the adjoint solves.

FaddeevU: U(theta) is the on-shell U of one channel for the potential
V = V0 + sum_k theta_k dV_k with the wave-packet basis and the resolvent held
fixed (the arguments of solve_faddeev_equations, tt_solve_faddeev_adjoint).
RunChannelU: U of one channel of a run as a function of its low-energy
constants, the total derivative, as a forward/backward pair on the run handle.
Backward returns Re(sum conj(grad_U) dU/dtheta_k), PyTorch's convention for
real parameters and complex outputs.  torch is needed only by this module."""
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


class RunChannelU(torch.autograd.Function):
    """U of one channel of a run as a function of offsets theta of the
    potential's low-energy constants (the run option lec_offsets).  forward is
    tt_run_adjoint_forward, which keeps the LU factors in the run; backward is
    tt_run_adjoint_backward with the cotangent: the total derivative (the SWP
    basis, deuteron energy and resolvent move with the constants), from the
    kept factors, one transposed solve per deuteron row and energy."""

    @staticmethod
    def forward(ctx, theta, opts, chn, precision):
        from . import Run

        th = theta.detach().cpu().numpy().astype(np.float64)
        run = Run(**opts, lec_offsets=",".join(repr(float(x)) for x in th))
        U, _ = run.adjoint_forward(chn, precision)
        ctx.run = run
        ctx.chn = chn
        return torch.from_numpy(U)

    @staticmethod
    def backward(ctx, grad_U):
        run = ctx.run
        dV = [run.lec_derivative(k) for k in range(len(run.lecs()))]
        g, _ = run.adjoint_backward(ctx.chn, np.stack([d[0] for d in dV]), np.stack([d[1] for d in dV]),
                                    grad_U.detach().cpu().numpy())
        run.close()
        return torch.from_numpy(g), None, None, None


def u_of_lecs(theta, opts, chn, precision=PRECISION_MIXED):
    """U of channel chn of the run configured by opts, for offsets theta
    (float64 tensor [n_lecs]) of its low-energy constants; differentiable."""
    return RunChannelU.apply(theta, opts, chn, precision)
