"""torch.autograd bindings of the design objective.

``WorstCaseObjective.apply(coeff, grid, params)`` returns the tensor
``[lambda_max, volume, ss]`` of the robust spline design at the control
coefficients ``coeff`` (float64 CUDA tensor, ``grid.n_coeff`` entries).  The
forward pass runs the worst-case load search (Lanczos over multigrid solves)
on the GPU; the backward pass uses the hand-written adjoint of the same call
(sensitivity -u_w^T dK/drho u_w, Heaviside chain, spline adjoint, analytic
self-support derivative), returned by ``rso_design_gradient`` in one pass.
"""
import torch

from .rso import IterParams


class WorstCaseObjective(torch.autograd.Function):
    @staticmethod
    def forward(ctx, coeff, grid, params=None):
        vals, gl, gv, gs = grid.design_gradient(coeff.detach(), params or IterParams())
        ctx.save_for_backward(torch.stack([gl, gv, gs]))
        return torch.tensor([vals["lambda"], vals["volume"], vals["ss"]], dtype=torch.float64, device=coeff.device)

    @staticmethod
    def backward(ctx, grad_out):
        (jac,) = ctx.saved_tensors
        return grad_out.to(jac.dtype) @ jac, None, None


def worst_case_objective(coeff, grid, params=None):
    """[lambda_max, volume, ss] of the design at `coeff`, differentiable in `coeff`."""
    return WorstCaseObjective.apply(coeff, grid, params)
