"""Differentiable solve: a torch.autograd.Function over the forward and the
adjoint C entry points (helm_solve / helm_solve_adjoint).

    u = helmholtz_solve(plan, f, lam, gl=None, gr=None)

``lam`` is a 0-dim float64 CUDA tensor holding the plan's lambda; it is an
input only so that autograd can return dL/dlambda (the plan's operators are
built for that value, and a different value is rejected).  Gradients:
dL/df from the transposed solve A^-T ubar (zero on the GLL boundary slots,
which the solve never reads), dL/dgl and dL/dgr from its boundary slots, and
dL/dlambda = sum over the interior nodes of (dL/df) * u.
"""
from __future__ import annotations

from typing import Optional

import torch

from .solver import _PlanBase


class HelmholtzSolveFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, f, lam, gl, gr, plan: _PlanBase):
        if abs(float(lam) - float(plan.Lambda)) > 1e-14 * max(1.0, abs(float(plan.Lambda))):
            raise ValueError("lam differs from the plan's lambda; build a plan for the new value")
        u = plan.SolvePDE(f.detach().contiguous(), None if gl is None else gl.detach().contiguous(),
                          None if gr is None else gr.detach().contiguous())
        ctx.plan = plan
        ctx.has_bc = (gl is not None, gr is not None)
        ctx.save_for_backward(u)
        return u

    @staticmethod
    def backward(ctx, ubar):
        (u,) = ctx.saved_tensors
        want_lam = ctx.needs_input_grad[1]
        want_bc = ctx.needs_input_grad[2] or ctx.needs_input_grad[3]
        fbar, lbar, glb, grb = ctx.plan.SolveAdjoint(ubar.contiguous().to(torch.float64),
                                                     u=u.to(torch.float64) if want_lam else None, want_bc=want_bc)
        gf = fbar.to(u.dtype) if ctx.needs_input_grad[0] else None
        gl_ = glb if (want_bc and ctx.has_bc[0] and ctx.needs_input_grad[2]) else None
        gr_ = grb if (want_bc and ctx.has_bc[1] and ctx.needs_input_grad[3]) else None
        return gf, (lbar.reshape(()) if want_lam else None), gl_, gr_, None


def helmholtz_solve(plan: _PlanBase, f: torch.Tensor, lam: torch.Tensor, gl: Optional[torch.Tensor] = None,
                    gr: Optional[torch.Tensor] = None) -> torch.Tensor:
    return HelmholtzSolveFunction.apply(f, lam, gl, gr, plan)
