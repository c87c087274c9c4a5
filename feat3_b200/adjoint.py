"""torch.autograd binding of the hand-written adjoint (gradient test harness only).

``PoissonObjective.apply(k, mg_factory, rhs_kind, u_target)`` returns
J(k) = 1/2 ||u(k) - u_target||^2 where A(k) u = f is solved by the native MG-PCG; its
backward pass calls ``fb_mg_adjoint_grad`` (transposed MG-PCG solve plus the element
gradient kernel) instead of differentiating through the solver.
"""
from __future__ import annotations

import torch


class PoissonObjective(torch.autograd.Function):
    @staticmethod
    def forward(ctx, k, mg_factory, rhs_kind, u_target):
        mg = mg_factory(k.detach())
        rhs = mg.assemble_rhs(rhs_kind)
        res = mg.solve(rhs, record=False)
        u = res["u"]
        d = u - u_target
        J = 0.5 * torch.dot(d, d)
        ctx.mg, ctx.u, ctx.u_target = mg, u, u_target
        return J

    @staticmethod
    def backward(ctx, gJ):
        _, g, _ = ctx.mg.adjoint_grad(ctx.u, ctx.u_target)
        return gJ * g, None, None, None
