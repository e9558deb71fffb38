"""Compliance and its design gradients as a torch.autograd.Function.

c(E, X) = f^T u with K(E, X) u = f (linear elasticity, design-independent load, zero
prescribed values). Forward: device assembly + device CG solve through the C ABI.
Backward: the closed-form adjoint kernel (cxg_adjoint_compliance), dc/dE per element
and dc/dX per node coordinate. The reference offers coordinate sensitivities by
central differences of the reduced operator (src/numerics/sensitivity.cpp:112-151)
and no per-element-modulus variable.
"""
from __future__ import annotations

import torch

from .assembly import Model, Plan


class ComplianceFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, young, coords, plan: Plan, f_ext, rtol, max_iter):
        plan.update_young(young.detach())
        plan.update_coords(coords.detach().reshape(-1))
        vals, rhs = plan.assemble_linear(f_ext)
        x, iters, rel = plan.solve_cg(vals, rhs, rtol=rtol, max_iter=max_iter)
        u = plan.expand(x)
        ctx.plan = plan
        ctx.save_for_backward(u)
        ctx.solve_info = (iters, rel)
        return torch.dot(rhs, x)

    @staticmethod
    def backward(ctx, grad_c):
        (u,) = ctx.saved_tensors
        dE, dX = ctx.plan.adjoint_compliance(u)
        return grad_c * dE, grad_c * dX, None, None, None, None


def compliance(young, coords, plan: Plan, f_ext, rtol=1e-12, max_iter=50000):
    """Differentiable compliance f^T u in young (E,) and coords (N, 3)."""
    f = torch.as_tensor(f_ext, dtype=torch.float64, device=plan.device)
    return ComplianceFunction.apply(young, coords, plan, f, rtol, max_iter)


def make_plan(model: Model) -> Plan:
    return Plan(model, "fp64")
