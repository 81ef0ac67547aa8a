"""torch.autograd bindings of the nonlinear term, the residual J and the
time stepper.

``rhs_nonlinear(box, uhat)`` is differentiable: its backward is the exact
adjoint kernel chain of libdnsbox_gpu.so (``dnsbox_rhs_nonlinear_vjp``), the
transpose of the linearised dealiased, projected nonlinear term of rhs.f90:18-135.
Gradients follow torch's convention for complex tensors (the Euclidean
gradient on the real and imaginary parts), so a real loss L gives
``uhat.grad = dL/dRe(uhat) + i dL/dIm(uhat)``.
"""
from __future__ import annotations

import torch


class RhsNonlinear(torch.autograd.Function):
    @staticmethod
    def forward(ctx, uh, box):
        out, _ = box.rhs_nonlinear(uh.detach().contiguous(), want_eband=False)
        ctx.box = box
        ctx.save_for_backward(uh)
        return out

    @staticmethod
    def backward(ctx, g):
        (uh,) = ctx.saved_tensors
        return ctx.box.rhs_nonlinear_vjp(uh.detach().contiguous(), g.contiguous()), None


def rhs_nonlinear(box, uh: torch.Tensor) -> torch.Tensor:
    """Differentiable rhs_nonlinear (N(uhat) including band/fixed forcing)."""
    return RhsNonlinear.apply(uh, box)


class Residual(torch.autograd.Function):
    """J(uhat) = 1/2 <r, H^-1 r>, r = L uhat + N(uhat) + f, with its exact gradient."""

    @staticmethod
    def forward(ctx, uh, box):
        J, grad = box.residual_grad(uh.detach().contiguous())
        ctx.save_for_backward(grad)
        return torch.tensor(J, dtype=torch.float64, device=uh.device)

    @staticmethod
    def backward(ctx, gJ):
        (grad,) = ctx.saved_tensors
        return grad * gJ.to(grad.real.dtype), None


def residual(box, uh: torch.Tensor) -> torch.Tensor:
    return Residual.apply(uh, box)


class HeunSteps(torch.autograd.Function):
    """u(T) = S^nsteps(u0) for fixed-dt IF-Heun steps; the backward is the
    checkpointed step-transpose chain (dnsbox_heun_steps_vjp)."""

    @staticmethod
    def forward(ctx, u0, box, nsteps, every):
        u = u0.detach().contiguous().clone()
        box.step(u, nsteps, diag=False)
        ctx.box, ctx.nsteps, ctx.every = box, nsteps, every
        ctx.save_for_backward(u0)
        return u

    @staticmethod
    def backward(ctx, gT):
        (u0,) = ctx.saved_tensors
        g0 = ctx.box.heun_steps_vjp(u0.detach().contiguous(), ctx.nsteps, gT.contiguous(), every=ctx.every)
        return g0, None, None, None


def heun_steps(box, u0: torch.Tensor, nsteps: int, every: int = 32) -> torch.Tensor:
    """Differentiable state after nsteps fixed-dt IF-Heun steps from u0."""
    return HeunSteps.apply(u0, box, nsteps, every)
