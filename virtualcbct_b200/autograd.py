"""Differentiable polychromatic projection for material decomposition.

``project(volumes, projector)`` maps six float element volumes (densities x
1000, layout [Z][nmat][N][N], CUDA float32) to the spectral projections
[V][H][W] through the CUDA forward kernel; its backward is the hand-written
adjoint kernel (``vcbct_projector_adjoint``), which recomputes each ray's
spectral state instead of storing it.  No reference counterpart: the
reference's nearest analogue is the unused sensitivity backprojection of
Release_CBCT_Projection_CM/lengthproj.cpp:10-131.
"""
from __future__ import annotations

import torch

from .projector import Projector, _volume_key


class _MbfpaProject(torch.autograd.Function):
    @staticmethod
    def forward(ctx, volumes: torch.Tensor, projector: Projector):
        if not volumes.is_cuda or volumes.dtype != torch.float32:
            raise TypeError("volumes must be a CUDA float32 tensor [Z][nmat][N][N]")
        vol = volumes.detach().contiguous()
        projector.load_volume_f32(vol)
        out = projector.forward()
        ctx.projector = projector
        ctx.save_for_backward(vol)
        return out

    @staticmethod
    def backward(ctx, grad_out: torch.Tensor):
        (vol,) = ctx.saved_tensors
        p: Projector = ctx.projector
        # the adjoint reads the float volume the forward used: reload it only
        # if the projector has been given another volume since
        if p.loaded != _volume_key("f32", vol):
            p.load_volume_f32(vol)
        grad = torch.zeros_like(vol)
        p.adjoint(grad_out.contiguous().float(), grad)
        return grad, None


def project(volumes: torch.Tensor, projector: Projector) -> torch.Tensor:
    """Differentiable spectral forward projection of float element volumes."""
    return _MbfpaProject.apply(volumes, projector)


def decomposition_step(volumes: torch.Tensor, target: torch.Tensor, projector: Projector,
                       lr: float = 0.0):
    """One gradient step of least-squares material decomposition:
    loss = 0.5 * sum (project(volumes) - target)^2.  Returns (loss, grad) and,
    when lr > 0, updates ``volumes`` in place (clamped at zero)."""
    v = volumes.detach().requires_grad_(True)
    pred = project(v, projector)
    loss = 0.5 * torch.sum((pred - target) ** 2)
    (grad,) = torch.autograd.grad(loss, v)
    if lr > 0.0:
        with torch.no_grad():
            volumes.sub_(lr * grad).clamp_(min=0.0)
    return loss.detach(), grad
