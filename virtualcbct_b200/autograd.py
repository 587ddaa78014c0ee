"""Differentiable polychromatic projection for material decomposition.

``project(volumes, projector)`` maps six float element volumes (densities x
1000, layout [Z][nmat][N][N], CUDA float32) to the spectral projections
[V][H][W] through the CUDA forward kernel; its backward is the hand-written
adjoint kernel, which recomputes each ray's spectral state (the per-energy
attenuation and its derivative) instead of storing it.  The six per-ray
element path integrals it is recomputed from are either kept from the
forward launch (``vcbct_projector_forward_state`` / ``_adjoint_state``, 24 B
per ray) or re-marched (``vcbct_projector_adjoint``) when keeping them would
exceed ``keep_limit`` bytes.  No reference counterpart: the reference's
nearest analogue is the unused sensitivity backprojection of
Release_CBCT_Projection_CM/lengthproj.cpp:10-131.
"""
from __future__ import annotations

import torch

from .projector import Projector, _volume_key


# Bytes of per-ray path integrals kept between the passes; None: keep them
# when they take at most a quarter of the device's free memory (11 GB for 720
# views of 800 x 800 is kept on a 180 GB GPU).
KEEP_LIMIT = None


def _keep(nbytes: int, keep_limit) -> bool:
    if keep_limit is None:
        free, _ = torch.cuda.mem_get_info()
        return nbytes <= free // 4
    return nbytes <= keep_limit


class _MbfpaProject(torch.autograd.Function):
    @staticmethod
    def forward(ctx, volumes: torch.Tensor, projector: Projector, keep_limit):
        if not volumes.is_cuda or volumes.dtype != torch.float32:
            raise TypeError("volumes must be a CUDA float32 tensor [Z][nmat][N][N]")
        vol = volumes.detach().contiguous()
        projector.load_volume_f32(vol)
        g = projector.geom
        if _keep(g.V * g.H * g.W * g.nmat * 4, keep_limit):
            out, L = projector.forward_state()
            ctx.save_for_backward(vol, L)
        else:
            out = projector.forward()
            ctx.save_for_backward(vol)
        ctx.projector = projector
        return out

    @staticmethod
    def backward(ctx, grad_out: torch.Tensor):
        saved = ctx.saved_tensors
        vol = saved[0]
        p: Projector = ctx.projector
        # the adjoint reads the float volume the forward used: reload it only
        # if the projector has been given another volume since
        if p.loaded != _volume_key("f32", vol):
            p.load_volume_f32(vol)
        grad = torch.zeros_like(vol)
        go = grad_out.contiguous().float()
        if len(saved) > 1:
            p.adjoint_state(saved[1], go, grad)
        else:
            p.adjoint(go, grad)
        return grad, None, None


def project(volumes: torch.Tensor, projector: Projector, keep_limit=KEEP_LIMIT) -> torch.Tensor:
    """Differentiable spectral forward projection of float element volumes.
    The per-ray path integrals are kept for the backward pass when they fit
    in ``keep_limit`` bytes (0: always re-march; None: a quarter of the free
    device memory)."""
    return _MbfpaProject.apply(volumes, projector, keep_limit)


def decomposition_step(volumes: torch.Tensor, target: torch.Tensor, projector: Projector,
                       lr: float = 0.0, keep_limit=KEEP_LIMIT):
    """One gradient step of least-squares material decomposition:
    loss = 0.5 * sum (project(volumes) - target)^2.  Returns (loss, grad) and,
    when lr > 0, updates ``volumes`` in place (clamped at zero)."""
    v = volumes.detach().requires_grad_(True)
    pred = project(v, projector, keep_limit)
    loss = 0.5 * torch.sum((pred - target) ** 2)
    (grad,) = torch.autograd.grad(loss, v)
    if lr > 0.0:
        with torch.no_grad():
            volumes.sub_(lr * grad).clamp_(min=0.0)
    return loss.detach(), grad
