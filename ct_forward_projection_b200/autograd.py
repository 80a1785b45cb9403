"""torch.autograd bindings of the forward projector (no reference counterpart).

`project(projector, *volumes)` returns (I, IAbsorb) as ctfp_forward computes
them; their backward is ctfp_backward from the L checkpoint saved by the
forward.  `LogIntensityLoss(projector)(target, *volumes)` is the scalar
sum (log I - log T)^2 with its gradient from the fused forward + loss + adjoint
kernel (ctfp_batch_forward_adjoint on a one-item batch), which needs no L
checkpoint.  The bindings hold no compute of their own: every direction calls
libctfp.so through `Projector` and `Batch`.
"""
from __future__ import annotations

import torch

from .projector import Batch, Projector


class _PolyForward(torch.autograd.Function):
    @staticmethod
    def forward(ctx, projector: Projector, *volumes):
        vols = [v.detach().contiguous() for v in volumes]
        out = projector.forward(vols, want_L=True)
        ctx.projector = projector
        ctx.save_for_backward(out["L"])
        ctx.mark_non_differentiable(out["I0"])
        return out["I"], out["IAbsorb"], out["I0"]

    @staticmethod
    def backward(ctx, gI, gIAbsorb, _gI0):
        (L,) = ctx.saved_tensors
        pr = ctx.projector
        grads = pr.backward(L, gI=None if gI is None else gI.contiguous(),
                            gIAbsorb=None if gIAbsorb is None else gIAbsorb.contiguous())
        return (None, *grads)


def project(projector: Projector, *volumes: torch.Tensor):
    """(I, IAbsorb, I0) of the M density maps `volumes`, differentiable in them."""
    if len(volumes) != projector.M:
        raise ValueError(f"expected {projector.M} volumes, got {len(volumes)}")
    return _PolyForward.apply(projector, *volumes)


class _FusedLogLoss(torch.autograd.Function):
    @staticmethod
    def forward(ctx, owner, target, *volumes):
        pr = owner.projector
        vols = [v.detach().contiguous() for v in volumes]
        grads = [torch.zeros_like(v) for v in vols]
        loss = torch.zeros(1, device=vols[0].device)
        owner.batch.forward_adjoint([vols], [target.detach().contiguous()], grads=[grads], loss=loss)
        ctx.save_for_backward(*grads)
        return loss.reshape(())

    @staticmethod
    def backward(ctx, g):
        return (None, None, *[g * x for x in ctx.saved_tensors])


class LogIntensityLoss:
    """loss = sum over rays of (log I - log T)^2 for one projector, computed
    with its gradient in one fused launch; T (the target intensities, shape of
    I, > 0) is a constant.  Owns a one-item batch: call close() (or use it as a
    context manager) before closing the projector."""

    def __init__(self, projector: Projector):
        self.projector = projector
        self.batch = Batch([projector])

    def __call__(self, target: torch.Tensor, *volumes: torch.Tensor) -> torch.Tensor:
        if len(volumes) != self.projector.M:
            raise ValueError(f"expected {self.projector.M} volumes, got {len(volumes)}")
        if tuple(target.shape) != tuple(self.projector.shape_proj):
            raise ValueError(f"target must have shape {tuple(self.projector.shape_proj)}")
        return _FusedLogLoss.apply(self, target, *volumes)

    def close(self) -> None:
        self.batch.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
