"""torch.autograd binding of the forward projector (no reference counterpart).

`project(projector, *volumes)` returns (I, IAbsorb) as ctfp_forward computes
them; their backward is ctfp_backward from the L checkpoint saved by the
forward.  The binding holds no compute of its own: both directions call
libctfp.so through `Projector`.
"""
from __future__ import annotations

import torch

from .projector import Projector


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
