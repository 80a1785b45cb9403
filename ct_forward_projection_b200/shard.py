"""One object's views split across the ranks of a torch.distributed group
(no reference counterpart; the reference runs one GPU).

Every ray of the forward is independent, so rank r projects the contiguous
views `view_range(P, r, world)` on its own GPU with `ctfp_forward_views`; the
projection needs no collective (an optional all-gather assembles the full
stack).  The adjoint of the view-sharded forward is the sum over ranks of each
rank's partial gradient, one all-reduce per material volume (NCCL over
NVLink on a multi-GPU node).
"""
from __future__ import annotations

from typing import Sequence


def view_range(n_views: int, rank: int, world: int) -> tuple[int, int]:
    """(first view, count) of `rank`: contiguous, sizes differ by at most one."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("need 0 <= rank < world")
    base, extra = divmod(int(n_views), world)
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


class ViewShardedProjector:
    """Wraps one rank's projector (a `Projector` on this rank's GPU, built for
    the full geometry) and the process group."""

    def __init__(self, projector, group=None):
        import torch.distributed as dist
        self.pr = projector
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        P = int(projector.shape_proj[0])
        self.views = view_range(P, self.rank, self.world)

    def forward(self, volumes: Sequence, want_L: bool = False, gather: bool = False) -> dict:
        """This rank's views (compact I, IAbsorb[, L]); with gather=True also
        "I_full" and "IAbsorb_full", the whole [P][V][U] stack on every rank."""
        out = self.pr.forward(volumes, want_L=want_L, views=self.views)
        if gather:
            out["I_full"] = self._gather(out["I"])
            out["IAbsorb_full"] = self._gather(out["IAbsorb"])
        return out

    def backward(self, L, gI=None, gIAbsorb=None, grads=None) -> list:
        """dLoss/drho_m of the whole projection on every rank: this rank's
        partial adjoint over its views, summed across ranks."""
        import torch.distributed as dist
        grads = self.pr.backward(L, gI=gI, gIAbsorb=gIAbsorb, grads=grads, views=self.views)
        for g in grads:
            dist.all_reduce(g, op=dist.ReduceOp.SUM, group=self.group)
        return grads

    def _gather(self, local):
        import torch
        import torch.distributed as dist
        P = int(self.pr.shape_proj[0])
        counts = [view_range(P, r, self.world)[1] for r in range(self.world)]
        n_max = max(counts)
        pad = torch.zeros((n_max,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
        pad[: local.shape[0]] = local
        parts = [torch.empty_like(pad) for _ in range(self.world)]
        dist.all_gather(parts, pad, group=self.group)
        return torch.cat([p[:c] for p, c in zip(parts, counts)], dim=0)
