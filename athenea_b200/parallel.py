"""Data parallelism over views: one process a GPU, the cloud replicated.

Views are independent units of the rasteriser's work, so a training step
shards them across ranks and needs one exchange: the per-Gaussian gradients,
summed over every rank's views, with one all-reduce of one flat FP32 buffer
(60 floats a Gaussian: means + opacity logit 4, log scales 4, quaternion 4, SH
48). The forward has no exchange at all. The reference is single-device
throughout and has none of this.
"""
from __future__ import annotations

import torch
import torch.distributed as dist

from .raster import Params


def shard_views(views: int, rank: int, world: int) -> range:
    """The views rank `rank` of `world` draws: contiguous, sizes differing by at most one."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    base, extra = divmod(views, world)
    first = rank * base + min(rank, extra)
    return range(first, first + base + (1 if rank < extra else 0))


class GradientBuffer:
    """A Gaussian cloud's gradients as views into one flat FP32 buffer, in
    ath_param_grads' layout, so that summing them over ranks is one all-reduce."""

    def __init__(self, count: int, sh_stride: int = 48, sh_degree: int = 3, device="cuda"):
        n = count
        self.flat = torch.zeros(n * (12 + sh_stride), dtype=torch.float32, device=device)
        f = self.flat
        self.params = Params(f[:4 * n].view(n, 4), f[4 * n:8 * n].view(n, 4), f[8 * n:12 * n].view(n, 4),
                             f[12 * n:].view(n, sh_stride), sh_degree)

    def allreduce(self, group=None) -> None:
        """Sums the buffer over the ranks of `group` (the default group when None)."""
        if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
            dist.all_reduce(self.flat, op=dist.ReduceOp.SUM, group=group)
