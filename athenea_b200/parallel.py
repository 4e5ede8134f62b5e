"""Data parallelism over views: one process a GPU, the cloud replicated.

Views are independent units of the rasteriser's work, so a training step
shards them across ranks and needs one exchange: the per-Gaussian gradients,
summed over every rank's views (60 floats a Gaussian: means + opacity logit 4,
log scales 4, quaternion 4, SH 48). The forward has no exchange at all. The
reference is single-device throughout and has none of this.

GradientBuffer sums them with one all-reduce of one flat FP32 buffer after the
step. BucketedGradients splits the Gaussians into consecutive buckets
(ath_gradient_bucket), each bucket's four arrays in one slice of its flat
buffer; the step's projection adjoint runs bucket by bucket and records an
event after each (ath_batch_set_buckets), so each bucket's all-reduce starts,
on a side stream, while the later buckets are still being computed.
"""
from __future__ import annotations

import ctypes as C

import torch
import torch.distributed as dist

from . import _native as N
from .raster import Params, _ptr


def gradient_bucket(count: int, buckets: int, k: int) -> tuple[int, int]:
    """ath_gradient_bucket: bucket k's first Gaussian and size (whole blocks of 128 Gaussians,
    sizes differing by at most one block, every Gaussian once)."""
    first, n = C.c_uint32(), C.c_uint32()
    N.check(N.lib().ath_gradient_bucket(count, buckets, k, C.byref(first), C.byref(n)))
    return first.value, n.value


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


class BucketedGradients:
    """A cloud's gradients in `buckets` consecutive Gaussian ranges: bucket k's means,
    scales, quats and SH (ath_param_grads' layout, its own Gaussians' rows) one after
    another in one contiguous slice of `flat`, so that one all-reduce sums a bucket."""

    def __init__(self, count: int, buckets: int, sh_stride: int = 48, sh_degree: int = 3, device="cuda"):
        self.count, self.sh_stride = count, sh_stride
        self.ranges = [gradient_bucket(count, buckets, k) for k in range(buckets)]
        per = 12 + sh_stride
        self.flat = torch.zeros(count * per, dtype=torch.float32, device=device)
        self.slices, self.params = [], []
        for first, n in self.ranges:
            f = self.flat[first * per:(first + n) * per]
            self.slices.append(f)
            self.params.append(Params(f[:4 * n].view(n, 4), f[4 * n:8 * n].view(n, 4), f[8 * n:12 * n].view(n, 4),
                                      f[12 * n:].view(n, sh_stride), sh_degree))

    def native(self):
        """The buckets' arrays as the array of ath_param_grads ath_batch_set_buckets takes."""
        arr = (N.ParamGrads * len(self.params))()
        for k, P in enumerate(self.params):
            arr[k] = N.ParamGrads(_ptr(P.means), _ptr(P.scales), _ptr(P.quats), _ptr(P.sh))
        return arr

    def gather(self) -> Params:
        """The whole cloud's gradients, each array in Gaussian order (a copy)."""
        return Params(*[torch.cat([getattr(P, name) for P in self.params]) for name in ("means", "scales", "quats",
                                                                                           "sh")],
                      self.params[0].sh_degree if self.params else 3)

    def allreduce_bucket(self, k: int, group=None, async_op: bool = False):
        """Sums bucket k over the ranks of `group`; with async_op, the work handle (or None alone)."""
        if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
            return dist.all_reduce(self.slices[k], op=dist.ReduceOp.SUM, group=group, async_op=async_op)
        return None
