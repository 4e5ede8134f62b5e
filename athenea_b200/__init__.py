"""athenea-b200: athenea's Gaussian-splat tile rasteriser for B200 (sm_100a).

The kernels live in libathenea_b200.so (csrc/, built by _build.py); this
package is the Python mirror of the reference's rasteriser interface over its
C ABI (include/athenea_raster.h), plus the training path the reference does
not have: differentiable frames (Params, TileRasterizer.render_params /
backward) and the batched mixed-precision step (MixedParams, BatchTrainer).
"""
from ._native import AtheneaError  # noqa: F401
from .parallel import BucketedGradients, GradientBuffer, gradient_bucket, shard_views  # noqa: F401
from .raster import (BatchTrainer, Camera, CloudCounts, CloudLoader, FrameStats, GpuSplats, Lens,  # noqa: F401
                     MixedParams, Params, RenderSettings, RenderTargets, SplatCounters, SplatEdit, SplatInstance,
                     TileRasterizer, check_bounded_wait, encoding_3dgs, l2_loss, measure_peaks, memory_held,
                     pinhole_for_vertical_fov, read_splat_ply, set_memory_budget)

__all__ = ["AtheneaError", "BatchTrainer", "BucketedGradients", "GradientBuffer", "gradient_bucket", "shard_views", "Camera", "CloudCounts", "CloudLoader",
           "FrameStats", "GpuSplats", "Lens", "MixedParams", "Params", "RenderSettings", "RenderTargets",
           "SplatCounters", "SplatEdit", "SplatInstance", "TileRasterizer", "check_bounded_wait", "encoding_3dgs",
           "l2_loss", "measure_peaks", "memory_held", "pinhole_for_vertical_fov", "read_splat_ply",
           "set_memory_budget"]
