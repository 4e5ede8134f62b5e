"""athenea-b200: athenea's Gaussian-splat tile rasteriser for B200 (sm_100a).

The kernels live in libathenea_b200.so (csrc/, built by _build.py); this
package is the Python mirror of the reference's rasteriser interface over its
C ABI (include/athenea_raster.h).
"""
from ._native import AtheneaError  # noqa: F401
from .raster import (Camera, CloudLoader, FrameStats, GpuSplats, Lens, Params, RenderSettings,  # noqa: F401
                     RenderTargets, SplatCounters, SplatEdit, SplatInstance, TileRasterizer, encoding_3dgs, l2_loss,
                     pinhole_for_vertical_fov)

__all__ = ["AtheneaError", "Camera", "CloudLoader", "FrameStats", "GpuSplats", "Lens", "Params", "l2_loss",
           "RenderSettings",
           "RenderTargets", "SplatCounters", "SplatEdit", "SplatInstance", "TileRasterizer", "encoding_3dgs",
           "pinhole_for_vertical_fov"]
