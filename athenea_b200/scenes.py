"""Seeded synthetic scenes with the shapes and distributions of the workloads
this rasteriser is measured on. No dataset is read: the captures the
reference's own numbers were taken on are not available, so these stand in.

Every scene is written as 3DGS records (x y z, normal, f_dc, f_rest colour-outer,
logit opacity, log scales, wxyz rotation) and goes through the same decode a
PLY does, so the packed values are quantised exactly as an upload quantises them.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .raster import encoding_3dgs

SEED = 20261203


@dataclass(frozen=True)
class Workload:
    """One workload: a scene and the views it is drawn from."""
    name: str
    count: int
    width: int
    height: int
    clustered: bool
    views: int = 1
    vfov: float = 60.0


# The five measured workloads: 0 a plain frame of 100k at 960x540 with uniform
# means; 1 a plain frame of 1.5M at 1920x1080, clustered; 2 differentiation,
# 500k at 1280x720; 3 64 views of mixed size of 2.36M; 4 50M, 8 views at 4K.
WORKLOADS = {
    0: Workload("uniform-100k-960x540", 100_000, 960, 540, False),
    1: Workload("clustered-1.5M-1920x1080", 1_500_000, 1920, 1080, True),
    2: Workload("clustered-500k-1280x720", 500_000, 1280, 720, True),
    3: Workload("clustered-2.36M-64views-mixed", 2_360_000, 1920, 1080, True, views=64),
    4: Workload("clustered-50M-8views-3840x2160", 50_000_000, 3840, 2160, True, views=8),
}

MIXED_RESOLUTIONS = ((320, 180), (640, 360), (960, 540), (1280, 720), (1920, 1080))


def gaussians(count: int, clustered: bool, seed: int, sh_degree: int = 3) -> dict:
    """`count` Gaussians: means uniform in [-1,1]^3, or from a mixture of 8
    isotropic normals (sigma 0.3) centred uniformly in [-1,1]^3; log-scales
    N(-4.5, 0.5) per axis; rotations uniform (a normalised 4D gaussian, w x y z);
    opacity logits N(0, 1) (opacity sigmoid(N(0,1))); SH of `sh_degree`, N(0, 0.3)
    with 0.5 added to the DC, rgb per basis with the DC first."""
    rng = np.random.default_rng(seed)
    rest = (0, 3, 8, 15)[sh_degree]
    if clustered:
        centres = rng.uniform(-1.0, 1.0, size=(8, 3))
        which = rng.integers(0, 8, size=count)
        means = centres[which] + rng.normal(0.0, 0.3, size=(count, 3))
    else:
        means = rng.uniform(-1.0, 1.0, size=(count, 3))
    shs = rng.normal(0.0, 0.3, size=(count, 3 + 3 * rest))
    shs[:, 0:3] += 0.5
    logits = rng.normal(0.0, 1.0, size=count)
    log_scales = rng.normal(-4.5, 0.5, size=(count, 3))
    q = rng.normal(0.0, 1.0, size=(count, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    return dict(means=means, logits=logits, log_scales=log_scales, quats=q, sh=shs, rest=rest)


def records(count: int, clustered: bool, seed: int, sh_degree: int = 3) -> tuple[np.ndarray, dict]:
    """The Gaussians of `gaussians` as 3DGS records (f_rest colour-outer, as a PLY has them)."""
    g = gaussians(count, clustered, seed, sh_degree)
    rest = g["rest"]
    enc = encoding_3dgs(rest)
    out = np.zeros((count, enc["stride"]), np.float32)
    out[:, 0:3] = g["means"]
    out[:, enc["dc0"]:enc["dc0"] + 3] = g["sh"][:, 0:3]
    if rest:
        restv = g["sh"][:, 3:].reshape(count, rest, 3)          # basis-major, rgb inner
        out[:, enc["rest_base"]:enc["rest_base"] + 3 * rest] = restv.transpose(0, 2, 1).reshape(count, 3 * rest)
    out[:, enc["opacity"]] = g["logits"]
    out[:, enc["scale0"]:enc["scale0"] + 3] = g["log_scales"]
    out[:, enc["rot_w"]:enc["rot_w"] + 4] = g["quats"]
    return out, enc


def params(count: int, clustered: bool, seed: int, sh_degree: int = 3) -> dict:
    """The Gaussians of `gaussians` in the FP32 training layout (ath_params): means (N,4) with the
    opacity logit fourth, scales (N,4) log scales, quats (N,4) w x y z, sh (N, 3 + 3 rest)."""
    g = gaussians(count, clustered, seed, sh_degree)
    means = np.zeros((count, 4), np.float32)
    means[:, :3] = g["means"]
    means[:, 3] = g["logits"]
    scales = np.zeros((count, 4), np.float32)
    scales[:, :3] = g["log_scales"]
    return dict(means=means, scales=scales, quats=g["quats"].astype(np.float32),
                sh=np.ascontiguousarray(g["sh"], np.float32), sh_degree=sh_degree)


def circle_eye(view: int, views: int, radius: float = 3.0, height: float = 0.0) -> tuple:
    """The eye of view `view` of a circular walk of `views` around the origin."""
    t = 2.0 * math.pi * view / max(views, 1)
    return (radius * math.sin(t), height, radius * math.cos(t))


def view_sizes(views: int, seed: int) -> list[tuple[int, int]]:
    """Resolutions drawn uniformly from {320x180, 640x360, 960x540, 1280x720, 1920x1080}."""
    rng = np.random.default_rng(seed + 77)
    return [MIXED_RESOLUTIONS[i] for i in rng.integers(0, len(MIXED_RESOLUTIONS), size=views)]
