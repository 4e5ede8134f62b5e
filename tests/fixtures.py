"""Synthetic clouds for the tests, restated from the reference's
tests/render/SplatFixtures.h: records in the 3DGS encoding, so they go through
the same decode a file does.
"""
from __future__ import annotations

import math

import numpy as np

SH0 = np.float32(0.28209479)

# SplatFixtures.h:22-31: 23 floats a record, degree 1, rest colour-outer.
ENC_BUILDER = dict(stride=23, x=0, y=1, z=2, opacity=3, scale0=4, scale1=5, scale2=6, rotW=7, rotX=8, rotY=9,
                   rotZ=10, dc0=11, dc1=12, dc2=13, restBase=14, filePerColour=3)


def product_encoding(enc: dict) -> dict:
    """The oracle's field names as ath_encoding's."""
    m = dict(rotW="rot_w", rotX="rot_x", rotY="rot_y", rotZ="rot_z", restBase="rest_base",
             filePerColour="file_per_colour")
    return {m.get(k, k): v for k, v in enc.items()}


class CloudBuilder:
    """SplatFixtures.h:20-50."""

    def __init__(self):
        self.rows = []

    def add(self, x, y, z, opacity, sx, sy, sz, wxyz, colour, rest=(0.0,) * 9):
        f = np.float32
        logit = np.log(f(opacity) / (f(1.0) - f(opacity)))
        r = [f(x), f(y), f(z), logit, np.log(f(sx)), np.log(f(sy)), np.log(f(sz)), f(wxyz[0]), f(wxyz[1]),
             f(wxyz[2]), f(wxyz[3]), (f(colour[0]) - f(0.5)) / SH0, (f(colour[1]) - f(0.5)) / SH0,
             (f(colour[2]) - f(0.5)) / SH0] + [f(v) for v in rest]
        self.rows.append(np.array(r, np.float32))
        return self

    def records(self) -> np.ndarray:
        return np.stack(self.rows).astype(np.float32) if self.rows else np.zeros((0, 23), np.float32)


class Lcg:
    """SplatFixtures.h:87-95."""

    def __init__(self, seed: int = 0):
        self.state = 0x853C49E6748FEA9B ^ seed

    def next(self) -> np.float32:
        self.state = (self.state * 6364136223846793005 + 1442695040888963407) & 0xFFFFFFFFFFFFFFFF
        return np.float32(((self.state >> 40) & 0xFFFFFF) / 16777216.0)

    def range(self, lo, hi) -> np.float32:
        lo, hi = np.float32(lo), np.float32(hi)
        return lo + (hi - lo) * self.next()


def random_cloud(count: int, seed: int, min_size=0.004, max_size=0.6, min_opacity=0.02, max_opacity=0.99):
    """SplatFixtures.h:97-128, draws in the same order."""
    b = CloudBuilder()
    rng = Lcg(seed)
    for _ in range(count):
        size = np.exp(rng.range(np.log(np.float32(min_size)), np.log(np.float32(max_size))))
        stretch = rng.range(0.05, 1.0)
        rest = [rng.range(-0.3, 0.3) for _ in range(9)]
        x = rng.range(-2.0, 2.0)
        y = rng.range(-1.5, 1.5)
        z = rng.range(-2.0, 2.0)
        opacity = rng.range(min_opacity, max_opacity)
        thin = rng.range(0.1, 1.0)
        turn = [rng.range(-1, 1) for _ in range(4)]
        dc = [rng.range(0.0, 1.2) for _ in range(3)]
        b.add(x, y, z, opacity, size, size * stretch, size * thin, turn, dc, rest)
    return b


def linear_to_srgb_code(c: np.ndarray) -> np.ndarray:
    """common/color.slang:20-23 then an 8-bit code (image_compare's measure)."""
    c = np.maximum(np.asarray(c, np.float64), 0.0)
    s = np.where(c <= 0.0031308, c * 12.92, 1.055 * np.power(c, 1.0 / 2.4) - 0.055)
    return np.clip(np.round(s * 255.0), 0, 255).astype(np.int32)


def look_at_rows(eye, target, up=(0.0, 1.0, 0.0)) -> np.ndarray:
    e, t, u = (np.asarray(v, np.float64) for v in (eye, target, up))
    z = e - t
    z /= np.linalg.norm(z)
    x = np.cross(u, z)
    x /= np.linalg.norm(x)
    y = np.cross(z, x)
    m = np.eye(4)
    m[:3, 0], m[:3, 1], m[:3, 2], m[:3, 3] = x, y, z, e
    return m


def rotation_y(degrees: float) -> np.ndarray:
    t = math.radians(degrees)
    m = np.eye(4)
    m[0, 0], m[0, 2], m[2, 0], m[2, 2] = math.cos(t), math.sin(t), -math.sin(t), math.cos(t)
    return m


def translation(v) -> np.ndarray:
    m = np.eye(4)
    m[:3, 3] = v
    return m


def scaling(v) -> np.ndarray:
    return np.diag([v[0], v[1], v[2], 1.0])
