"""Image error of the batched mixed-precision path against the FP64 oracle.

The FP64 oracle (oracle/oracle_f64.cpp) renders the same stored parameters:
the SH as the mixed layout holds them (BF16 DC and band 1, FP8 e4m3 bands 2-3
times a per-Gaussian scale), dequantised to FP32, then taken to double. So the
error below is the arithmetic's: the fast exponential, FMA contraction, FP32
accumulation and the factored conic. It is the largest absolute difference over
r g b a of every sampled pixel whose FP64 walk takes no decision near its
threshold, where a rounding can move a whole splat in or out of the pixel: the
cutoff, alpha = 1/255 and 0.99 within a relative 1e-4 (a footprint's FP32
centre is a rounding of a pixel coordinate, up to 1.2e-4 px at x = 1920,
which moves its power at the cutoff by up to about 1e-4 relative); the stop at
T = 1e-4 within a relative 1e-3 (T is a product of as many FP32 factors as
the walk blends). The blend order is not an arithmetic result but the method's
choice: both orders follow the FP32 depth key, as the reference computes it. PSNR (peak 1)
is over all sampled pixels, near decisions included. What the quantisation
itself does to the image (FP64 of the FP32 coefficients against FP64 of the
stored ones) is printed beside it.
"""
import math

import numpy as np
import pytest
import torch

import athenea_b200 as A
from athenea_b200 import scenes

pytestmark = pytest.mark.gpu

TOLERANCE = 1e-4   # max-abs against FP64, pixels clear of a decision
MARGIN = 1e-4      # the relative window of a decision

# name: (Gaussians, clustered, seed, view sizes, tile stride of the FP64 sample)
CASES = {
    "uniform-100k-960x540": (100_000, False, 20261203 + 0, [(960, 540)], 2),
    "clustered-1.5M-1920x1080": (1_500_000, True, 20261203 + 1, [(1920, 1080)] * 2, 23),
    "clustered-500k-mixed-5-views": (500_000, True, 20261203 + 3,
                                     [(320, 180), (640, 360), (960, 540), (1280, 720), (1920, 1080)], 5),
}


def _gpu_params(p):
    return A.Params(*[torch.from_numpy(np.ascontiguousarray(p[k])).cuda() for k in ("means", "scales", "quats", "sh")],
                    p["sh_degree"])


def _views(sizes, eye_at=None):
    out = []
    for v, (W, H) in enumerate(sizes):
        eye = eye_at if eye_at is not None else scenes.circle_eye(v, max(len(sizes), 1) * 4, 3.0, 0.3)
        cam = A.pinhole_for_vertical_fov(eye, (0, 0, 0), W, H, 60.0)
        out.append((cam.projection_for(W, H), W, H))
    return out


def _batched_images(M, views):
    b = A.BatchTrainer()
    b.set_views(views)
    colour = torch.empty((b.pixels, 4), device="cuda")
    target = torch.zeros((b.pixels, 3), device="cuda")
    loss = torch.zeros(1, device="cuda")
    n = M.count
    grads = A.Params(torch.zeros((n, 4), device="cuda"), torch.zeros((n, 4), device="cuda"),
                     torch.zeros((n, 4), device="cuda"), torch.zeros((n, 48), device="cuda"), 3)
    b.step(M, target, colour, loss, grads)
    stats = b.check()
    torch.cuda.synchronize()
    img = colour.cpu().numpy()
    out, base = [], 0
    for _, W, H in views:
        out.append(img[base:base + W * H])
        base += W * H
    return out, stats


def _plain_image(P, proj, W, H):
    raster = A.TileRasterizer.create()
    t = A.RenderTargets.make(W, H)
    raster.render_params(proj, P, A.RenderSettings(width=W, height=H), t)
    torch.cuda.synchronize()
    return t.colour.cpu().numpy()


def _f64(O, proj, W, H, p, sh, stride, offset):
    from tests import gpu_helpers as G
    f64 = O.frame64(G.oracle_projection(O, proj), np.eye(4), W, H, rest_per_colour=15, sh_words=23)
    return O.render_params_sampled_f64(f64, p["means"], p["scales"], p["quats"], sh, p["sh_degree"], margin=MARGIN,
                                       tile_stride=stride, tile_offset=offset)


def _errors(img, ref):
    sampled = ~np.isnan(ref["colour"][:, 0])
    clear = sampled & (ref["near"] == 0)
    diff = np.abs(img.astype(np.float64) - ref["colour"])
    mse = float(np.mean(diff[sampled] ** 2))
    worst = np.where(clear)[0][np.argmax(diff[clear].max(axis=1))]
    return dict(max_abs=float(diff[clear].max()), psnr=10 * math.log10(1.0 / max(mse, 1e-30)),
                sampled=int(sampled.sum()), near=float(1.0 - clear.sum() / max(sampled.sum(), 1)),
                worst_pixel=int(worst), worst_fp64_T=float(1.0 - ref["colour"][worst, 3]))


@pytest.mark.parametrize("name", list(CASES))
def test_mixed_precision_image_error_against_fp64(oracle, name):
    count, clustered, seed, sizes, stride = CASES[name]
    p = scenes.params(count, clustered, seed, 3)
    P = _gpu_params(p)
    M = A.MixedParams.from_params(P)
    stored_sh = M.dequantized_sh().cpu().numpy()
    views = _views(sizes)
    images, stats = _batched_images(M, views)
    for v, ((proj, W, H), img) in enumerate(zip(views, images)):
        ref = _f64(oracle, proj, W, H, p, stored_sh, stride, v % stride)
        e = _errors(img, ref)
        full = _f64(oracle, proj, W, H, p, p["sh"], stride, v % stride)
        q = _errors(ref["colour"], full)
        print(f"{name} view {v} {W}x{H}: max-abs {e['max_abs']:.3g} (pixels clear of a decision), "
              f"PSNR {e['psnr']:.1f} dB over {e['sampled']} sampled pixels ({100 * e['near']:.3f}% near a decision); "
              f"quantisation alone: PSNR {q['psnr']:.1f} dB, max-abs {q['max_abs']:.3g}")
        assert e["max_abs"] <= TOLERANCE, (name, v, e)
        assert e["near"] < 0.03, (name, v, e)
    assert stats["degenerate"] == 0   # these scenes hold no near-degenerate footprint


def _needles(base_count=20_000, seed=11):
    """A clustered cloud plus long thin needles across the view of a camera at
    (0, 0, 3): 1.5 long, 2e-4 thick, 0.7 in front of it, turned about the view
    axis so that their screen covariance is far from diagonal."""
    p = scenes.params(base_count, True, seed, 3)
    angles = [30.0, 45.0, 60.0, 100.0, 135.0, 160.0]
    k = len(angles)
    means = np.zeros((k, 4), np.float32)
    scales = np.zeros((k, 4), np.float32)
    quats = np.zeros((k, 4), np.float32)
    rng = np.random.default_rng(seed)
    sh = (rng.normal(0.0, 0.3, size=(k, 48))).astype(np.float32)
    sh[:, :3] += 0.5
    for j, a in enumerate(angles):
        means[j] = (0.08 * (j - 2.5), 0.05 * ((j % 3) - 1), 2.3, 0.5)
        scales[j] = (math.log(1.5), math.log(2e-4), math.log(2e-4), 0.0)
        h = math.radians(a) / 2
        quats[j] = (math.cos(h), 0.0, 0.0, math.sin(h))
    for key, extra in (("means", means), ("scales", scales), ("quats", quats), ("sh", sh)):
        p[key] = np.ascontiguousarray(np.concatenate([p[key], extra]))
    return p, k


def test_near_degenerate_footprints_take_fp64_and_stay_within_tolerance(oracle):
    p, needles = _needles()
    P = _gpu_params(p)
    M = A.MixedParams.from_params(P)
    stored_sh = M.dequantized_sh().cpu().numpy()
    W, H = 960, 540
    views = _views([(W, H)], eye_at=(0.0, 0.0, 3.0))
    images, stats = _batched_images(M, views)
    assert stats["degenerate"] >= needles, stats
    ref = _f64(oracle, views[0][0], W, H, p, stored_sh, 1, 0)
    e = _errors(images[0], ref)
    Pq = A.Params(P.means, P.scales, P.quats, M.dequantized_sh().contiguous(), 3)
    plain = _errors(_plain_image(Pq, views[0][0], W, H), ref)
    print(f"needles: {stats['degenerate']} FP64 footprints; mixed path max-abs {e['max_abs']:.3g}, "
          f"PSNR {e['psnr']:.1f} dB; plain FP32 path on the same footprints: max-abs {plain['max_abs']:.3g}, "
          f"PSNR {plain['psnr']:.1f} dB")
    assert e["max_abs"] <= TOLERANCE, e
    assert e["near"] < 0.05, e


def test_50m_gaussians_at_4k_against_fp64(oracle):
    """The precision-at-scale workload: 50M clustered Gaussians, a 3840x2160
    view (pairs take the wide key form: 26 Gaussian bits + 24 + 15 tile bits),
    every 97th tile checked against FP64."""
    count, W, H, stride = 50_000_000, 3840, 2160, 97
    p = scenes.params(count, True, 20261203 + 4, 3)
    P = _gpu_params(p)
    M = A.MixedParams.from_params(P)
    stored_sh = M.dequantized_sh().cpu().numpy()
    P.sh = None   # the mixed layout holds the SH now; free the FP32 copy
    torch.cuda.empty_cache()
    views = _views([(W, H)])
    images, stats = _batched_images(M, views)
    assert stats["degenerate"] == 0
    ref = _f64(oracle, views[0][0], W, H, p, stored_sh, stride, 0)
    e = _errors(images[0], ref)
    print(f"50M at 3840x2160: {stats['pairs']} pairs; max-abs {e['max_abs']:.3g} (pixels clear of a decision), "
          f"PSNR {e['psnr']:.1f} dB over {e['sampled']} sampled pixels ({100 * e['near']:.3f}% near a decision)")
    assert e["max_abs"] <= TOLERANCE, e
    assert e["near"] < 0.05, e
