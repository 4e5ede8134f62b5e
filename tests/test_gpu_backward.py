"""The differentiable path through the C ABI (ath_raster_render_params /
ath_raster_backward), on a B200.

- the forward from FP32 training parameters matches the CPU restatement bit for bit;
- the colour part of the per-record gradient equals the reference's own
  gradient (splat_blend.slang:381-398, contributionMode 4: the sum over pixels of
  weight * dL/dpixel), unquantised, and its quantised form;
- dL/dparameters match FP64 central finite differences (eps = 1e-3) with the
  blend's decisions frozen at the base parameters;
- a torch.autograd.Function built on the pair (test harness only) gives the
  same gradients as the fused loss kernel.
"""
import numpy as np
import pytest
import torch

import athenea_b200 as A
from athenea_b200 import scenes

pytestmark = pytest.mark.gpu

GROUPS = {"means": slice(0, 3), "logit": slice(3, 4), "log_scales": slice(4, 7), "quats": slice(7, 11),
          "sh_dc": slice(11, 14), "sh_rest": slice(14, 59)}


def _params_gpu(p: dict) -> A.Params:
    t = {k: torch.from_numpy(np.ascontiguousarray(p[k])).cuda() for k in ("means", "scales", "quats", "sh")}
    return A.Params(t["means"], t["scales"], t["quats"], t["sh"], p["sh_degree"])


def _frame(W, H, eye=(0.0, 0.0, 3.0)):
    cam = A.pinhole_for_vertical_fov(eye, (0, 0, 0), W, H, 60.0)
    return cam.projection_for(W, H)


def _step(raster, proj, P: A.Params, W, H, target: torch.Tensor):
    s = A.RenderSettings(width=W, height=H)
    t = A.RenderTargets.make(W, H)
    stats = raster.render_params(proj, P, s, t)
    dl = torch.empty_like(t.colour)
    loss = torch.zeros(1, device="cuda")
    A.l2_loss(t.colour, target, dl, loss)
    grads = P.zeros_like()
    raster.backward(dl, grads)
    torch.cuda.synchronize()
    return stats, t, dl, loss, grads


def _grad_rows(grads: A.Params, which) -> np.ndarray:
    m = grads.means.cpu().numpy()[which]
    s = grads.scales.cpu().numpy()[which]
    q = grads.quats.cpu().numpy()[which]
    sh = grads.sh.cpu().numpy()[which]
    return np.concatenate([m[:, :3], m[:, 3:4], s[:, :3], q, sh], axis=1).astype(np.float64)


def _fd(O, proj, p, W, H, target, which, eps):
    from tests import gpu_helpers as G
    op = G.oracle_projection(O, proj)
    f64 = O.frame64(op, np.eye(4), W, H, rest_per_colour=15, sh_words=23)
    means = p["means"][:, :3].astype(np.float64)
    fd, loss = O.fd_gradients_f64(f64, means, p["scales"][:, :3].astype(np.float64), p["quats"].astype(np.float64),
                                  p["means"][:, 3].astype(np.float64), p["sh"].astype(np.float64), p["sh_degree"],
                                  target, which, eps)
    return fd, loss


# cos, median and 95th percentile of the relative error against FP64 central differences
# (Richardson-combined), for every parameter group; the C2 workload reaches cos 1.0 and
# p95 of a few 1e-5, so these leave a decade
COS_MIN, MEDIAN_MAX, P95_MAX = 0.9999, 1e-4, 1e-3


def _check_groups(ours, fd, label):
    report = {}
    for name, sl in GROUPS.items():
        a, b = ours[:, sl].ravel(), fd[:, sl].ravel()
        scale = np.sqrt(np.mean(b * b)) + 1e-30
        err = np.abs(a - b) / (np.abs(b) + 0.05 * scale)
        cos = float(np.dot(a, b) / (np.linalg.norm(a) * np.linalg.norm(b) + 1e-30))
        report[name] = (cos, float(np.median(err)), float(np.percentile(err, 95)))
    print(label, {k: (round(r[0], 7), float(f"{r[1]:.3g}"), float(f"{r[2]:.3g}")) for k, r in report.items()})
    for name, (cos, med, p95) in report.items():
        assert cos > COS_MIN, (label, name, report[name])
        assert med < MEDIAN_MAX, (label, name, report[name])
        assert p95 < P95_MAX, (label, name, report[name])
    return report


@pytest.fixture(scope="module")
def raster(native):
    return A.TileRasterizer.create()


def test_params_forward_matches_the_restatement(oracle, raster):
    from tests import gpu_helpers as G
    p = scenes.params(20_000, True, 4242, 3)
    W, H = 320, 240
    proj = _frame(W, H)
    P = _params_gpu(p)
    t = A.RenderTargets.make(W, H)
    stats = raster.render_params(proj, P, A.RenderSettings(width=W, height=H), t)
    torch.cuda.synchronize()
    got = G.frame_buffers(raster)
    op = G.oracle_projection(oracle, proj)
    f = oracle.frame_for(op, np.eye(4), W, H, rest_per_colour=15, sh_words=23)
    pr = oracle.project_params(f, p["means"], p["scales"], p["quats"], p["sh"], p["sh"].shape[1])
    binned = oracle.bin_(f, pr)
    want = oracle.blend(f, binned, pr)
    np.testing.assert_array_equal(got["keys"], pr["keys"])
    kept = pr["visible"] != 0
    np.testing.assert_array_equal(got["records"][kept].view(np.uint32), pr["records"][kept].view(np.uint32))
    assert stats.pairs == binned["pairs"]
    np.testing.assert_array_equal(got["pair_splats"], binned["pair_splats"])
    np.testing.assert_array_equal(got["ranges"].reshape(-1), binned["ranges"])
    assert np.abs(t.colour.cpu().numpy() - want["colour"]).max() <= 1e-5


def test_colour_gradient_is_the_references(oracle, raster):
    """contributionMode 4's sums (splat_blend.slang:381-398), exact and quantised."""
    from tests import gpu_helpers as G
    p = scenes.params(20_000, True, 77, 3)
    W, H = 320, 240
    proj = _frame(W, H)
    target = torch.rand((W * H, 3), generator=torch.Generator().manual_seed(5)).cuda()
    _, t, dl, _, _ = _step(raster, proj, _params_gpu(p), W, H, target)
    fb = G.frame_buffers(raster)
    import ctypes as C
    from athenea_b200 import _native as N
    b = N.FrameBuffers()
    N.check(N.lib().ath_raster_frame_buffers(raster._h, C.byref(b)))
    grads10 = G.fetch(b.grads, (fb["slots"], 10), np.float32)
    op = G.oracle_projection(oracle, proj)
    f = oracle.frame_for(op, np.eye(4), W, H, rest_per_colour=15, sh_words=23)
    pr = oracle.project_params(f, p["means"], p["scales"], p["quats"], p["sh"], p["sh"].shape[1])
    binned = oracle.bin_(f, pr)
    dln = dl.cpu().numpy()
    exact = oracle.colour_gradient_exact(f, binned, pr, dln)
    ours = grads10[:, 6:9].astype(np.float64)
    scale = np.abs(exact).max()
    assert np.abs(ours - exact).max() <= 1e-4 * scale
    # The quantised form, at the per-pixel scale it is made for (a derivative of
    # order one a pixel: the sum of squares, not its mean): hash-dithered rounding
    # to 1/256 is unbiased, so the sums agree to about sqrt(pixels)/256.
    big = dln * (3.0 * W * H)
    quant = oracle.colour_gradient(f, binned, pr, big)[:, :3] / 256.0
    exact_big = oracle.colour_gradient_exact(f, binned, pr, big)
    live = np.abs(exact_big) > 0
    assert np.corrcoef(quant[live], exact_big[live])[0, 1] > 0.99
    assert np.abs(quant - exact_big).mean() < 0.1


def test_gradients_match_fp64_finite_differences(oracle, raster):
    p = scenes.params(4_000, True, 11, 3)
    W, H = 192, 144
    proj = _frame(W, H)
    rng = np.random.default_rng(3)
    target_np = rng.uniform(0, 1, size=(W * H, 3)).astype(np.float32)
    target = torch.from_numpy(target_np).cuda()
    _, _, _, loss, grads = _step(raster, proj, _params_gpu(p), W, H, target)
    from tests import gpu_helpers as G
    keys = G.frame_buffers(raster)["keys"]
    visible = np.nonzero(keys < 0xFF000000)[0]
    which = np.sort(rng.choice(visible, size=min(48, visible.size), replace=False)).astype(np.uint32)
    fd1, l64 = _fd(oracle, proj, p, W, H, target_np, which, 1e-3)
    fd2, _ = _fd(oracle, proj, p, W, H, target_np, which, 5e-4)
    fd = (4.0 * fd2 - fd1) / 3.0   # Richardson: the O(eps^2) term cancels
    assert abs(float(loss.item()) - l64) <= 1e-4 * l64
    _check_groups(_grad_rows(grads, which), fd, "small")


def test_c2_gradients_match_fp64_finite_differences(oracle, raster):
    """The differentiation workload itself: 500k clustered Gaussians at 1280x720, target uniform in
    [0,1]^3, 256 random Gaussians, eps = 1e-3 (and 5e-4, combined by Richardson)."""
    p = scenes.params(500_000, True, scenes.SEED + 2, 3)
    W, H = 1280, 720
    proj = _frame(W, H)
    rng = np.random.default_rng(scenes.SEED + 2)
    target_np = rng.uniform(0, 1, size=(W * H, 3)).astype(np.float32)
    target = torch.from_numpy(target_np).cuda()
    _, _, _, loss, grads = _step(raster, proj, _params_gpu(p), W, H, target)
    from tests import gpu_helpers as G
    keys = G.frame_buffers(raster)["keys"]
    visible = np.nonzero(keys < 0xFF000000)[0]
    which = np.sort(rng.choice(visible, size=256, replace=False)).astype(np.uint32)
    fd1, l64 = _fd(oracle, proj, p, W, H, target_np, which, 1e-3)
    fd2, _ = _fd(oracle, proj, p, W, H, target_np, which, 5e-4)
    assert abs(float(loss.item()) - l64) <= 1e-4 * l64
    _check_groups(_grad_rows(grads, which), (4.0 * fd2 - fd1) / 3.0, "c2")


class _Raster(torch.autograd.Function):
    """The forward/backward pair as an autograd function (test harness only)."""

    @staticmethod
    def forward(ctx, means, scales, quats, sh, raster, proj, W, H):
        P = A.Params(means.detach().contiguous(), scales.detach().contiguous(), quats.detach().contiguous(),
                     sh.detach().contiguous(), 3)
        t = A.RenderTargets.make(W, H)
        raster.render_params(proj, P, A.RenderSettings(width=W, height=H), t)
        ctx.raster, ctx.P = raster, P
        return t.colour

    @staticmethod
    def backward(ctx, dl_dcolour):
        g = ctx.P.zeros_like()
        ctx.raster.backward(dl_dcolour.contiguous(), g)
        return g.means, g.scales, g.quats, g.sh, None, None, None, None


def test_autograd_function_matches_the_fused_loss(raster):
    p = scenes.params(10_000, True, 5, 3)
    W, H = 256, 160
    proj = _frame(W, H)
    target = torch.rand((W * H, 3), generator=torch.Generator().manual_seed(9)).cuda()
    _, _, _, loss, grads = _step(raster, proj, _params_gpu(p), W, H, target)
    leaves = [torch.from_numpy(np.ascontiguousarray(p[k])).cuda().requires_grad_(True)
              for k in ("means", "scales", "quats", "sh")]
    colour = _Raster.apply(*leaves, raster, proj, W, H)
    torch_loss = ((colour[:, :3] - target) ** 2).mean()
    torch_loss.backward()
    assert abs(torch_loss.item() - loss.item()) <= 1e-5 * loss.item()
    for leaf, ours in zip(leaves, (grads.means, grads.scales, grads.quats, grads.sh)):
        a, b = leaf.grad.cpu().numpy(), ours.cpu().numpy()
        assert np.abs(a - b).max() <= 1e-4 * (np.abs(b).max() + 1e-12)
