"""The blend's contribution hooks (TileRasterizer.h:351-371, splat_blend.slang:
364-407) on a B200, against the CPU restatement: mode 1 (each splat's summed
weight in 1/4096), mode 2 (the squared colour change taking it away would
leave, in 2^-24, a 64-bit sum a slot), mode 3 (a mask lifted to the splats, in
1/1024) and mode 4 (each splat's colour gradient in 1/256 with the
hash-dithered rounding, and its weight) are integer sums of the same FP32
weights, so they must match word for word; frames add into the buffer."""
import numpy as np
import pytest
import torch

import athenea_b200 as A
from tests.fixtures import random_cloud

pytestmark = pytest.mark.gpu


def _frame(oracle, W=250, H=190, **settings):
    from tests import gpu_helpers as G
    from tests.test_gpu_parity import _decode
    packed = _decode(oracle, random_cloud(3000, 7))
    cam = A.Camera.looking_at((1.5, 1.0, 6.0), (0, 0, 0))
    cam.lens.focal = 30.0
    proj = cam.projection_for(W, H)
    splats = G.upload(packed)
    want = oracle.render([(packed[0], packed[1], packed[2], packed[3], packed[4], np.eye(4), 0)],
                         G.oracle_projection(oracle, proj), W, H, **settings)
    return proj, splats, want


def test_mode_1_weights_are_the_references(oracle):
    W, H = 250, 190
    proj, splats, want = _frame(oracle, W, H)
    words = torch.zeros(splats.count, dtype=torch.int32, device="cuda")
    raster = A.TileRasterizer.create()
    t = A.RenderTargets.make(W, H)
    s = A.RenderSettings(width=W, height=H, contribution_mode=1, contribution=words)
    raster.render(proj, [A.SplatInstance(splats)], s, t)
    raster.render(proj, [A.SplatInstance(splats)], s, t)   # frames add in
    torch.cuda.synchronize()
    ref = oracle.contribution_weight(want["frame"], want["binned"], want["proj"]).astype(np.uint64)
    got = words.cpu().numpy().view(np.uint32).astype(np.uint64)
    np.testing.assert_array_equal(got, 2 * ref)
    assert ref.sum() > 0


def test_mode_4_colour_gradients_are_the_references(oracle):
    W, H = 250, 190
    proj, splats, want = _frame(oracle, W, H)
    dl = torch.randn((W * H, 4), generator=torch.Generator().manual_seed(9)) * 1e-3
    words = torch.zeros((splats.count, 4), dtype=torch.int32, device="cuda")
    raster = A.TileRasterizer.create()
    t = A.RenderTargets.make(W, H)
    s = A.RenderSettings(width=W, height=H, contribution_mode=4, contribution=words, final_colour=dl.cuda())
    raster.render(proj, [A.SplatInstance(splats)], s, t)
    torch.cuda.synchronize()
    ref = oracle.colour_gradient(want["frame"], want["binned"], want["proj"], dl.numpy())
    np.testing.assert_array_equal(words.cpu().numpy(), ref)
    assert np.abs(ref[:, :3]).sum() > 0


def test_mode_2_squared_changes_are_the_references(oracle):
    """Mode 2: each splat's squared colour change against the frame drawn whole,
    a 64-bit sum in two words a slot (low, high); two frames add in."""
    W, H = 250, 190
    proj, splats, want = _frame(oracle, W, H)
    raster = A.TileRasterizer.create()
    t = A.RenderTargets.make(W, H)
    raster.render(proj, [A.SplatInstance(splats)], A.RenderSettings(width=W, height=H), t)
    whole = t.colour.clone()
    words = torch.zeros((splats.count, 2), dtype=torch.int32, device="cuda")
    s = A.RenderSettings(width=W, height=H, contribution_mode=2, contribution=words, final_colour=whole)
    raster.render(proj, [A.SplatInstance(splats)], s, t)
    raster.render(proj, [A.SplatInstance(splats)], s, t)
    torch.cuda.synchronize()
    ref = oracle.contribution_change(want["frame"], want["binned"], want["proj"], whole.cpu().numpy())
    w = words.cpu().numpy().view(np.uint32).astype(np.uint64)
    r = ref.astype(np.uint64)
    np.testing.assert_array_equal(w[:, 0] + (w[:, 1] << np.uint64(32)), 2 * (r[:, 0] + (r[:, 1] << np.uint64(32))))
    assert r[:, 0].sum() > 0


def test_mode_3_lifted_mask_is_the_references(oracle):
    """Mode 3: each splat's weight times the mask (clamped to [0, 1]) and its
    weight, in 1/1024, two words a slot."""
    W, H = 250, 190
    proj, splats, want = _frame(oracle, W, H)
    mask = torch.rand((W * H,), generator=torch.Generator().manual_seed(11)) * 1.4 - 0.2
    words = torch.zeros((splats.count, 2), dtype=torch.int32, device="cuda")
    raster = A.TileRasterizer.create()
    t = A.RenderTargets.make(W, H)
    s = A.RenderSettings(width=W, height=H, contribution_mode=3, contribution=words, lift_mask=mask.cuda())
    raster.render(proj, [A.SplatInstance(splats)], s, t)
    torch.cuda.synchronize()
    ref = oracle.contribution_lift(want["frame"], want["binned"], want["proj"], mask.numpy())
    np.testing.assert_array_equal(words.cpu().numpy().view(np.uint32), ref)
    assert ref[:, 1].sum() > ref[:, 0].sum() > 0


@pytest.mark.parametrize("hard", [False, True])
def test_lifted_matte_is_the_references(oracle, hard):
    """A mask lifted to the splats (contribution mode 3), then the matte the
    blend sums from those words (TileRasterizer.h:319-326): every pixel equals
    the restatement's, soft and hard (threshold 0.4)."""
    W, H = 250, 190
    proj, splats, want = _frame(oracle, W, H)
    mask = torch.zeros((H, W))
    mask[:, :W // 2] = 1.0   # the left half is inside
    words = torch.zeros((splats.count, 2), dtype=torch.int32, device="cuda")
    raster = A.TileRasterizer.create()
    t = A.RenderTargets.make(W, H)
    raster.render(proj, [A.SplatInstance(splats)],
                  A.RenderSettings(width=W, height=H, contribution_mode=3, contribution=words,
                                   lift_mask=mask.reshape(-1).cuda()), t)
    matte = torch.full((W * H,), -1.0, device="cuda")
    raster.render(proj, [A.SplatInstance(splats)],
                  A.RenderSettings(width=W, height=H, matte_lift=words, matte=matte, matte_hard=hard,
                                   matte_threshold=0.4), t)
    torch.cuda.synchronize()
    ref = oracle.matte_lift(want["frame"], want["binned"], want["proj"], words.cpu().numpy().view(np.uint32),
                            hard, 0.4)
    np.testing.assert_array_equal(matte.cpu().numpy(), ref)
    m = ref.reshape(H, W)
    assert m[:, :W // 4].mean() > m[:, 3 * W // 4:].mean()


def test_trace_is_the_references(oracle):
    """The trace (TileRasterizer.h:282-288, splat_trace.slang): each pixel's four
    heaviest splats, their depths and weights, and the weight the list had no
    room for, word for word the restatement's; the weights and the rest sum to
    the pixel's coverage (within the halves' rounding)."""
    W, H = 250, 190
    proj, splats, want = _frame(oracle, W, H)
    tr = torch.zeros((11, W * H), dtype=torch.int32, device="cuda")
    raster = A.TileRasterizer.create()
    t = A.RenderTargets.make(W, H)
    raster.render(proj, [A.SplatInstance(splats)], A.RenderSettings(width=W, height=H, trace=tr), t)
    torch.cuda.synchronize()
    got = tr.cpu().numpy().view(np.uint32)
    ref = oracle.trace(want["frame"], want["binned"], want["proj"])
    empty = ref[0] == 0xFFFFFFFE
    np.testing.assert_array_equal(got[0], ref[0])
    np.testing.assert_array_equal(got[:, ~empty], ref[:, ~empty])
    halves = got[8:11, ~empty].astype(np.uint32)
    parts = np.concatenate([(halves & 0xFFFF).astype(np.uint16).view(np.float16)[None],
                            (halves >> 16).astype(np.uint16).view(np.float16)[None]]).astype(np.float64)
    held_and_rest = parts[0, 0] + parts[1, 0] + parts[0, 1] + parts[1, 1] + parts[0, 2]
    coverage = t.colour.cpu().numpy()[~empty, 3].astype(np.float64)
    assert np.abs(held_and_rest - coverage).max() <= 4e-3
    assert (~empty).sum() > 1000


def test_contribution_modes_need_their_inputs(oracle):
    """Modes 0 to 4 only; mode 2 needs the whole frame and mode 3 its mask."""
    W, H = 64, 48
    proj, splats, _ = _frame(oracle, W, H)
    words = torch.zeros((splats.count, 4), dtype=torch.int32, device="cuda")
    raster = A.TileRasterizer.create()
    t = A.RenderTargets.make(W, H)
    for mode, code in ((5, 4), (2, 3), (3, 3)):
        with pytest.raises(A.AtheneaError) as e:
            raster.render(proj, [A.SplatInstance(splats)],
                          A.RenderSettings(width=W, height=H, contribution_mode=mode, contribution=words), t)
        assert e.value.code == code, mode


def test_composite_over_an_under_layer_is_the_references(oracle):
    """TileRasterizer::render's `under` (splat_blend.slang's composite path): the
    walk stops at the layer, which takes the rest of the pixel; a pixel whose
    layer depth is 0 has nothing under it."""
    W, H = 250, 190
    gen = torch.Generator().manual_seed(21)
    under = A.RenderTargets.make(W, H)
    under.colour.copy_(torch.rand((W * H, 4), generator=gen).cuda())
    depth = 5.0 + torch.rand(W * H, generator=gen) * 3.0   # the cloud spans about 5 to 7.5 from this camera
    depth[torch.rand(W * H, generator=gen) < 0.2] = 0.0
    under.depth.copy_(depth.cuda())
    for mode in (0, 1):
        proj, splats, want = _frame(oracle, W, H, depth_mode=mode)
        raster = A.TileRasterizer.create()
        t = A.RenderTargets.make(W, H)
        raster.render(proj, [A.SplatInstance(splats)], A.RenderSettings(width=W, height=H, depth_mode=mode), t,
                      under=under)
        torch.cuda.synchronize()
        ref = oracle.blend_over(want["frame"], want["binned"], want["proj"], under.colour.cpu().numpy(),
                                depth.numpy())
        assert np.abs(t.colour.cpu().numpy() - ref["colour"]).max() <= 1e-5, mode
        assert np.abs(t.depth.cpu().numpy() - ref["depth"]).max() <= 1e-4, mode
        # the layer shows where it is nearer than the splats
        assert np.abs(t.colour.cpu().numpy() - want["colour"]).max() > 0.1
    with pytest.raises(A.AtheneaError) as e:
        A.TileRasterizer.create().render(proj, [A.SplatInstance(splats)], A.RenderSettings(width=W, height=H),
                                         A.RenderTargets.make(W, H), under=A.RenderTargets.make(W - 1, H))
    assert e.value.code == 3


def test_cryptomatte_layers_are_the_references(oracle):
    """The matte path (splat_blend.slang:88-143,420-421,525-534): 6 ids a pixel by
    summed weight, alone and over an under layer with ids of its own."""
    W, H = 250, 190
    proj, splats, want = _frame(oracle, W, H)
    rng = np.random.default_rng(5)
    ids = rng.integers(0, 40, size=splats.count).astype(np.uint32)   # few ids, so they share pixels; 0 names nothing
    gen = torch.Generator().manual_seed(8)
    under = A.RenderTargets.make(W, H)
    under.colour.copy_(torch.rand((W * H, 4), generator=gen).cuda())
    depth = 5.0 + torch.rand(W * H, generator=gen) * 3.0
    depth[torch.rand(W * H, generator=gen) < 0.3] = 0.0
    under.depth.copy_(depth.cuda())
    under_ids = rng.integers(1, 1000, size=W * H).astype(np.uint32)
    for with_under in (False, True):
        crypto = torch.zeros((3, W * H, 4), dtype=torch.float32, device="cuda")
        s = A.RenderSettings(width=W, height=H, crypto_ids=torch.from_numpy(ids.view(np.int32)).cuda(), crypto=crypto,
                             under_crypto=torch.from_numpy(under_ids.view(np.int32)).cuda())
        t = A.RenderTargets.make(W, H)
        A.TileRasterizer.create().render(proj, [A.SplatInstance(splats)], s, t,
                                         under=under if with_under else None)
        torch.cuda.synchronize()
        ref = oracle.blend_matte(want["frame"], want["binned"], want["proj"], ids,
                                 depth.numpy() if with_under else None, under_ids if with_under else None)
        got = crypto.cpu().numpy()
        np.testing.assert_array_equal(got.view(np.uint32), ref.view(np.uint32))
        assert (got[0, :, 1] > 0).mean() > 0.3
