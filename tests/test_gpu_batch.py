"""The batched, mixed-precision training step (ath_batch_*) against the plain
per-view path (ath_raster_render_params / ath_raster_backward), on a B200.

With the SH first quantised to the mixed layout (so both paths see the same
coefficients), the only differences left are the blend's fast exponential and
fused multiply-adds: pairs, their order and the tile ranges must be identical
to the bit, images and gradients equal within those roundings. The tile size
and record batch the autotuner picks between change no image bit.
"""
import numpy as np
import pytest
import torch

import athenea_b200 as A
from athenea_b200 import scenes
from athenea_b200.raster import BatchTrainer, MixedParams

pytestmark = pytest.mark.gpu

SIZES = [(320, 180), (640, 360), (480, 270)]


def _scene(count=50_000, seed=31, squeeze=1.0):
    p = scenes.params(count, True, seed, 3)
    p["means"][:, :3] *= squeeze
    P = A.Params(*[torch.from_numpy(np.ascontiguousarray(p[k])).cuda() for k in ("means", "scales", "quats", "sh")], 3)
    M = MixedParams.from_params(P)
    # the plain path sees the same (quantised) coefficients
    Pq = A.Params(P.means, P.scales, P.quats, M.dequantized_sh().contiguous(), 3)
    return Pq, M


def _views(n=len(SIZES)):
    out = []
    for v in range(n):
        W, H = SIZES[v % len(SIZES)]
        eye = scenes.circle_eye(v, 8, 3.0, 0.3)
        cam = A.pinhole_for_vertical_fov(eye, (0, 0, 0), W, H, 60.0)
        out.append((cam.projection_for(W, H), W, H))
    return out


def _plain(Pq, views, targets):
    from tests import gpu_helpers as G
    raster = A.TileRasterizer.create()
    grads = Pq.zeros_like()
    loss = torch.zeros(1, device="cuda")
    images, frames = [], []
    for (proj, W, H), target in zip(views, targets):
        t = A.RenderTargets.make(W, H)
        raster.render_params(proj, Pq, A.RenderSettings(width=W, height=H), t)
        dl = torch.empty_like(t.colour)
        A.l2_loss(t.colour, target, dl, loss)
        frames.append(G.frame_buffers(raster))
        raster.backward(dl, grads)
        images.append(t.colour.clone())
    torch.cuda.synchronize()
    return images, frames, loss, grads


def _batched(M, views, targets, tile=16, block_batch=256, trainer=None):
    b = trainer or BatchTrainer()
    b.set_views(views)
    b.set_tuning(tile, block_batch)
    colour = torch.empty((b.pixels, 4), device="cuda")
    target = torch.cat(targets).contiguous()
    loss = torch.zeros(1, device="cuda")
    grads = A.Params(torch.zeros_like(M.means), torch.zeros_like(M.scales), torch.zeros_like(M.quats),
                     torch.zeros((M.count, 48), device="cuda"), 3)
    b.step(M, target, colour, loss, grads)
    stats = b.check()
    torch.cuda.synchronize()
    return b, colour, loss, grads, stats


def _depth_keys(field, buf):
    """The 24-bit depth keys of packed pairs' depth fields: as they are, or with the
    renumbered exponent (depth_bits < 24) put back from exp_base."""
    if buf["depth_bits"] >= 24:
        return field
    return (((field >> np.uint64(16)) + np.uint64(buf["exp_base"])) << np.uint64(16)) | (field & np.uint64(0xFFFF))


def _same_pairs(b, frames):
    """The batched step's sorted pairs and tile ranges against the plain path's, view by view, to the bit."""
    from tests import gpu_helpers as G
    buf = b.buffers()
    assert buf["pairs"] == sum(f["pairs"] for f in frames)
    keys = G.fetch(buf["sorted_pairs"], (buf["pairs"],), np.uint64)
    ranges = G.fetch(buf["ranges"], (buf["total_tiles"], 2), np.uint32)
    tiles = (keys >> np.uint64(buf["key_shift"])).astype(np.int64)
    if buf["sorted_values"] is None:
        splats = (keys & np.uint64((1 << buf["slot_bits"]) - 1)).astype(np.uint32)
        depths = _depth_keys((keys >> np.uint64(buf["slot_bits"])) & np.uint64((1 << buf["depth_bits"]) - 1), buf)
    else:
        splats = G.fetch(buf["sorted_values"], (buf["pairs"],), np.uint32)
        depths = keys & np.uint64(0xFFFFFF)
    start = 0
    for v, f in enumerate(frames):
        n = f["pairs"]
        # this view's pairs: its tiles, its depths, its Gaussians, in its order
        np.testing.assert_array_equal(tiles[start:start + n] - buf["tile_bases"][v],
                                      (f["pair_keys"] >> np.uint64(24)).astype(np.int64))
        np.testing.assert_array_equal(depths[start:start + n], f["pair_keys"] & np.uint64(0xFFFFFF))
        np.testing.assert_array_equal(splats[start:start + n], f["pair_splats"])
        r = ranges[buf["tile_bases"][v]:buf["tile_bases"][v] + f["tiles"]].astype(np.int64)
        live = r[:, 1] > r[:, 0]
        np.testing.assert_array_equal(r[live] - start, f["ranges"].astype(np.int64)[live])
        assert np.all(r[~live, 1] == r[~live, 0])
        start += n
    return np.diff(ranges.astype(np.int64), axis=1).ravel()


def test_batched_step_matches_the_plain_path(oracle):
    from tests import gpu_helpers as G
    Pq, M = _scene()
    views = _views()
    gen = torch.Generator().manual_seed(3)
    targets = [torch.rand((W * H, 3), generator=gen).cuda() for _, W, H in views]
    images, frames, loss_p, grads_p = _plain(Pq, views, targets)
    b, colour, loss_b, grads_b, stats = _batched(M, views, targets)
    assert stats["pairs"] == sum(f["pairs"] for f in frames)
    _same_pairs(b, frames)
    # images: the fast exponential, within 1e-4 but for the odd blend decision at its threshold
    got = colour.cpu().numpy()
    base = 0
    for (proj, W, H), img in zip(views, images):
        d = np.abs(got[base:base + W * H] - img.cpu().numpy()).max(axis=1)
        assert np.mean(d <= 1e-4) >= 0.9999, float(np.mean(d <= 1e-4))
        assert d.max() <= 2e-2
        base += W * H
    assert abs(loss_b.item() - loss_p.item()) <= 1e-4 * loss_p.item()
    for name in ("means", "scales", "quats", "sh"):
        a = getattr(grads_b, name).cpu().numpy().ravel().astype(np.float64)
        c = getattr(grads_p, name).cpu().numpy().ravel().astype(np.float64)
        cos = np.dot(a, c) / (np.linalg.norm(a) * np.linalg.norm(c) + 1e-30)
        assert cos > 0.9999, (name, cos)
        assert abs(np.linalg.norm(a) / np.linalg.norm(c) - 1.0) < 1e-3, name


def test_tile_size_and_block_batch_change_no_image_bit():
    Pq, M = _scene(30_000, 8)
    views = _views()
    gen = torch.Generator().manual_seed(4)
    targets = [torch.rand((W * H, 3), generator=gen).cuda() for _, W, H in views]
    ref = None
    for tile in (8, 16, 32):
        for nb in (64, 256):
            _, colour, _, _, _ = _batched(M, views, targets, tile, nb)
            img = colour.cpu().numpy()
            if ref is None:
                ref = img
            else:
                np.testing.assert_array_equal(img, ref, err_msg=f"tile {tile}, batch {nb}")


def test_one_trainer_through_tile_and_view_changes_draws_as_fresh_ones():
    """ath_batch_set_tuning to a smaller tile (four times the tiles) and
    ath_batch_set_views with more views, after steps on the same trainer: its
    buffers grow with them, and each step draws what a new trainer draws."""
    Pq, M = _scene(30_000, 12)
    gen = torch.Generator().manual_seed(6)
    every = _views(6)
    targets = [torch.rand((W * H, 3), generator=gen).cuda() for _, W, H in every]
    b = BatchTrainer()
    for n, tile, nb in ((2, 32, 512), (2, 8, 256), (6, 16, 128), (3, 32, 64)):
        views, tg = every[:n], targets[:n]
        _, colour, _, _, stats = _batched(M, views, tg, tile, nb, trainer=b)
        _, fresh, _, _, fresh_stats = _batched(M, views, tg, tile, nb)
        np.testing.assert_array_equal(colour.cpu().numpy(), fresh.cpu().numpy(), err_msg=f"{n} views, tile {tile}")
        assert stats["pairs"] == fresh_stats["pairs"]


def test_replayed_step_draws_the_same_image_and_tune_picks_a_setting():
    Pq, M = _scene(30_000, 9)
    views = _views()
    gen = torch.Generator().manual_seed(5)
    targets = [torch.rand((W * H, 3), generator=gen).cuda() for _, W, H in views]
    b, colour, loss, grads, _ = _batched(M, views, targets)
    first = colour.cpu().numpy().copy()
    b.step(M, torch.cat(targets).contiguous(), colour, loss, grads)   # same pointers? a new target tensor: recaptured
    torch.cuda.synchronize()
    np.testing.assert_array_equal(colour.cpu().numpy(), first)
    best = b.tune(M, torch.cat(targets).contiguous(), colour, loss, grads, repeats=2)
    assert best["tile"] in (8, 16, 32) and best["block_batch"] in (64, 128, 256, 512) and best["ms_per_step"] > 0


def test_wide_pairs_sort_and_draw_as_the_packed_ones():
    """ath_batch_set_key_mode: the wide (key, Gaussian) pairs come out in the
    packed pairs' order and draw the same image; the gradients agree."""
    from tests import gpu_helpers as G
    Pq, M = _scene(40_000, 12)
    views = _views()
    gen = torch.Generator().manual_seed(6)
    targets = [torch.rand((W * H, 3), generator=gen).cuda() for _, W, H in views]
    out = {}
    for mode in (1, 2):
        b = BatchTrainer()
        b.set_key_mode(mode)
        b, colour, loss, grads, stats = _batched(M, views, targets, trainer=b)
        buf = b.buffers()
        n = buf["pairs"]
        keys = G.fetch(buf["sorted_pairs"], (n,), np.uint64)
        if mode == 1:
            assert buf["sorted_values"] is None
            gauss = (keys & np.uint64((1 << buf["slot_bits"]) - 1)).astype(np.uint32)
            tile_depth = keys >> np.uint64(buf["slot_bits"])
        else:
            assert buf["slot_bits"] == 0 and buf["key_shift"] == 24
            gauss = G.fetch(buf["sorted_values"], (n,), np.uint32)
            tile_depth = keys
        out[mode] = (tile_depth, gauss, G.fetch(buf["ranges"], (buf["total_tiles"], 2), np.uint32),
                     colour.cpu().numpy(), grads)
    np.testing.assert_array_equal(out[1][0], out[2][0])
    np.testing.assert_array_equal(out[1][1], out[2][1])
    np.testing.assert_array_equal(out[1][2], out[2][2])
    np.testing.assert_array_equal(out[1][3], out[2][3])
    for name in ("means", "scales", "quats", "sh"):
        a = getattr(out[1][4], name).cpu().numpy().ravel().astype(np.float64)
        c = getattr(out[2][4], name).cpu().numpy().ravel().astype(np.float64)
        # the record and parameter gradients are sums by float atomics, in no fixed order
        assert np.abs(a - c).max() <= 1e-5 * (np.abs(c).max() + 1e-30) + 1e-12, name


def test_renumbered_depth_pairs_sort_and_draw_as_the_plain_path():
    """Key mode 3: the packed pairs' depth field holds the depth key's exponent
    byte renumbered from the sizing's planned base. The sorted pairs and ranges
    are the plain path's to the bit, and the image is the 24-bit packed form's."""
    Pq, M = _scene(40_000, 13)
    views = _views()
    gen = torch.Generator().manual_seed(7)
    targets = [torch.rand((W * H, 3), generator=gen).cuda() for _, W, H in views]
    _, frames, _, _ = _plain(Pq, views, targets)
    b = BatchTrainer()
    b.set_key_mode(3)
    b, colour, _, _, stats = _batched(M, views, targets, trainer=b)
    buf = b.buffers()
    assert buf["depth_bits"] < 24 and buf["sorted_values"] is None
    assert buf["key_shift"] == buf["depth_bits"] + buf["slot_bits"]
    assert stats["pairs"] == sum(f["pairs"] for f in frames)
    _same_pairs(b, frames)
    b1 = BatchTrainer()
    b1.set_key_mode(1)
    _, colour1, _, _, _ = _batched(M, views, targets, trainer=b1)
    np.testing.assert_array_equal(colour.cpu().numpy(), colour1.cpu().numpy())


def test_depths_leaving_the_planned_range_are_reported_and_planned_again():
    """A renumbered depth field covers the exponents its sizing saw, two to spare
    on each side. A step whose cloud has moved eight times nearer the eye falls
    outside: ath_batch_check reports Capacity, and the next step plans again and
    draws what a new trainer draws."""
    _, M = _scene(20_000, 14)
    views = _views(1)
    gen = torch.Generator().manual_seed(8)
    targets = [torch.rand((W * H, 3), generator=gen).cuda() for _, W, H in views]
    b = BatchTrainer()
    b.set_key_mode(3)
    b, colour, loss, grads, _ = _batched(M, views, targets, trainer=b)
    planned = b.buffers()["exp_base"]
    eye = torch.tensor(scenes.circle_eye(0, 8, 3.0, 0.3), dtype=torch.float32, device="cuda")
    with torch.no_grad():
        M.means[:, :3] = eye + (M.means[:, :3] - eye) * 0.125   # in place: the same arrays
    target = torch.cat(targets).contiguous()
    b.step(M, target, colour, loss, grads)
    with pytest.raises(A.AtheneaError) as e:
        b.check()
    assert e.value.name == "Capacity"
    b.step(M, target, colour, loss, grads)
    b.check()
    assert b.buffers()["exp_base"] < planned
    _, fresh, _, _, _ = _batched(M, views, targets)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(colour.cpu().numpy(), fresh.cpu().numpy())


def _sorted_pairs(b):
    """(tile, depth, Gaussian) of the batched step's sorted pairs, and its ranges."""
    from tests import gpu_helpers as G
    buf = b.buffers()
    n = buf["pairs"]
    keys = G.fetch(buf["sorted_pairs"], (n,), np.uint64)
    tiles = (keys >> np.uint64(buf["key_shift"])).astype(np.int64)
    if buf["sorted_values"] is None:
        splats = (keys & np.uint64((1 << buf["slot_bits"]) - 1)).astype(np.int64)
        depths = _depth_keys((keys >> np.uint64(buf["slot_bits"])) & np.uint64((1 << buf["depth_bits"]) - 1),
                             buf).astype(np.int64)
    else:
        splats = G.fetch(buf["sorted_values"], (n,), np.uint32).astype(np.int64)
        depths = (keys & np.uint64(0xFFFFFF)).astype(np.int64)
    return tiles, depths, splats, G.fetch(buf["ranges"], (buf["total_tiles"], 2), np.uint32).astype(np.int64)


@pytest.mark.parametrize("mode", [1, 2, 3])
def test_dense_tiles_sort_as_the_plain_path(mode):
    """A cloud squeezed to a few tiles (tiles of a few pairs up to tens of
    thousands), in packed, wide and renumbered-depth pairs, against the plain
    path's pairs to the bit (at its tile size, 16)."""
    Pq, M = _scene(40_000, 21, squeeze=0.04)
    views = _views()
    gen = torch.Generator().manual_seed(8)
    targets = [torch.rand((W * H, 3), generator=gen).cuda() for _, W, H in views]
    _, frames, _, _ = _plain(Pq, views, targets)
    b = BatchTrainer()
    b.set_key_mode(mode)
    b, colour, _, _, stats = _batched(M, views, targets, tile=16, trainer=b)
    sizes = _same_pairs(b, frames)
    assert sizes.max() > 4096 and np.any((sizes > 512) & (sizes <= 4096)) and np.any((sizes >= 2) & (sizes <= 512))


def test_dense_tiles_at_tile_32_are_sorted_and_ranged():
    """The same squeezed cloud at tile 32 (no plain-path counterpart): pairs in
    strictly increasing (tile, depth, Gaussian), each tile's range exactly its
    pairs, and the packed and wide pairs alike."""
    _, M = _scene(40_000, 21, squeeze=0.04)
    views = _views()
    gen = torch.Generator().manual_seed(8)
    targets = [torch.rand((W * H, 3), generator=gen).cuda() for _, W, H in views]
    got = {}
    for mode in (1, 2):
        b = BatchTrainer()
        b.set_key_mode(mode)
        b, _, _, _, stats = _batched(M, views, targets, tile=32, trainer=b)
        tiles, depths, splats, ranges = _sorted_pairs(b)
        assert tiles.size == stats["pairs"]
        step = np.stack([np.diff(tiles), np.diff(depths), np.diff(splats)], axis=1)
        first = np.argmax(step != 0, axis=1)
        assert np.all(step[np.arange(len(step)), first] > 0), "not strictly increasing"
        counts = np.bincount(tiles, minlength=ranges.shape[0])
        np.testing.assert_array_equal(ranges[:, 1] - ranges[:, 0], counts)
        live = counts > 0
        np.testing.assert_array_equal(ranges[live, 0], np.searchsorted(tiles, np.nonzero(live)[0]))
        assert counts.max() > 4096
        got[mode] = (tiles, depths, splats)
    for k in range(3):
        np.testing.assert_array_equal(got[1][k], got[2][k])


def test_alternating_target_buffers_replay_their_own_steps():
    """Two target buffers used in turn (an upload into one while the other is in use):
    each call replays the step captured for its buffer, and reads that buffer."""
    _, M = _scene(30_000, 17)
    views = _views()
    gen = torch.Generator().manual_seed(9)
    first = torch.cat([torch.rand((W * H, 3), generator=gen) for _, W, H in views]).cuda()
    second = torch.cat([torch.rand((W * H, 3), generator=gen) for _, W, H in views]).cuda()
    b = BatchTrainer()
    b.set_views(views)
    b.set_tuning(16, 256)
    colour = torch.empty((b.pixels, 4), device="cuda")
    loss = torch.zeros(1, device="cuda")
    grads = A.Params(torch.zeros_like(M.means), torch.zeros_like(M.scales), torch.zeros_like(M.quats),
                     torch.zeros((M.count, 48), device="cuda"), 3)
    seen = []
    for target in (first, second, first, second):
        b.step(M, target, colour, loss, grads)
        torch.cuda.synchronize()
        seen.append((loss.item(), colour.cpu().numpy().copy(), grads.means.cpu().numpy().copy()))
    b.check()
    assert seen[0][0] != seen[1][0]
    for k in (0, 1):
        # the loss is a sum by float atomics, in no fixed order
        assert abs(seen[k][0] - seen[k + 2][0]) <= 1e-5 * abs(seen[k][0])
        np.testing.assert_array_equal(seen[k][1], seen[k + 2][1])
        g, h = seen[k][2], seen[k + 2][2]
        assert np.abs(g - h).max() <= 1e-5 * np.abs(g).max()


def test_batched_render_draws_the_training_steps_colour():
    """ath_batch_render: every view's forward alone gives, to the bit, the colour a
    training step draws on the same cloud and views; the plain path's images agree
    within the fast exponential's rounding; a render does not disturb the next step."""
    Pq, M = _scene(40_000, 23)
    views = _views()
    gen = torch.Generator().manual_seed(10)
    targets = [torch.rand((W * H, 3), generator=gen).cuda() for _, W, H in views]
    images, _, _, _ = _plain(Pq, views, targets)
    b, colour, loss, grads, _ = _batched(M, views, targets)
    drawn = torch.full_like(colour, -1.0)
    b.render(M, drawn)
    torch.cuda.synchronize()
    b.check()
    np.testing.assert_array_equal(drawn.cpu().numpy(), colour.cpu().numpy())
    got = drawn.cpu().numpy()
    base = 0
    for (proj, W, H), img in zip(views, images):
        d = np.abs(got[base:base + W * H] - img.cpu().numpy()).max(axis=1)
        assert np.mean(d <= 1e-4) >= 0.9999
        base += W * H
    # a training step after the render still trains (its own captured graph)
    first_loss = loss.item()
    b.step(M, torch.cat(targets).contiguous(), colour, loss, grads)
    torch.cuda.synchronize()
    assert abs(loss.item() - first_loss) <= 1e-5 * abs(first_loss)


@pytest.mark.parametrize("mode", [0, 1])
def test_batched_render_depth_is_the_plain_paths(mode):
    """ath_batch_render's depth, in the mean and in the threshold mode, against the
    plain path's depth target on the same cloud and views: equal but for the rare
    blend decision the fast exponential takes the other way."""
    Pq, M = _scene(40_000, 24)
    views = _views()
    settings = lambda W, H: A.RenderSettings(width=W, height=H, depth_mode=mode, depth_threshold=0.4)
    raster = A.TileRasterizer.create()
    plain = []
    for proj, W, H in views:
        t = A.RenderTargets.make(W, H)
        raster.render_params(proj, Pq, settings(W, H), t)
        plain.append((t.colour.clone(), t.depth.clone()))
    b = BatchTrainer()
    b.set_views(views, settings(1, 1))
    b.set_tuning(16, 256)
    colour = torch.empty((b.pixels, 4), device="cuda")
    depth = torch.full((b.pixels,), -1.0, device="cuda")
    b.render(M, colour, depth)
    torch.cuda.synchronize()
    b.check()
    got = depth.cpu().numpy()
    base = 0
    for (_, W, H), (pc, pd) in zip(views, plain):
        d, want = got[base:base + W * H], pd.cpu().numpy()
        covered = pc.cpu().numpy()[:, 3] > 1e-2
        rel = np.abs(d - want) / np.maximum(np.abs(want), 1e-6)
        assert np.all(d[~covered] >= 0.0)
        assert np.mean(rel[covered] <= 1e-4) >= 0.999, float(np.mean(rel[covered] <= 1e-4))
        base += W * H


def test_gradient_buckets_give_the_same_gradients_and_signal_each_bucket():
    """ath_batch_set_buckets: the projection adjoint bucket by bucket, an event after each. A
    side stream that waits on bucket k's event and copies that bucket out (where a multi-GPU
    step posts its all-reduce) sees it final; the gradients equal the one-set step's to the rounding
    of their atomic sums, whose order varies from run to run."""
    Pq, M = _scene(40_000, 21)
    views = _views()
    gen = torch.Generator().manual_seed(8)
    targets = [torch.rand((W * H, 3), generator=gen).cuda() for _, W, H in views]
    b, _, loss_one, grads_one, _ = _batched(M, views, targets)
    buckets = A.BucketedGradients(M.count, 4, 48, 3, device="cuda")
    events = [torch.cuda.Event() for _ in range(4)]
    b.set_buckets(buckets, events)
    colour = torch.empty((b.pixels, 4), device="cuda")
    loss = torch.zeros(1, device="cuda")
    target = torch.cat(targets).contiguous()
    side = torch.cuda.Stream()
    copies = [torch.empty_like(s) for s in buckets.slices]
    for _ in range(2):   # the first step captures its graph, the second replays it
        buckets.flat.fill_(float("nan"))
        b.step(M, target, colour, loss, None)
        for k, e in enumerate(events):
            side.wait_event(e)
            with torch.cuda.stream(side):
                copies[k].copy_(buckets.slices[k])
        torch.cuda.current_stream().wait_stream(side)
        b.check()
        torch.cuda.synchronize()
        for k in range(4):
            np.testing.assert_array_equal(copies[k].cpu().numpy(), buckets.slices[k].cpu().numpy())
        got = buckets.gather()
        for name in ("means", "scales", "quats", "sh"):
            want = getattr(grads_one, name).cpu().numpy()
            np.testing.assert_allclose(getattr(got, name).cpu().numpy(), want, rtol=1e-4,
                                       atol=1e-5 * float(np.abs(want).max()), err_msg=name)
        # the loss is a float atomic sum over blocks, in an order that varies from run to run
        assert abs(loss.item() - loss_one.item()) <= 2e-5 * loss_one.item()
    b.set_buckets(None)


@pytest.mark.gpu
def test_a_step_whose_blends_wait_for_the_target_upload_equals_the_step():
    """ath_batch_train_step_after: the target is copied from pinned host memory on a side
    stream while the step's projection and sort run; only the blends wait for its event.
    Twice on each of two device buffers (captured, then replayed), the image, the loss and
    the gradients equal the plain step's (to the rounding of atomic sums, whose order varies)."""
    Pq, M = _scene(40_000, 23)
    views = _views()
    gen = torch.Generator().manual_seed(9)
    targets = [torch.rand((W * H, 3), generator=gen).cuda() for _, W, H in views]
    b, colour_one, loss_one, grads_one, _ = _batched(M, views, targets)
    host = torch.cat(targets).cpu().pin_memory()
    staging = [torch.empty_like(host, device="cuda") for _ in range(2)]
    ready = [torch.cuda.Event() for _ in range(2)]
    side = torch.cuda.Stream()
    colour = torch.empty_like(colour_one)
    loss = torch.zeros(1, device="cuda")
    grads = A.Params(torch.zeros_like(M.means), torch.zeros_like(M.scales), torch.zeros_like(M.quats),
                     torch.zeros((M.count, 48), device="cuda"), 3)
    main = torch.cuda.current_stream()
    for k in range(4):
        torch.cuda.synchronize()
        staging[k % 2].zero_()
        side.wait_stream(main)
        with torch.cuda.stream(side):
            staging[k % 2].copy_(host, non_blocking=True)
            ready[k % 2].record(side)
        b.step(M, staging[k % 2], colour, loss, grads, stream=main, target_ready=ready[k % 2])
        b.check()
        torch.cuda.synchronize()
        np.testing.assert_array_equal(colour.cpu().numpy(), colour_one.cpu().numpy())
        assert abs(loss.item() - loss_one.item()) <= 2e-5 * loss_one.item()
        for name in ("means", "scales", "quats", "sh"):
            want = getattr(grads_one, name).cpu().numpy()
            np.testing.assert_allclose(getattr(grads, name).cpu().numpy(), want, rtol=1e-4,
                                       atol=1e-5 * float(np.abs(want).max()), err_msg=name)


@pytest.mark.gpu
def test_gradients_of_many_views_are_the_sums_of_their_halves():
    """The projection adjoint reads only the records of the views that gave a Gaussian a
    gradient, from a word of view bits (up to 64 views; past 64, every view). 70 small
    views in one step (past 64) and as two steps of 35 (within 64): the gradients and the
    loss of the whole are the sums of the halves' (to the rounding of atomic sums)."""
    _, M = _scene(20_000, 27)
    views = []
    for v in range(70):
        cam = A.pinhole_for_vertical_fov(scenes.circle_eye(v, 70, 3.0, 0.3), (0, 0, 0), 64, 48, 60.0)
        views.append((cam.projection_for(64, 48), 64, 48))
    gen = torch.Generator().manual_seed(27)
    targets = [torch.rand((64 * 48, 3), generator=gen).cuda() for _ in views]
    _, _, loss_all, grads_all, _ = _batched(M, views, targets, 16, 128)
    _, _, loss_a, grads_a, _ = _batched(M, views[:35], targets[:35], 16, 128)
    _, _, loss_b, grads_b, _ = _batched(M, views[35:], targets[35:], 16, 128)
    assert abs(loss_all.item() - (loss_a.item() + loss_b.item())) <= 1e-4 * loss_all.item()
    for name in ("means", "scales", "quats", "sh"):
        want = (getattr(grads_a, name) + getattr(grads_b, name)).cpu().numpy()
        got = getattr(grads_all, name).cpu().numpy()
        assert np.abs(want).max() > 0, name
        np.testing.assert_allclose(got, want, rtol=1e-3, atol=1e-5 * float(np.abs(want).max()), err_msg=name)
