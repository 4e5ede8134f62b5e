"""Edge cases of the batched step (ath_batch_*) on a B200: an empty cloud, a
cloud no view can see, the cloud changing size between steps on one trainer,
views of one pixel and of ragged sizes at every tile size, and the pair form
switched between steps. Each is held against the plain path, a fresh trainer,
or the background it must draw."""
import numpy as np
import pytest
import torch

import athenea_b200 as A
from athenea_b200 import scenes
from athenea_b200.raster import BatchTrainer, MixedParams

from tests.test_gpu_batch import _batched, _plain, _same_pairs, _scene, _views

pytestmark = pytest.mark.gpu

BG = (0.25, 0.5, 0.75, 1.0)


def _empty_grads(n):
    return A.Params(torch.zeros((n, 4), device="cuda"), torch.zeros((n, 4), device="cuda"),
                    torch.zeros((n, 4), device="cuda"), torch.zeros((n, 48), device="cuda"), 3)


def _background_loss(views, targets):
    bg = np.array(BG[:3], np.float64)
    return sum(float(np.mean((bg[None, :] - t.cpu().numpy().astype(np.float64)) ** 2)) for t in targets)


def _step_with_background(M, views, targets, grads):
    b = BatchTrainer()
    b.set_views(views, A.RenderSettings(background=BG))
    colour = torch.full((b.pixels, 4), float("nan"), device="cuda")
    loss = torch.zeros(1, device="cuda")
    b.step(M, torch.cat(targets).contiguous(), colour, loss, grads)
    stats = b.check()
    torch.cuda.synchronize()
    return b, colour, loss, stats


def test_an_empty_cloud_draws_the_background_and_its_loss():
    views = _views(2)
    M = MixedParams.from_params(_empty_grads(0))
    gen = torch.Generator().manual_seed(21)
    targets = [torch.rand((W * H, 3), generator=gen).cuda() for _, W, H in views]
    b, colour, loss, stats = _step_with_background(M, views, targets, _empty_grads(0))
    assert stats["pairs"] == 0 and stats["kept"] == 0
    np.testing.assert_array_equal(colour.cpu().numpy(), np.tile(np.array(BG, np.float32), (b.pixels, 1)))
    want = _background_loss(views, targets)
    assert abs(loss.item() - want) <= 1e-5 * want
    # the batched render of the same: the background again
    again = torch.full_like(colour, float("nan"))
    b.render(M, again)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(again.cpu().numpy(), colour.cpu().numpy())


def test_a_cloud_behind_the_camera_draws_the_background_and_has_zero_gradients():
    views = _views(1)
    eye = np.array(scenes.circle_eye(0, 8, 3.0, 0.3))
    Pq, _ = _scene(5_000, 22)
    means = Pq.means.clone()
    behind = torch.tensor(eye * 1.7, dtype=torch.float32, device="cuda")   # past the eye, away from the target
    means[:, :3] = behind + 0.05 * (means[:, :3] - means[:, :3].mean(0))
    P = A.Params(means, Pq.scales, Pq.quats, Pq.sh, 3)
    M = MixedParams.from_params(P)
    gen = torch.Generator().manual_seed(22)
    targets = [torch.rand((W * H, 3), generator=gen).cuda() for _, W, H in views]
    grads = _empty_grads(P.count)
    for g in (grads.means, grads.scales, grads.quats, grads.sh):
        g.fill_(float("nan"))   # the step overwrites every row
    b, colour, loss, stats = _step_with_background(M, views, targets, grads)
    assert stats["pairs"] == 0 and stats["kept"] == 0
    np.testing.assert_array_equal(colour.cpu().numpy(), np.tile(np.array(BG, np.float32), (b.pixels, 1)))
    want = _background_loss(views, targets)
    assert abs(loss.item() - want) <= 1e-5 * want
    for g in (grads.means, grads.scales, grads.quats, grads.sh):
        assert torch.count_nonzero(g).item() == 0


def test_the_cloud_shrinking_and_growing_back_draws_as_fresh_trainers():
    _, M = _scene(30_000, 23)
    views = _views()
    gen = torch.Generator().manual_seed(23)
    targets = [torch.rand((W * H, 3), generator=gen).cuda() for _, W, H in views]
    b = BatchTrainer()
    for n in (30_000, 10_000, 0, 30_000, 20_000):
        part = MixedParams(M.means[:n], M.scales[:n], M.quats[:n], M.sh_low[:n], M.sh_high[:n], M.sh_scale[:n], 3)
        _, colour, loss, _, stats = _batched(part, views, targets, trainer=b)
        _, fresh, fresh_loss, _, fresh_stats = _batched(part, views, targets)
        np.testing.assert_array_equal(colour.cpu().numpy(), fresh.cpu().numpy(), err_msg=f"{n} Gaussians")
        assert stats["pairs"] == fresh_stats["pairs"] and stats["kept"] == fresh_stats["kept"]
        assert abs(loss.item() - fresh_loss.item()) <= 1e-5 * fresh_loss.item()
        if n == 0:
            assert stats["pairs"] == 0 and not colour.any()


def test_views_of_one_pixel_and_ragged_sizes_match_the_plain_path():
    Pq, M = _scene(50_000, 24)
    sizes = [(1, 1), (33, 17), (7, 300), (300, 7), (65, 33)]
    views = []
    for v, (W, H) in enumerate(sizes):
        cam = A.pinhole_for_vertical_fov(scenes.circle_eye(v, 8, 3.0, 0.3), (0, 0, 0), W, H, 60.0)
        views.append((cam.projection_for(W, H), W, H))
    gen = torch.Generator().manual_seed(24)
    targets = [torch.rand((W * H, 3), generator=gen).cuda() for _, W, H in views]
    images, frames, loss_p, grads_p = _plain(Pq, views, targets)
    plain = np.concatenate([img.cpu().numpy() for img in images])
    ref = None
    for tile in (16, 8, 32):
        b, colour, loss_b, grads_b, stats = _batched(M, views, targets, tile, 64)
        if tile == 16:   # the plain path's tile: the same pairs, to the bit
            assert stats["pairs"] == sum(f["pairs"] for f in frames)
            _same_pairs(b, frames)
        got = colour.cpu().numpy()
        d = np.abs(got - plain).max(axis=1)
        assert int(np.sum(d > 1e-4)) <= 5 and d.max() <= 2e-2, (tile, int(np.sum(d > 1e-4)), float(d.max()))
        assert abs(loss_b.item() - loss_p.item()) <= 1e-4 * loss_p.item()
        if ref is None:
            ref = got
            for name in ("means", "sh"):
                a = getattr(grads_b, name).cpu().numpy().ravel().astype(np.float64)
                c = getattr(grads_p, name).cpu().numpy().ravel().astype(np.float64)
                assert np.dot(a, c) / (np.linalg.norm(a) * np.linalg.norm(c) + 1e-30) > 0.999, name
        else:
            np.testing.assert_array_equal(got, ref, err_msg=f"tile {tile}")


def test_the_pair_form_switched_between_steps_draws_the_same_image():
    _, M = _scene(30_000, 25)
    views = _views()
    gen = torch.Generator().manual_seed(25)
    targets = [torch.rand((W * H, 3), generator=gen).cuda() for _, W, H in views]
    b = BatchTrainer()
    first = None
    for mode in (0, 2, 1, 0):
        b.set_key_mode(mode)
        _, colour, loss, _, stats = _batched(M, views, targets, trainer=b)
        img = colour.cpu().numpy()
        if first is None:
            first = (img, stats["pairs"], loss.item())
        else:
            np.testing.assert_array_equal(img, first[0], err_msg=f"key mode {mode}")
            assert stats["pairs"] == first[1]
            assert abs(loss.item() - first[2]) <= 1e-5 * first[2]
