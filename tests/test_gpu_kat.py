"""The reference's known-answer render tests (tests/render/test_splat_render.cpp),
run against the CUDA path through its public API."""
import numpy as np
import pytest
import torch

import athenea_b200 as A
from athenea_b200 import AtheneaError
from tests.fixtures import ENC_BUILDER, CloudBuilder, product_encoding, random_cloud

pytestmark = pytest.mark.gpu


def _upload(b: CloudBuilder, max_degree=3) -> A.GpuSplats:
    recs = torch.from_numpy(b.records().reshape(-1)).cuda()
    return A.CloudLoader.upload(recs, product_encoding(ENC_BUILDER), max_degree)


def _draw(raster, cam, clouds, W, H, **kw):
    s = A.RenderSettings(width=W, height=H)
    for k, v in kw.items():
        setattr(s, k, v)
    t = A.RenderTargets.make(W, H)
    stats = raster.render(cam, [A.SplatInstance(c) for c in clouds], s, t)
    torch.cuda.synchronize()
    return stats, t.colour.cpu().numpy(), t.depth.cpu().numpy()


@pytest.fixture(scope="module")
def raster(native):
    return A.TileRasterizer.create()


def test_single_splat_lands_on_the_pixel_the_camera_arithmetic_says(raster):   # :130-157
    cloud = _upload(CloudBuilder().add(1.0, 0.5, -10.0, 0.9, 0.02, 0.02, 0.02, (1, 0, 0, 0), (1, 1, 1)))
    cam = A.Camera()
    cam.lens.focal = cam.lens.haperture
    _, c, _ = _draw(raster, cam, [cloud], 320, 240)
    best = int(np.argmax(c[:, 3]))
    assert abs(best % 320 - 192) <= 1 and abs(best // 320 - 136) <= 1


def test_nearer_splat_wins_from_either_side_and_left_stays_left(raster):   # :159-206
    b = CloudBuilder()
    b.add(0.0, 0.0, -1.0, 0.99, 0.5, 0.5, 0.05, (1, 0, 0, 0), (1, 0, 0))
    b.add(0.0, 0.0, 1.0, 0.99, 0.5, 0.5, 0.05, (1, 0, 0, 0), (0, 0, 1))
    b.add(-3.0, 0.0, 0.0, 0.99, 0.3, 0.3, 0.3, (1, 0, 0, 0), (0, 1, 0))
    cloud = _upload(b)
    _, c, _ = _draw(raster, A.Camera.looking_at((0, 0, 10), (0, 0, 0)), [cloud], 200, 100)
    centre = c[50 * 200 + 100]
    assert centre[2] > 0.9 and centre[0] < 0.1 and int(np.argmax(c[50 * 200:51 * 200, 1])) < 100
    _, c, _ = _draw(raster, A.Camera.looking_at((0, 0, -10), (0, 0, 0)), [cloud], 200, 100)
    centre = c[50 * 200 + 100]
    assert centre[0] > 0.9 and centre[2] < 0.1 and int(np.argmax(c[50 * 200:51 * 200, 1])) > 100


def test_antialiasing_pays_back_the_energy_dilation_adds(raster):   # :208-235
    cloud = _upload(CloudBuilder().add(0.0, 0.0, -50.0, 0.9, 0.002, 0.002, 0.002, (1, 0, 0, 0), (1, 1, 1)))
    e = {aa: float(_draw(raster, A.Camera(), [cloud], 64, 64, antialias=aa)[1][:, 3].astype(np.float64).sum())
         for aa in (True, False)}
    assert e[False] > 0.0 and e[True] < 0.6 * e[False]


def test_counters_say_how_many_were_kept_and_why(native):   # :1831-1917
    raster = A.TileRasterizer.create()
    first = CloudBuilder()
    for k in range(10):
        first.add(-0.9 + 0.2 * k, 0.0, -10.0, 0.8, 0.05, 0.05, 0.05, (1, 0, 0, 0), (1, 1, 1))
    for k in range(4):
        first.add(0.1 * k, 0.0, 5.0, 0.8, 0.05, 0.05, 0.05, (1, 0, 0, 0), (1, 1, 1))
    for k in range(3):
        first.add(0.1 * k, 0.3, -10.0, 0.8, 1.0e-5, 1.0e-5, 1.0e-5, (1, 0, 0, 0), (1, 1, 1))
    for k in range(5):
        first.add(200.0 + k, 0.0, -10.0, 0.8, 0.05, 0.05, 0.05, (1, 0, 0, 0), (1, 1, 1))
    second = CloudBuilder()
    for k in range(6):
        second.add(-0.5 + 0.2 * k, -0.4, -8.0, 0.8, 0.05, 0.05, 0.05, (1, 0, 0, 0), (1, 1, 1))
    a, b = _upload(first), _upload(second)
    assert a.count == 22 and b.count == 6
    cam = A.Camera()
    cam.lens.focal = cam.lens.haperture
    assert raster.latest_counters() is None
    for tag in (41, 42):
        # the frame is waited for (ath_raster_check), so its counts are the newest finished
        stats, _, _ = _draw(raster, cam, [a, b], 320, 240, count_splats=True, counters_tag=tag)
        c = raster.latest_counters()
        assert c is not None and c.tag == tag
        assert c.slots == 28 and c.visible == 16 == stats.visible and c.pairs == stats.pairs
        assert c.max_tiles >= 1
        assert c.culled[2] == 4 and c.culled[4] == 3 and c.culled[5] == 5
        assert c.culled[1] == 0 and c.culled[0] == 0
        assert sum(c.culled) + c.visible == c.slots
        # per cloud (:1900-1903)
        assert len(c.clouds) == 2
        assert c.clouds[0].visible == 10 and c.clouds[1].visible == 6
        assert c.clouds[0].pairs + c.clouds[1].pairs == c.pairs
    _draw(raster, cam, [a, b], 320, 240, count_splats=False)
    assert raster.latest_counters().tag == 42


def test_counters_come_back_without_waiting(native):
    """latestCounters never waits (TileRasterizer.h:373-374): frames drawn without a check
    return at once, and the counters name the newest counted frame the device finished."""
    raster = A.TileRasterizer.create()
    cloud = _upload(random_cloud(3000, 7))
    cam = A.Camera.looking_at((1.5, 1.0, 6.0), (0, 0, 0))
    s = A.RenderSettings(width=250, height=190, count_splats=True)
    t = A.RenderTargets.make(250, 190)
    seen = []
    for tag in range(1, 8):
        s.counters_tag = tag
        stats = raster.render(cam, [A.SplatInstance(cloud)], s, t, do_check=False)
        assert stats.splats == 3000
        c = raster.latest_counters()
        if c is not None:
            seen.append(c.tag)
    assert seen == sorted(seen)   # never an older frame after a newer one
    torch.cuda.synchronize()
    c = raster.latest_counters()
    assert c.tag == 7 and c.slots == 3000 and len(c.clouds) == 1 and c.clouds[0].visible == c.visible
    assert raster.check().pairs == c.pairs


def test_a_frame_past_its_capacity_is_reported_then_grown(oracle, native):
    """A frame is drawn with no read back: its pairs are sized from what earlier frames
    needed. A frame that outgrows that is reported (ATH_E_CAPACITY) and the next is drawn
    whole, equal to the restatement."""
    from tests import gpu_helpers as G
    raster = A.TileRasterizer.create()
    cam = A.Camera.looking_at((1.5, 1.0, 6.0), (0, 0, 0))
    W, H = 250, 190
    small = _upload(random_cloud(300, 7))
    big_rec = random_cloud(3000, 7)
    big = _upload(big_rec)
    _draw(raster, cam, [small], W, H)   # the handle's first frame sizes the pairs for the small cloud
    s = A.RenderSettings(width=W, height=H)
    t = A.RenderTargets.make(W, H)
    raster.render(cam, [A.SplatInstance(big)], s, t, do_check=False)
    with pytest.raises(AtheneaError) as e:
        raster.check()
    assert e.value.name == "Capacity"
    stats = raster.render(cam, [A.SplatInstance(big)], s, t)   # grown from the frame before
    got = G.frame_buffers(raster)
    pos, shape, sh, _, shw = oracle.decode(big_rec.records().reshape(-1), ENC_BUILDER, 3)
    want = oracle.render([(pos, shape, sh, 3, shw, np.eye(4), 0)], G.oracle_projection(oracle, cam.projection_for(W, H)),
                         W, H)
    assert stats.pairs == got["pairs"] == want["binned"]["pairs"]
    np.testing.assert_array_equal(got["pair_splats"], want["binned"]["pair_splats"])
    np.testing.assert_array_equal(got["ranges"].reshape(-1), want["binned"]["ranges"])
    assert np.abs(t.colour.cpu().numpy() - want["colour"]).max() <= 1e-5


def test_a_frame_of_no_splats_draws_the_background(raster):   # :1919-1954, the splat half
    cloud = _upload(random_cloud(3000, 11))
    cam = A.Camera.looking_at((1.5, 1.0, 6.0), (0, 0, 0))
    _draw(raster, cam, [cloud], 250, 190)
    for _ in range(2):
        stats, c, d = _draw(raster, cam, [], 250, 190, background=(0.1, 0.2, 0.3, 0.4))
        assert stats.pairs == 0
        assert np.all(c == np.array([0.1, 0.2, 0.3, 0.4], np.float32)) and np.all(d == 0.0)


def test_errors_are_the_references(raster):   # TileRasterizer.cpp:302-325
    cloud = _upload(random_cloud(10, 1))
    with pytest.raises(AtheneaError) as e:
        _draw(raster, A.Camera(), [cloud], 0, 10)
    assert e.value.name == "InvalidArgument"
    s = A.RenderSettings(width=64, height=64)
    t = A.RenderTargets.make(32, 32)
    with pytest.raises(AtheneaError) as e:
        raster.render(A.Camera(), [A.SplatInstance(cloud)], s, t)
    assert e.value.name == "InvalidArgument"


def test_release_scratch_then_draw_again(raster):   # TileRasterizer.cpp:178-191
    cloud = _upload(random_cloud(3000, 7))
    cam = A.Camera.looking_at((1.5, 1.0, 6.0), (0, 0, 0))
    _, c1, _ = _draw(raster, cam, [cloud], 250, 190)
    raster.release_scratch()
    _, c2, _ = _draw(raster, cam, [cloud], 250, 190)
    np.testing.assert_array_equal(c1, c2)


def test_timed_stages_fill_the_stats(raster):   # TileRasterizer.cpp:38-59
    cloud = _upload(random_cloud(3000, 7))
    stats, _, _ = _draw(raster, A.Camera.looking_at((1.5, 1.0, 6.0), (0, 0, 0)), [cloud], 250, 190, time_stages=True)
    assert stats.project_ms > 0 and stats.blend_ms > 0 and stats.total_ms >= stats.blend_ms
