"""The CPU restatement (oracle/) pinned against the reference's own known-answer
tests, run on the CPU. Each test names the reference test it restates.
"""
import math

import numpy as np
import pytest

from tests.fixtures import ENC_BUILDER, CloudBuilder, linear_to_srgb_code, random_cloud


def _decode(O, b: CloudBuilder, keep=3):
    return O.decode(b.records().reshape(-1), ENC_BUILDER, keep)


def _render(O, cam, packed_list, width, height, o2w_list=None, **settings):
    proj = O.projection_for(cam, width, height)
    inst = []
    for k, (pos, shape, sh, _, shw) in enumerate(packed_list):
        o2w = o2w_list[k] if o2w_list else np.eye(4)
        inst.append((pos, shape, sh, 3 if shw == 5 else 0 if shw == 1 else 15, shw, o2w, 0))
    return O.render(inst, proj, width, height, **settings), proj


# ---- scalar arithmetic -------------------------------------------------------
def test_exp_log_pow_accuracy(oracle):
    xs = np.concatenate([np.linspace(-103.0, 88.0, 20001), np.linspace(-1, 1, 2001)]).astype(np.float32)
    got = np.array([oracle.exp(x) for x in xs], np.float64)
    want = np.exp(xs.astype(np.float64))
    rel = np.abs(got - want) / np.maximum(want, 1e-300)
    normal = want > 1.2e-38
    assert rel[normal].max() < 4e-7       # a few ulp
    ys = np.concatenate([np.geomspace(1e-30, 1e30, 20001), np.linspace(0.5, 2.0, 2001)]).astype(np.float32)
    got = np.array([oracle.log(y) for y in ys], np.float64)
    want = np.log(ys.astype(np.float64))
    assert np.max(np.abs(got - want) / np.maximum(np.abs(want), 1e-3)) < 4e-7
    for c in np.linspace(0.05, 3.0, 301, dtype=np.float32):
        assert abs(oracle.pow_(c, 2.4) - float(c) ** 2.4) <= 8e-7 * float(c) ** 2.4


def test_f16_round_to_nearest_even(oracle):
    rng = np.random.default_rng(1)
    vals = np.concatenate([rng.normal(0, 10, 4000), rng.normal(0, 1e-5, 2000), rng.uniform(-65000, 65000, 2000),
                           [0.0, -0.0, 1.0, 65504.0, 65519.0, 6.0e-8, 2.98e-8, 1e-9]]).astype(np.float32)
    for v in vals:
        assert oracle.f32_to_f16(v) == int(np.float16(v).view(np.uint16)), v
        h = int(np.float16(v).view(np.uint16))
        assert oracle.f16_to_f32(h) == float(np.float16(v))


def test_quaternion_round_trip(oracle):
    rng = np.random.default_rng(2)
    for _ in range(2000):
        q = rng.normal(size=4).astype(np.float32)
        q /= np.linalg.norm(q)
        d = oracle.decode_quaternion(oracle.encode_quaternion(q))
        # packing.slang:26: "within a tenth of a degree" (q and -q are the same turn)
        assert min(np.abs(d - q).max(), np.abs(d + q).max()) < 2e-3


# ---- decode: tests/scene/test_loading.cpp:91-166 ----------------------------
def test_decode_known_answers(oracle):
    enc = dict(stride=26, x=0, y=1, z=2, opacity=3, scale0=4, scale1=5, scale2=6, rotW=7, rotX=8, rotY=9, rotZ=10,
               dc0=11, dc1=12, dc2=13, restBase=14, filePerColour=3)

    def record(x, y, z, opacity, scales, rot, dc, rest):
        r = np.zeros(26, np.float32)
        r[0:3] = (x, y, z)
        r[3] = opacity
        r[4:7] = scales
        r[7:11] = rot
        r[11:14] = dc
        r[14:23] = rest
        return r

    rest = [0.1 * (k + 1) for k in range(9)]   # r: .1 .2 .3  g: .4 .5 .6  b: .7 .8 .9
    first = record(1, 2, 3, 0.0, (0.0, 0.6931472, -0.6931472), (2, 0, 0, 0), (0, 0, 0), rest)
    faint = first.copy(); faint[3] = -10.0
    broken = first.copy(); broken[0] = np.nan
    last = first.copy(); last[0:3] = (-4, 5, -6); last[3] = 1.0986123; last[7] = 0.0; last[10] = -3.0
    last[11] = 1.0 / 0.28209479
    recs = np.concatenate([first, faint, broken, last])
    pos, shape, sh, origin, shw = oracle.decode(recs, enc, 3)
    assert pos.shape[0] == 2 and list(origin) == [0, 3]
    f16 = lambda h: float(np.uint16(h).view(np.float16))
    a = pos[0]
    assert tuple(a[:3]) == (1.0, 2.0, 3.0)
    assert abs(a[3] - 0.5) <= 1e-6
    s = shape[0]
    assert math.isclose(math.exp(f16(s[1] & 0xFFFF)), 1.0, rel_tol=2e-3)
    assert math.isclose(math.exp(f16(s[1] >> 16)), 2.0, rel_tol=2e-3)
    assert math.isclose(math.exp(f16(s[2] & 0xFFFF)), 0.5, rel_tol=2e-3)
    q = oracle.decode_quaternion(int(s[0]))
    assert abs(q[3] - 1.0) <= 1e-3               # w
    assert abs(f16(s[2] >> 16) - 0.5) <= 1e-3    # base colour r
    flat = []
    for w in sh[0]:
        flat += [f16(int(w) & 0xFFFF), f16(int(w) >> 16)]
    assert abs(flat[0] - 0.1) <= 1e-3 and abs(flat[1] - 0.4) <= 1e-3 and abs(flat[2] - 0.7) <= 1e-3
    assert abs(flat[3] - 0.2) <= 1e-3
    b = pos[1]
    assert b[0] == -4.0 and abs(b[3] - 0.75) <= 1e-5
    qb = oracle.decode_quaternion(int(shape[1][0]))
    assert abs(abs(qb[2]) - 1.0) <= 1e-3
    assert abs(f16(shape[1][2] >> 16) - 1.5) <= 1e-3
    # degree capped at 0: no harmonics kept (one dummy word)
    assert oracle.decode(recs, enc, 0)[4] == 1


# ---- tests/render/test_splat_render.cpp:130-157 ------------------------------
def test_single_splat_lands_where_the_camera_arithmetic_says(oracle):
    b = CloudBuilder().add(1.0, 0.5, -10.0, 0.9, 0.02, 0.02, 0.02, (1, 0, 0, 0), (1, 1, 1))
    pos, shape, sh, _, shw = _decode(oracle, b)
    cam = oracle.default_camera()
    cam.focal = cam.haperture   # fx = width
    out, _ = _render(oracle, cam, [(pos, shape, sh, None, shw)], 320, 240)
    alpha = out["colour"][:, 3]
    best = int(np.argmax(alpha))
    x, y = best % 320, best // 320
    assert abs(x - 192) <= 1 and abs(y - 136) <= 1   # 160 + 320/10, 120 + 320*0.5/10, bottom-up


# ---- :159-206 -----------------------------------------------------------------
def test_nearer_splat_wins_from_either_side_and_left_stays_left(oracle):
    b = CloudBuilder()
    b.add(0.0, 0.0, -1.0, 0.99, 0.5, 0.5, 0.05, (1, 0, 0, 0), (1, 0, 0))
    b.add(0.0, 0.0, 1.0, 0.99, 0.5, 0.5, 0.05, (1, 0, 0, 0), (0, 0, 1))
    b.add(-3.0, 0.0, 0.0, 0.99, 0.3, 0.3, 0.3, (1, 0, 0, 0), (0, 1, 0))
    packed = _decode(oracle, b)
    W, H = 200, 100

    def centre(c):
        return c[(50 * W + 100)][:3]

    def brightest_x(c, ch):
        row = c[50 * W:(50 * W + W), ch]
        return int(np.argmax(row))

    out, _ = _render(oracle, oracle.looking_at((0, 0, 10), (0, 0, 0)), [packed], W, H)
    c = out["colour"]
    assert centre(c)[2] > 0.9 and centre(c)[0] < 0.1 and brightest_x(c, 1) < 100
    out, _ = _render(oracle, oracle.looking_at((0, 0, -10), (0, 0, 0)), [packed], W, H)
    c = out["colour"]
    assert centre(c)[0] > 0.9 and centre(c)[2] < 0.1 and brightest_x(c, 1) > 100


# ---- :208-235 -----------------------------------------------------------------
def test_antialiasing_pays_back_the_energy_dilation_adds(oracle):
    b = CloudBuilder().add(0.0, 0.0, -50.0, 0.9, 0.002, 0.002, 0.002, (1, 0, 0, 0), (1, 1, 1))
    packed = _decode(oracle, b)
    cam = oracle.default_camera()
    energy = {}
    for aa in (1, 0):
        out, _ = _render(oracle, cam, [packed], 64, 64, antialias=aa)
        energy[aa] = float(out["colour"][:, 3].astype(np.float64).sum())
    assert energy[0] > 0.0 and energy[1] < 0.6 * energy[0]


# ---- :1831-1917 ---------------------------------------------------------------
def test_cull_counters_say_why(oracle):
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
    a, b = _decode(oracle, first), _decode(oracle, second)
    assert a[0].shape[0] == 22 and b[0].shape[0] == 6
    cam = oracle.default_camera()
    cam.focal = cam.haperture
    out, _ = _render(oracle, cam, [a, b], 320, 240)
    keys = out["proj"]["keys"]
    culled = keys[keys >= 0xFF000000] & 7
    assert keys.shape[0] == 28
    assert int((keys < 0xFF000000).sum()) == 16 == out["binned"]["visible"]
    assert int((culled == 2).sum()) == 4     # Depth
    assert int((culled == 4).sum()) == 3     # Faint
    assert int((culled == 5).sum()) == 5     # Offscreen
    assert int((culled == 1).sum()) == 0     # Edit
    assert int((keys[:22] < 0xFF000000).sum()) == 10 and int((keys[22:] < 0xFF000000).sum()) == 6


# ---- :1919-1954 (the splat half: a frame of no splats draws the background) ---
def test_frame_of_no_splats_draws_the_background(oracle):
    proj = oracle.projection_for(oracle.looking_at((1.5, 1.0, 6.0), (0, 0, 0)), 250, 190)
    out = oracle.render([], proj, 250, 190, bg=(0.1, 0.2, 0.3, 0.4))
    assert out["binned"]["pairs"] == 0
    assert np.all(out["colour"] == np.array([0.1, 0.2, 0.3, 0.4], np.float32))
    assert np.all(out["depth"] == 0.0)


# ---- the two-sort form and one 64-bit sort give one order (frame.slang:17-20) --
def test_depth_sort_then_stable_tile_sort_equals_one_64bit_sort(oracle):
    packed = _decode(oracle, random_cloud(3000, 7))
    out, _ = _render(oracle, oracle.looking_at((1.5, 1.0, 6.0), (0, 0, 0)), [packed], 250, 190)
    p = out["proj"]
    f = out["frame"]
    # emit in slot order with the same tile test, then one stable sort on (tile << 24 | depth key)
    keys, vals = [], []
    for s in np.nonzero(p["visible"])[0]:
        x0, y0, x1, y1 = p["rects"][s]
        tiles = []
        for ty in range(y0, y1 + 1):
            for tx in range(x0, x1 + 1):
                tiles.append(ty * f.tilesX + tx)
        keys += tiles
        vals += [s] * len(tiles)
    # keep only the tiles the oracle's emit kept (the exact test), in slot order
    kept = set(zip(out["binned"]["pair_tiles"].tolist(), out["binned"]["pair_splats"].tolist()))
    pairs = [(t, s) for t, s in zip(keys, vals) if (t, s) in kept]
    order = sorted(range(len(pairs)), key=lambda i: (pairs[i][0] << 24) | int(p["keys"][pairs[i][1]]))
    sorted_pairs = [pairs[i] for i in order]
    assert len(sorted_pairs) == out["binned"]["pairs"]
    assert [s for _, s in sorted_pairs] == out["binned"]["pair_splats"].tolist()
    assert [t for t, _ in sorted_pairs] == out["binned"]["pair_tiles"].tolist()


def test_sampled_binning_keeps_each_sampled_tile_whole(oracle):
    """orc_bin_sampled: the pairs of every tile t % 7 == 3, each tile's run as orc_bin has it."""
    packed = _decode(oracle, random_cloud(3000, 7))
    out, _ = _render(oracle, oracle.looking_at((1.5, 1.0, 6.0), (0, 0, 0)), [packed], 250, 190)
    f, p, full = out["frame"], out["proj"], out["binned"]
    part = oracle.bin_sampled(f, p, 7, 3)
    keep = full["pair_tiles"] % 7 == 3
    np.testing.assert_array_equal(part["pair_tiles"], full["pair_tiles"][keep])
    np.testing.assert_array_equal(part["pair_splats"], full["pair_splats"][keep])
    r = full["ranges"].reshape(-1, 2)
    rp = part["ranges"].reshape(-1, 2)
    tiles = np.arange(r.shape[0])
    np.testing.assert_array_equal(np.diff(rp, axis=1)[tiles % 7 == 3], np.diff(r, axis=1)[tiles % 7 == 3])


@pytest.mark.parametrize("tile", [8, 32])
def test_other_tile_sizes_bin_each_pixel_to_the_same_records(oracle, tile):
    """At tile 8 or 32 a pixel's records (its tile's pairs whose footprint holds the
    pixel centre) are the tile-16 frame's, in the same order, and the image is the same."""
    packed = _decode(oracle, random_cloud(3000, 7))
    cam = oracle.looking_at((1.5, 1.0, 6.0), (0, 0, 0))
    W, H = 250, 190
    base, _ = _render(oracle, cam, [packed], W, H)
    proj = oracle.projection_for(cam, W, H)
    f = oracle.set_tile(oracle.frame_for(proj, np.eye(4), W, H, rest_per_colour=3, sh_words=5), tile)
    assert f.tilesX == (W + tile - 1) // tile
    pr = oracle.project(f, *packed[:3])
    binned = oracle.bin_(f, pr)
    img = oracle.blend(f, binned, pr)
    np.testing.assert_array_equal(pr["keys"][pr["visible"] != 0], base["proj"]["keys"][pr["visible"] != 0])
    np.testing.assert_array_equal(img["colour"], base["colour"])


# ---- :77-128: the raster against the ground truth, 250x190, randomCloud(3000, 7) --
@pytest.mark.parametrize("section", ["perspective", "frustum", "orthographic", "no-aa-window-roll"])
def test_raster_matches_the_fp64_ground_truth(oracle, section):
    packed = _decode(oracle, random_cloud(3000, 7))
    W, H = 250, 190
    settings = {}
    if section == "perspective":
        cam = oracle.looking_at((1.5, 1.0, 6.0), (0, 0, 0)); cam.focal = 30.0
    elif section == "frustum":
        cam = oracle.looking_at((0.3, -0.2, 2.2), (0, 0, 0)); cam.focal = 18.0
    elif section == "orthographic":
        cam = oracle.looking_at((0.0, 3.0, 5.0), (0, 0, 0)); cam.orthographic = 1; cam.focal = 5.0
    elif section == "no-aa-window-roll":
        cam = oracle.looking_at((-2.0, 0.5, 5.0), (0, 0, 0))
        cam.windowTranslate[0] = 0.2; cam.windowScale[1] = 1.3; cam.windowRoll = 25.0
        settings["antialias"] = 0
    out, proj = _render(oracle, cam, [packed], W, H, **settings)
    pos, shape, sh, _, shw = packed
    f64 = oracle.frame64(proj, np.eye(4), W, H, antialias=settings.get("antialias", 1), rest_per_colour=3,
                         sh_words=shw)
    truth = oracle.render_f64(f64, pos, shape, sh)["colour"]
    ours = linear_to_srgb_code(out["colour"][:, :3])
    ref = linear_to_srgb_code(truth[:, :3])
    d = np.abs(ours - ref).max(axis=1)
    assert np.percentile(d, 99) <= 2
    assert d.max() <= 16


# ---- contributionMode 2 and 3 (splat_blend.slang:366-380, :399-407) ----------
def test_lifted_mask_and_squared_change_contributions(oracle):
    """Mode 3 with a mask of one lifts each splat's weight itself, and with a mask
    of zero nothing. Mode 2 against the frame's own colour: one splat over an
    empty background changes each pixel by its weight times its colour, so its
    sum is the squared weights times |colour|^2, in 2^-24."""
    b = CloudBuilder().add(0.0, 0.0, -5.0, 0.8, 0.3, 0.3, 0.3, (1, 0, 0, 0), (0.8, 0.4, 0.2))
    pos, shape, sh, _, shw = _decode(oracle, b)
    out, _ = _render(oracle, oracle.default_camera(), [(pos, shape, sh, None, shw)], 160, 120)
    f, binned, proj = out["frame"], out["binned"], out["proj"]
    ones = oracle.contribution_lift(f, binned, proj, np.ones(160 * 120, np.float32))
    assert ones[0, 1] > 0 and ones[0, 0] == ones[0, 1]
    zeros = oracle.contribution_lift(f, binned, proj, np.full(160 * 120, -0.5, np.float32))   # clamped to 0
    assert zeros[0, 0] == 0 and zeros[0, 1] == ones[0, 1]
    words = oracle.contribution_change(f, binned, proj, out["colour"])
    got = int(words[0, 0]) + (int(words[0, 1]) << 32)
    colour = proj["records"][0, 8:11].astype(np.float64)
    alpha = out["colour"][:, 3].astype(np.float64)   # one splat: the coverage is its weight
    want = np.sum(np.minimum(alpha ** 2 * np.dot(colour, colour), 1.0) * 16777216.0)
    assert got > 0 and abs(got - want) <= 1e-4 * want + alpha.size


# ---- the trace (splat_trace.slang) ------------------------------------------------
def test_trace_ranks_by_weight_and_sums_to_the_coverage(oracle):
    """Each pixel's ranks come heaviest first, empty ranks last, and the ranked
    weights plus the rest the list had no room for are the pixel's coverage
    (within the halves' rounding); a pixel nothing reached is marked empty."""
    packed = _decode(oracle, random_cloud(400, 3))
    out, _ = _render(oracle, oracle.default_camera(), [packed], 96, 64)
    tr = oracle.trace(out["frame"], out["binned"], out["proj"])
    empty = tr[0] == 0xFFFFFFFE
    coverage = out["colour"][:, 3].astype(np.float64)
    assert np.all(coverage[empty] == 0) and (~empty).sum() > 100
    words = tr[8:11, ~empty]
    lo = (words & 0xFFFF).astype(np.uint16).view(np.float16).astype(np.float64)
    hi = (words >> 16).astype(np.uint16).view(np.float16).astype(np.float64)
    w = np.stack([lo[0], hi[0], lo[1], hi[1]])
    assert np.all(np.diff(w, axis=0) <= 0)                      # heaviest first
    slots = tr[0:4, ~empty]
    assert np.all((slots == 0xFFFFFFFF) == (w == 0))            # an empty rank weighs nothing
    assert np.abs(w.sum(axis=0) + lo[2] - coverage[~empty]).max() <= 4e-3
