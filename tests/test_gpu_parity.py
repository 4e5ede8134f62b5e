"""The CUDA path against the CPU restatement, through the C ABI, on a B200.

Integer work (depth keys and cull reasons, tile rects, tiles touched, sorted
pairs, tile ranges) must match bit for bit; so must the projection records.
Images must be within 1e-5 max-abs per channel (they are expected to match to
the bit: both sides run the same float operations in the same order).
"""
import numpy as np
import pytest
import torch

import athenea_b200 as A
from tests.fixtures import ENC_BUILDER, CloudBuilder, product_encoding, random_cloud, rotation_y, scaling, translation

pytestmark = pytest.mark.gpu

IMAGE_TOL = 1e-5


@pytest.fixture(scope="module")
def raster(native):
    return A.TileRasterizer.create()


def _settings(W, H, **kw):
    s = A.RenderSettings(width=W, height=H)
    for k, v in kw.items():
        setattr(s, k, v)
    return s


def _compare(O, H_, raster, packed_list, o2w_list, proj, s: A.RenderSettings, linear=False, edit=None):
    """Draws with both and checks every intermediate and output."""
    from tests import gpu_helpers as G
    splats = [G.upload(p) for p in packed_list]
    for sp in splats:
        sp.linear = linear
    inst = [A.SplatInstance(sp, o) for sp, o in zip(splats, o2w_list)]
    if edit is not None:
        inst[0].edit = edit
    targets = A.RenderTargets.make(s.width, s.height, position=True)
    stats = raster.render(proj, inst, s, targets)
    torch.cuda.synchronize()
    got = dict(colour=targets.colour.cpu().numpy(), depth=targets.depth.cpu().numpy(),
               position=targets.position.cpu().numpy())
    got.update(G.frame_buffers(raster))
    op = G.oracle_projection(O, proj)
    oedit = None
    if edit is not None:
        oedit = O.Edit(active=1, shape=edit.shape, mode=edit.mode, invert=int(edit.invert))
        oedit.centre[:], oedit.size[:], oedit.tint[:] = list(edit.centre), list(edit.size), list(edit.tint)
        oedit.saturation, oedit.brightness, oedit.opacity = edit.saturation, edit.brightness, edit.opacity
        oedit.minOpacity, oedit.maxScale = edit.min_opacity, edit.max_scale
    inst_o = [(p[0], p[1], p[2], p[3], p[4], o, int(linear)) for p, o in zip(packed_list, o2w_list)]
    want = O.render(inst_o, op, s.width, s.height, antialias=int(s.antialias), max_sh_degree=s.max_sh_degree,
                    bg=s.background, depth_mode=s.depth_mode, depth_threshold=s.depth_threshold,
                    edit=oedit)
    wp = want["proj"]
    slots = wp["keys"].shape[0]
    assert got["slots"] == slots == stats.splats
    # depth keys and cull reasons
    np.testing.assert_array_equal(got["keys"], wp["keys"])
    kept = wp["visible"] != 0
    assert stats.visible == int(kept.sum()) == want["binned"]["visible"]
    # tiles touched and rects, kept slots
    np.testing.assert_array_equal(G.touched_of(got), wp["touched"].astype(np.int64))
    r = got["rects"][kept]
    rects = np.stack([r[:, 0] & 0xFFFF, r[:, 0] >> 16, r[:, 1] & 0xFFFF, r[:, 1] >> 16], axis=1)
    np.testing.assert_array_equal(rects, wp["rects"][kept])
    # the records, bit for bit
    np.testing.assert_array_equal(got["records"][kept].view(np.uint32), wp["records"][kept].view(np.uint32))
    # the sorted pairs and the ranges
    assert got["pairs"] == want["binned"]["pairs"] == stats.pairs
    np.testing.assert_array_equal((got["pair_keys"] >> np.uint64(24)).astype(np.uint32), want["binned"]["pair_tiles"])
    np.testing.assert_array_equal(got["pair_splats"], want["binned"]["pair_splats"])
    np.testing.assert_array_equal(got["ranges"].reshape(-1), want["binned"]["ranges"])
    # images
    err_c = np.abs(got["colour"] - want["colour"]).max() if got["colour"].size else 0.0
    err_d = np.abs(got["depth"] - want["depth"]).max() if got["depth"].size else 0.0
    assert err_c <= IMAGE_TOL and err_d <= IMAGE_TOL * max(1.0, float(np.abs(want["depth"]).max()))
    pos_want = O.position(want["frame"], op, want["depth"])
    np.testing.assert_allclose(got["position"], pos_want, rtol=1e-5, atol=1e-5)
    return got, want


def _decode(O, b, keep=3):
    pos, shape, sh, _, shw = O.decode(b.records().reshape(-1), ENC_BUILDER, keep)
    rpc = {1: 0, 5: 3, 12: 8, 23: 15}[shw]
    return pos, shape, sh, rpc, shw


# ---- the reference's comparison scenes (test_splat_render.cpp:77-128) -----------
@pytest.mark.parametrize("section", ["perspective", "frustum", "orthographic", "no-aa-window-roll", "two-instances"])
def test_frame_matches_the_restatement(oracle, native, raster, section):
    packed = _decode(oracle, random_cloud(3000, 7))
    W, H = 250, 190
    s = _settings(W, H)
    o2w = [np.eye(4)]
    if section == "perspective":
        cam = A.Camera.looking_at((1.5, 1.0, 6.0), (0, 0, 0)); cam.lens.focal = 30.0
    elif section == "frustum":
        cam = A.Camera.looking_at((0.3, -0.2, 2.2), (0, 0, 0)); cam.lens.focal = 18.0
    elif section == "orthographic":
        cam = A.Camera.looking_at((0.0, 3.0, 5.0), (0, 0, 0)); cam.lens.orthographic = True; cam.lens.focal = 5.0
    elif section == "no-aa-window-roll":
        cam = A.Camera.looking_at((-2.0, 0.5, 5.0), (0, 0, 0))
        cam.lens.window_translate = (0.2, 0.0); cam.lens.window_scale = (1.0, 1.3); cam.lens.window_roll = 25.0
        s.antialias = False
    else:
        cam = A.Camera.looking_at((2.0, 1.5, 7.0), (0, 0, -0.5))
        o2w = [np.eye(4), translation((0.5, 0.0, -1.5)) @ rotation_y(40.0) @ scaling((1.0, 0.7, 1.3))]
    _compare(oracle, None, raster, [packed] * len(o2w), o2w, cam.projection_for(W, H), s)


def test_frame_options_match(oracle, native, raster):
    """A linear cloud, a background, threshold depth, an active edit, SH capped at degree 1."""
    packed = _decode(oracle, random_cloud(2000, 11))
    W, H = 200, 150
    cam = A.Camera.looking_at((1.0, 0.5, 5.0), (0, 0, 0))
    s = _settings(W, H, background=(0.1, 0.2, 0.3, 0.5), depth_mode=1, depth_threshold=0.4, max_sh_degree=1)
    edit = A.SplatEdit(active=True, shape=1, mode=2, centre=(0.2, 0.0, 0.0), size=(1.2, 1.0, 1.0),
                       tint=(1.0, 0.5, 0.8), saturation=0.7, brightness=1.3, opacity=0.8)
    _compare(oracle, None, raster, [packed], [np.eye(4)], cam.projection_for(W, H), s, linear=True, edit=edit)


def test_degree3_clustered_scene_matches(oracle, native, raster):
    from athenea_b200 import scenes
    recs, enc = scenes.records(60_000, True, scenes.SEED + 1)
    e = {("rotW" if k == "rot_w" else "rotX" if k == "rot_x" else "rotY" if k == "rot_y" else "rotZ" if k == "rot_z"
          else "restBase" if k == "rest_base" else "filePerColour" if k == "file_per_colour" else k): v
         for k, v in enc.items()}
    pos, shape, sh, _, shw = oracle.decode(recs.reshape(-1), e, 15)
    W, H = 480, 270
    cam = A.pinhole_for_vertical_fov((0, 0, 3), (0, 0, 0), W, H, 60.0)
    _compare(oracle, None, raster, [(pos, shape, sh, 15, shw)], [np.eye(4)], cam.projection_for(W, H), _settings(W, H))


def test_uniform_100k_at_960x540_matches(oracle, native, raster):
    """The plain forward's own workload (100k uniform means, 960x540), whole."""
    from athenea_b200 import scenes
    recs, enc = scenes.records(100_000, False, scenes.SEED)
    e = {("rotW" if k == "rot_w" else "rotX" if k == "rot_x" else "rotY" if k == "rot_y" else "rotZ" if k == "rot_z"
          else "restBase" if k == "rest_base" else "filePerColour" if k == "file_per_colour" else k): v
         for k, v in enc.items()}
    pos, shape, sh, _, shw = oracle.decode(recs.reshape(-1), e, 15)
    W, H = 960, 540
    cam = A.pinhole_for_vertical_fov((0, 0, 3), (0, 0, 0), W, H, 60.0)
    _compare(oracle, None, raster, [(pos, shape, sh, 15, shw)], [np.eye(4)], cam.projection_for(W, H), _settings(W, H))


# ---- the decode (scene/splat_decode.slang, splat_validate.slang) ------------------
def test_decode_matches_the_restatement(oracle, native):
    from athenea_b200 import scenes
    recs, enc = scenes.records(20_000, True, 99)
    recs[5, 0] = np.nan                                    # dropped: a NaN position
    recs[6, enc["opacity"]] = -10.0                        # dropped: too faint
    recs[7, enc["scale0"]] = -40.0                         # a surfel's flat axis: kept
    recs[8, enc["scale0"]] = -40.0
    recs[8, enc["scale1"]] = -40.0                         # two flat axes: dropped
    recs[9, enc["scale2"]] = 70.0                          # past e^60: dropped
    recs[10, enc["dc0"]] = 1e6                             # clamped to 65000 before f16
    recs[11, enc["rot_w"]:enc["rot_w"] + 4] = 0.0          # no rotation: identity
    e = {("rotW" if k == "rot_w" else "rotX" if k == "rot_x" else "rotY" if k == "rot_y" else "rotZ" if k == "rot_z"
          else "restBase" if k == "rest_base" else "filePerColour" if k == "file_per_colour" else k): v
         for k, v in enc.items()}
    for keep in (15, 8, 3, 0):
        pos, shape, sh, origin, shw = oracle.decode(recs.reshape(-1), e, keep)
        g = A.CloudLoader.upload(torch.from_numpy(recs.reshape(-1)).cuda(), enc,
                                 max_degree={15: 3, 8: 2, 3: 1, 0: 0}[keep])
        assert g.count == pos.shape[0] == 20_000 - 4
        assert g.sh_words == shw
        np.testing.assert_array_equal(g.positions.cpu().numpy()[:g.count].view(np.uint32), pos.view(np.uint32))
        np.testing.assert_array_equal(g.shape.cpu().numpy()[:g.count].view(np.uint32), shape)
        np.testing.assert_array_equal(g.sh.cpu().numpy()[:g.count].view(np.uint32), sh)


# ---- the sort (tests/gpu/test_algo.cpp:347-379) ---------------------------------
def _pcg(v):
    state = (v.astype(np.uint64) * np.uint64(747796405) + np.uint64(2891336453)) & np.uint64(0xFFFFFFFF)
    word = (((state >> ((state >> np.uint64(28)) + np.uint64(4))) ^ state) * np.uint64(277803737)) & np.uint64(0xFFFFFFFF)
    return ((word >> np.uint64(22)) ^ word) & np.uint64(0xFFFFFFFF)


def _generate(count, mode, key_bits):
    """shaders/athenea/test/sort_generate.slang's patterns, keyed as test_algo.cpp:52-66 seeds them."""
    i = np.arange(count, dtype=np.uint64)
    seed = np.uint64((0x9E3779B9 ^ count ^ (mode << 8)) & 0xFFFFFFFF)
    if mode == 0:
        lo = _pcg(i ^ seed)
        hi = _pcg((lo + seed) & np.uint64(0xFFFFFFFF))
    elif mode == 1:
        lo = np.full(count, 0x5A5A5A5A, np.uint64); hi = np.full(count, 0x0000A5A5, np.uint64)
    elif mode == 2:
        lo = i.copy(); hi = np.zeros(count, np.uint64)
    elif mode == 3:
        lo = np.uint64(count - 1) - i; hi = np.full(count, 7, np.uint64)
    else:
        lo = _pcg(i ^ seed) % np.uint64(13); hi = _pcg((i + seed) & np.uint64(0xFFFFFFFF)) % np.uint64(3)
    mask_lo = 0xFFFFFFFF if key_bits >= 32 else (1 << key_bits) - 1
    mask_hi = 0 if key_bits <= 32 else 0xFFFFFFFF if key_bits >= 64 else (1 << (key_bits - 32)) - 1
    keys = (lo & np.uint64(mask_lo)) | ((hi & np.uint64(mask_hi)) << np.uint64(32))
    return keys, np.arange(count, dtype=np.uint32)


@pytest.mark.parametrize("count,key_bits", [(1, 32), (2, 32), (4097, 13), (65537, 32), (300007, 24), (250001, 64),
                                            (100000, 40)])
def test_radix_sort_orders_keeps_ties_stable_and_loses_nothing(native, count, key_bits):
    import ctypes as C
    from athenea_b200 import _native as N
    h = C.c_void_p()
    N.check(N.lib().ath_sorter_create(C.byref(h)))
    try:
        for mode in range(5):
            keys, vals = _generate(count, mode, key_bits)
            k = torch.from_numpy(keys.view(np.int64)).cuda()
            v = torch.from_numpy(vals.view(np.int32)).cuda()
            sk = torch.empty_like(k)
            sv = torch.empty_like(v)
            stream = torch.cuda.current_stream().cuda_stream
            N.check(N.lib().ath_sorter_sort(h, C.c_void_p(k.data_ptr()), C.c_void_p(v.data_ptr()),
                                            C.c_void_p(sk.data_ptr()), C.c_void_p(sv.data_ptr()), count, key_bits,
                                            C.c_void_p(stream)))
            torch.cuda.synchronize()
            gk = k.cpu().numpy().view(np.uint64)
            gv = v.cpu().numpy().view(np.uint32)
            order = np.argsort(keys, kind="stable")
            np.testing.assert_array_equal(gk, keys[order])
            np.testing.assert_array_equal(gv, vals[order])
            # sort_stats.slang's facts: ordered, stable on ties, the same pairs permuted
            assert np.all((gk[1:] > gk[:-1]) | ((gk[1:] == gk[:-1]) & (gv[1:] > gv[:-1])))
            assert int(gk.sum(dtype=np.uint64)) == int(keys.sum(dtype=np.uint64))
            assert np.bitwise_xor.reduce(gv) == np.bitwise_xor.reduce(vals)
    finally:
        N.lib().ath_sorter_destroy(h)
