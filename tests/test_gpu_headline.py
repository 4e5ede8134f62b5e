"""Parity on the workloads the speed-ups are quoted on, on a B200.

- The plain path at its own 1.5M workload (1.5M clustered Gaussians, one
  1920x1080 view, tile 16): depth keys and cull reasons, rects, tiles touched,
  records, sorted pairs and tile ranges bit for bit against the CPU
  restatement, the image within 1e-5.
- The batched step's sorted pairs and tile ranges against the restatement,
  view by view and bit for bit: 1.5M clustered in 8 views of 1920x1080 at
  tile 32 (what the autotuner picks) and at tile 16; 2.36M clustered in 64
  views of mixed size (every 4th tile of each view); 50M clustered in 8 views
  of 3840x2160 (every 97th tile). The restatement bins at the same tile size
  (orc_frame_set_tile) in the reference's two-sort form (a stable 24-bit depth
  sort, then a stable tile sort), which one stable sort of (tile, depth) keys
  emitted in Gaussian order reproduces (splat/frame.slang:17-20).
"""
import numpy as np
import pytest
import torch

import athenea_b200 as A
from athenea_b200 import scenes
from athenea_b200.raster import BatchTrainer, MixedParams

pytestmark = pytest.mark.gpu

SEED = scenes.SEED


def _oracle_encoding(enc: dict) -> dict:
    m = dict(rot_w="rotW", rot_x="rotX", rot_y="rotY", rot_z="rotZ", rest_base="restBase",
             file_per_colour="filePerColour")
    return {m.get(k, k): v for k, v in enc.items()}


def test_plain_path_at_1_5m_1080p_matches_the_restatement(oracle, native):
    """The plain forward's 1.5M workload, whole: every intermediate bit for bit."""
    from tests.test_gpu_parity import _compare, _settings
    recs, enc = scenes.records(1_500_000, True, SEED + 1)
    pos, shape, sh, _, shw = oracle.decode(recs.reshape(-1), _oracle_encoding(enc), 15)
    del recs
    W, H = 1920, 1080
    cam = A.pinhole_for_vertical_fov((0, 0, 3), (0, 0, 0), W, H, 60.0)
    got, want = _compare(oracle, None, A.TileRasterizer.create(), [(pos, shape, sh, 15, shw)], [np.eye(4)],
                         cam.projection_for(W, H), _settings(W, H))
    print(f"1.5M at 1920x1080: {got['pairs']} pairs, {int((want['proj']['visible'] != 0).sum())} kept, "
          f"image max-abs {float(np.abs(got['colour'] - want['colour']).max()):.3g}")


# ---- the batched step against the restatement, per view ----------------------------
def _walk(views: int, sizes, first_views: int | None = None):
    """[(projection, W, H)]: the views of a circular walk of radius 3 at height 0.3 (as bench.py's)."""
    out = []
    for v in range(views):
        W, H = sizes[v]
        eye = scenes.circle_eye(v, (first_views or views) * 4, 3.0, 0.3)
        cam = A.pinhole_for_vertical_fov(eye, (0, 0, 0), W, H, 60.0)
        out.append((cam.projection_for(W, H), W, H))
    return out


def _device_keys(buf) -> torch.Tensor:
    from tests.gpu_helpers import _DeviceView
    n = int(buf["pairs"])
    view = _DeviceView(buf["sorted_pairs"], (n,), "<i8")
    return torch.as_tensor(view, device="cuda")


def _view_pairs(keys: torch.Tensor, buf, v: int, tiles_v: int, stride: int, offset: int):
    """View v's sorted pairs whose view tile t has t % stride == offset, as (tiles, depth keys,
    Gaussians) on the host, selected on the device a chunk at a time."""
    shift, slot_bits, depth_bits = buf["key_shift"], buf["slot_bits"], buf["depth_bits"]
    base = int(buf["tile_bases"][v])
    tile_mask = (1 << max(1, (buf["total_tiles"] - 1).bit_length())) - 1
    out_t, out_d, out_g = [], [], []
    chunk = 1 << 27
    for s in range(0, keys.shape[0], chunk):
        k = keys[s:s + chunk]
        t = (k >> shift) & tile_mask
        local = t - base
        sel = (local >= 0) & (local < tiles_v)
        if stride > 1:
            sel &= torch.remainder(local, stride) == offset
        k = k[sel]
        if k.numel() == 0:
            continue
        out_t.append(((k >> shift) & tile_mask).sub_(base).cpu().numpy())
        field = ((k >> slot_bits) & ((1 << depth_bits) - 1)).cpu().numpy().astype(np.uint64)
        if depth_bits < 24:   # the renumbered exponent put back
            field = (((field >> np.uint64(16)) + np.uint64(buf["exp_base"])) << np.uint64(16)) | (field & np.uint64(0xFFFF))
        out_d.append(field)
        out_g.append((k & ((1 << slot_bits) - 1)).cpu().numpy().astype(np.uint32))
    if not out_t:
        return np.zeros(0, np.int64), np.zeros(0, np.uint64), np.zeros(0, np.uint32)
    return np.concatenate(out_t), np.concatenate(out_d), np.concatenate(out_g)


def _check_batched_against_oracle(O, p, views, tile, stride=1, label=""):
    """A batched render of `views` at `tile`, its pairs and ranges compared view by view with the
    restatement binning at the same tile size (tiles t % stride == v % stride)."""
    from tests import gpu_helpers as G
    P = A.Params(*[torch.from_numpy(np.ascontiguousarray(p[k])).cuda() for k in ("means", "scales", "quats", "sh")],
                 3)
    M = MixedParams.from_params(P)
    del P
    b = BatchTrainer()
    b.set_views(views)
    b.set_tuning(tile, 512)
    colour = torch.empty((b.pixels, 4), device="cuda")
    b.render(M, colour)
    stats = b.check()
    assert stats["degenerate"] == 0
    buf = b.buffers()
    assert buf["sorted_values"] is None   # packed pairs on every workload here
    keys = _device_keys(buf)
    ranges = G.fetch(buf["ranges"], (buf["total_tiles"], 2), np.uint32).astype(np.int64)
    checked = 0
    for v, (proj, W, H) in enumerate(views):
        f = O.set_tile(O.frame_for(G.oracle_projection(O, proj), np.eye(4), W, H, rest_per_colour=15, sh_words=23),
                       tile)
        pr = O.project_params(f, p["means"], p["scales"], p["quats"], p["sh"], p["sh"].shape[1])
        off = v % stride
        want = O.bin_sampled(f, pr, stride, off) if stride > 1 else O.bin_(f, pr)
        tiles_v = f.tilesX * f.tilesY
        t, d, g = _view_pairs(keys, buf, v, tiles_v, stride, off)
        assert t.shape[0] == want["pairs"], (label, v, t.shape[0], want["pairs"])
        np.testing.assert_array_equal(t, want["pair_tiles"].astype(np.int64), err_msg=f"{label} view {v} tiles")
        np.testing.assert_array_equal(g, want["pair_splats"], err_msg=f"{label} view {v} Gaussians")
        np.testing.assert_array_equal(d, pr["keys"][want["pair_splats"]].astype(np.uint64),
                                      err_msg=f"{label} view {v} depth keys")
        # ranges: each sampled tile's length, and its start where the restatement has every tile
        base = int(buf["tile_bases"][v])
        r = ranges[base:base + tiles_v]
        wr = want["ranges"].reshape(-1, 2).astype(np.int64)
        sampled = np.arange(tiles_v) % stride == off
        np.testing.assert_array_equal((r[:, 1] - r[:, 0])[sampled], (wr[:, 1] - wr[:, 0])[sampled],
                                      err_msg=f"{label} view {v} range lengths")
        if stride == 1:
            first = int(r[r[:, 1] > r[:, 0], 0].min()) if (r[:, 1] > r[:, 0]).any() else 0
            live = r[:, 1] > r[:, 0]
            np.testing.assert_array_equal(r[live] - first, wr[live], err_msg=f"{label} view {v} ranges")
        checked += t.shape[0]
        del pr, want
    print(f"{label}: {stats['pairs']} pairs a step, {checked} compared bit for bit (tile {tile}, stride {stride})")
    return stats


@pytest.mark.parametrize("tile", [32, 16])
def test_batched_pairs_at_1_5m_8x1080p_equal_the_restatement(oracle, native, tile):
    p = scenes.params(1_500_000, True, SEED + 1, 3)
    _check_batched_against_oracle(oracle, p, _walk(8, [(1920, 1080)] * 8), tile, 1, f"1.5M 8x1080p tile {tile}")


def test_batched_pairs_at_2_36m_64_mixed_views_equal_the_restatement(oracle, native):
    p = scenes.params(2_360_000, True, SEED + 3, 3)
    sizes = scenes.view_sizes(64, SEED)
    _check_batched_against_oracle(oracle, p, _walk(64, sizes), 32, 4, "2.36M 64 mixed views")


def test_batched_pairs_at_50m_8x4k_sampled_equal_the_restatement(oracle, native):
    """The 50M workload's pairs take the packed form with the depth exponent renumbered;
    every 97th tile of each view is compared whole."""
    p = scenes.params(50_000_000, True, SEED + 4, 3)
    stats = _check_batched_against_oracle(oracle, p, _walk(8, [(3840, 2160)] * 8), 32, 97, "50M 8x4K")
    assert stats["pairs"] > 2_000_000_000
