"""The multi-GPU path's host logic on CPU ranks (gloo, world size 2): views
sharded across ranks, each rank's per-Gaussian gradients from its own views,
summed over ranks by GradientBuffer.allreduce, must equal one process's sum
over every view. The per-view gradient is the oracle's colour gradient (the
reference's contributionMode 4 sums, exact form), so no GPU is needed."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

VIEWS = 5
COUNT = 3000
W, H = 96, 64


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _view_gradient(O, p, v):
    """dL/d(colour) a Gaussian for view v of the scene: mean L2 against a seeded target."""
    import athenea_b200 as A
    from athenea_b200 import scenes
    from tests import gpu_helpers as G
    eye = scenes.circle_eye(v, VIEWS * 2, 3.0, 0.3)
    cam = A.pinhole_for_vertical_fov(eye, (0, 0, 0), W, H, 60.0)
    proj = G.oracle_projection(O, cam.projection_for(W, H))
    f = O.frame_for(proj, np.eye(4), W, H, rest_per_colour=15, sh_words=23)
    pr = O.project_params(f, p["means"], p["scales"], p["quats"], p["sh"], p["sh"].shape[1])
    binned = O.bin_(f, pr)
    out = O.blend(f, binned, pr)
    target = np.random.default_rng(100 + v).uniform(0, 1, size=(W * H, 3)).astype(np.float32)
    dl = np.zeros((W * H, 4), np.float32)
    dl[:, :3] = 2.0 * (out["colour"][:, :3] - target) / (3.0 * W * H)
    return O.colour_gradient_exact(f, binned, pr, dl)


def _scene():
    from athenea_b200 import scenes
    return scenes.params(COUNT, True, 77, 3)


def _rank_buckets(rank, world, port, out_path, buckets):
    """As _rank, with the gradients in buckets, each summed over ranks by its own all-reduce,
    the buckets' all-reduces in flight together (as a step posts them while it runs)."""
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        import athenea_b200 as A
        from oracle import oracle as O
        p = _scene()
        buf = A.BucketedGradients(COUNT, buckets, 48, 3, device="cpu")
        for v in A.shard_views(VIEWS, rank, world):
            g = torch.from_numpy(_view_gradient(O, p, v).astype(np.float32))
            for (first, n), P in zip(buf.ranges, buf.params):
                P.sh[:, :3] += g[first:first + n]
        works = [buf.allreduce_bucket(k, async_op=True) for k in range(buckets)]
        for w in works:
            w.wait()
        if rank == 0:
            np.save(out_path, buf.gather().sh.numpy())
    finally:
        dist.destroy_process_group()


def _rank(rank, world, port, out_path):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        import athenea_b200 as A
        from oracle import oracle as O
        p = _scene()
        buf = A.GradientBuffer(COUNT, 48, 3, device="cpu")
        for v in A.shard_views(VIEWS, rank, world):
            g = _view_gradient(O, p, v)
            buf.params.sh[:, :3] += torch.from_numpy(g.astype(np.float32))
        buf.allreduce()
        if rank == 0:
            np.save(out_path, buf.flat.numpy())
    finally:
        dist.destroy_process_group()


def test_shard_views_covers_every_view_once():
    import athenea_b200 as A
    for views in (1, 5, 8, 64):
        for world in (1, 2, 3, 8):
            got = [list(A.shard_views(views, r, world)) for r in range(world)]
            assert sum(got, []) == list(range(views))
            sizes = [len(s) for s in got]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        A.shard_views(4, 2, 2)


def test_gradients_summed_over_two_ranks_equal_one_process(oracle, tmp_path):
    out_path = str(tmp_path / "flat.npy")
    mp.start_processes(_rank, args=(2, _free_port(), out_path), nprocs=2, join=True, start_method="spawn")
    got = np.load(out_path)
    import athenea_b200 as A
    p = _scene()
    want = A.GradientBuffer(COUNT, 48, 3, device="cpu")
    for v in range(VIEWS):
        want.params.sh[:, :3] += torch.from_numpy(_view_gradient(oracle, p, v).astype(np.float32))
    assert np.abs(want.flat.numpy()).max() > 0
    np.testing.assert_allclose(got, want.flat.numpy(), rtol=1e-6, atol=1e-9)


def test_gradient_buckets_cover_every_gaussian_once():
    import athenea_b200 as A
    for count in (0, 1, 127, 128, 129, 3000, 1_500_000, 50_000_000):
        for buckets in (1, 2, 3, 4, 7, 16):
            ranges = [A.gradient_bucket(count, buckets, k) for k in range(buckets)]
            at = 0
            for first, n in ranges:
                assert first == at and (n % 128 == 0 or first + n == count)
                at += n
            assert at == count
            blocks = [(n + 127) // 128 for _, n in ranges]   # whole blocks of the projection adjoint
            assert max(blocks) - min(blocks) <= 1
    with pytest.raises(A.AtheneaError):
        A.gradient_bucket(10, 2, 2)


def test_bucketed_gradients_summed_over_two_ranks_equal_one_process(oracle, tmp_path):
    out_path = str(tmp_path / "sh.npy")
    buckets = 3
    mp.start_processes(_rank_buckets, args=(2, _free_port(), out_path, buckets), nprocs=2, join=True,
                       start_method="spawn")
    got = np.load(out_path)
    p = _scene()
    want = np.zeros((COUNT, 48), np.float32)
    for v in range(VIEWS):
        want[:, :3] += _view_gradient(oracle, p, v).astype(np.float32)
    assert np.abs(want).max() > 0
    np.testing.assert_allclose(got, want, rtol=1e-6, atol=1e-9)
