"""The committed golden fixtures (tests/golden/, written by make_golden.py):
the CPU restatement must still produce them bit for bit (CPU), and the CUDA
path must produce the same keys, pairs and ranges and the same image within
1e-5 (GPU)."""
import hashlib
import os

import numpy as np
import pytest

from tests.golden import make_golden as MG

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "raster_random3000_250x190.npz")


def _sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, np.float32).tobytes()).hexdigest()


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN)


def test_restatement_reproduces_the_golden_frame(oracle, golden):
    records, packed, proj = MG.scene()
    assert _sha(records) == str(golden["records_sha256"])
    out = MG.render(oracle, packed, proj)
    np.testing.assert_array_equal(out["proj"]["keys"], golden["keys"])
    np.testing.assert_array_equal(out["proj"]["visible"], golden["visible"])
    np.testing.assert_array_equal(out["proj"]["touched"], golden["touched"])
    np.testing.assert_array_equal(out["binned"]["pair_tiles"], golden["pair_tiles"])
    np.testing.assert_array_equal(out["binned"]["pair_splats"], golden["pair_splats"])
    np.testing.assert_array_equal(out["binned"]["ranges"], golden["ranges"])
    assert _sha(out["colour"]) == str(golden["colour_sha256"])
    assert _sha(out["depth"]) == str(golden["depth_sha256"])


@pytest.mark.gpu
def test_cuda_path_reproduces_the_golden_frame(golden):
    import torch
    import athenea_b200 as A
    from tests import gpu_helpers as G
    _, packed, proj = MG.scene()
    raster = A.TileRasterizer.create()
    targets = A.RenderTargets.make(MG.W, MG.H)
    stats = raster.render(proj, [A.SplatInstance(G.upload(packed))], A.RenderSettings(width=MG.W, height=MG.H),
                          targets)
    torch.cuda.synchronize()
    got = G.frame_buffers(raster)
    np.testing.assert_array_equal(got["keys"], golden["keys"])
    assert stats.pairs == golden["pair_splats"].shape[0]
    np.testing.assert_array_equal((got["pair_keys"] >> np.uint64(24)).astype(np.uint32), golden["pair_tiles"])
    np.testing.assert_array_equal(got["pair_splats"], golden["pair_splats"])
    np.testing.assert_array_equal(got["ranges"].reshape(-1), golden["ranges"])
    colour = targets.colour.cpu().numpy()
    depth = targets.depth.cpu().numpy()
    assert np.abs(colour[::MG.STRIDE] - golden["colour_sample"]).max() <= 1e-5
    assert np.abs(depth[::MG.STRIDE] - golden["depth_sample"]).max() <= 1e-5
    print("golden frame bit-identical on the GPU:", _sha(colour) == str(golden["colour_sha256"]))
