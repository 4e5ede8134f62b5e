"""Failure detection without a GPU fault: the device-memory budget (the
reference's ATHENEA_GPU_BUDGET, modules/gpu/src/Device.cpp:434-449) turning an
allocation into OutOfMemory on the host side, and the library's bounded
device-side wait running out on a flag nothing sets, with the context usable
after both."""
import numpy as np
import pytest
import torch

import athenea_b200 as A
from tests.fixtures import ENC_BUILDER, CloudBuilder, product_encoding

pytestmark = pytest.mark.gpu


def _cloud():
    b = CloudBuilder()
    rng = np.random.default_rng(5)
    for _ in range(200):
        x, y, z = rng.uniform(-1, 1, 3)
        b.add(x, y, z, 0.8, 0.05, 0.05, 0.05, (1, 0, 0, 0), tuple(rng.uniform(0, 1, 3)))
    recs = torch.from_numpy(b.records().reshape(-1)).cuda()
    return A.CloudLoader.upload(recs, product_encoding(ENC_BUILDER), 3)


def _frame(raster, cloud, W=256, H=192):
    s = A.RenderSettings(width=W, height=H)
    t = A.RenderTargets.make(W, H)
    raster.render(A.Camera.looking_at((0.0, 0.0, 4.0), (0, 0, 0)), [A.SplatInstance(cloud)], s, t)
    torch.cuda.synchronize()
    return t.colour.cpu().numpy()


def test_a_budget_turns_scratch_into_out_of_memory_and_release_gives_it_back(native):
    cloud = _cloud()
    want = _frame(A.TileRasterizer.create(), cloud)
    raster = A.TileRasterizer.create()
    import gc
    gc.collect()                                    # what earlier tests left is freed now, not mid-test
    held_before, _ = A.memory_held()
    try:
        A.set_memory_budget(1)                      # room for no new buffer, whatever is held
        assert A.memory_held()[1] == 1
        with pytest.raises(A.AtheneaError) as e:
            _frame(raster, cloud)
        assert e.value.code == 9                    # OutOfMemory
        A.set_memory_budget(0)
        got = _frame(raster, cloud)                 # the same rasteriser, usable again
        np.testing.assert_array_equal(got, want)
        held_after, budget = A.memory_held()
        assert budget == 0 and held_after > 0
        raster.release_scratch()
        assert A.memory_held()[0] < held_after
    finally:
        A.set_memory_budget(0)


def test_a_wait_on_a_flag_nothing_sets_gives_up_with_timeout(native):
    with pytest.raises(A.AtheneaError) as e:
        A.check_bounded_wait(0, 1000)
    assert e.value.code == 12                       # Timeout
    assert A.check_bounded_wait(1, 1000) == 0       # a set flag: no spin at all
    with pytest.raises(A.AtheneaError) as e:
        A.check_bounded_wait(1, 0)                  # a limit of none is refused
    assert e.value.code == 3
    # the context is still usable: a frame renders after the timeout
    assert _frame(A.TileRasterizer.create(), _cloud())[:, 3].max() > 0
