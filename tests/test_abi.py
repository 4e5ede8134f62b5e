"""The C ABI without a GPU: the library builds and loads, exports every symbol
include/*.h declares, and its host-only entry points (camera, projection,
settings) agree with the CPU restatement. No kernel is launched here.
"""
import ctypes as C
import glob
import os
import re

import numpy as np
import pytest

from tests.conftest import ROOT, gpu_available


def _declared() -> set[str]:
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(ath_[a-z0-9_]+)\s*\(", text))
    return names


def test_library_exports_every_declared_symbol(native):
    lib = native.lib()
    declared = _declared()
    assert declared, "no declarations found"
    for name in declared:
        assert hasattr(lib, name), f"{name} is declared but not exported"
    assert declared == set(native.SIGNATURES), "the ctypes table and the header disagree"
    assert lib.ath_version().decode().count(".") == 2


def test_camera_and_projection_match_the_restatement(native, oracle):
    lib = native.lib()
    for eye, target, w, h in [((1.5, 1.0, 6.0), (0, 0, 0), 250, 190), ((0, 0, 3), (0, 0, 0), 1920, 1080),
                              ((-2.0, 0.5, 5.0), (0.2, -0.1, 0.3), 960, 540)]:
        cam = native.Camera()
        e = np.asarray(eye, np.float64)
        t = np.asarray(target, np.float64)
        assert lib.ath_camera_looking_at(e.ctypes.data_as(C.c_void_p), t.ctypes.data_as(C.c_void_p), None,
                                         C.byref(cam)) == 0
        cam.window_roll = 25.0
        cam.window_translate[0] = 0.2
        cam.window_scale[1] = 1.3
        p = native.Projection()
        assert lib.ath_projection_for(C.byref(cam), w, h, C.byref(p)) == 0
        ocam = oracle.looking_at(eye, target)
        ocam.windowRoll, ocam.windowTranslate[0], ocam.windowScale[1] = 25.0, 0.2, 1.3
        op = oracle.projection_for(ocam, w, h)
        np.testing.assert_allclose(p.world_to_view[:], op.worldToView[:], atol=1e-12)
        for a, b in [("focal_x", "focalX"), ("focal_y", "focalY"), ("centre_x", "centreX"), ("centre_y", "centreY"),
                     ("near_z", "nearZ"), ("far_z", "farZ")]:
            assert abs(getattr(p, a) - getattr(op, b)) <= 1e-12 * max(1.0, abs(getattr(op, b)))


def test_settings_defaults_are_the_references(native):
    s = native.Settings()
    assert native.lib().ath_settings_default(C.byref(s)) == 0
    assert (s.width, s.height, s.antialias, s.antialias_override, s.surfels, s.max_sh_degree) == (1920, 1080, 1, -1, 1, 3)
    assert s.depth_threshold == pytest.approx(0.5) and list(s.background) == [0, 0, 0, 0]
    assert s.matte_threshold == pytest.approx(0.5) and not s.matte_lift and not s.matte and s.matte_hard == 0


def test_argument_errors_come_back_as_status_codes(native):
    lib = native.lib()
    assert lib.ath_camera_looking_at(None, None, None, None) == 3   # InvalidArgument
    assert b"null" in lib.ath_last_error_message()
    assert lib.ath_raster_render(None, None, None, 0, None, None, None, None) == 3
    assert lib.ath_sorter_sort(None, None, None, None, None, 0, 32, None) == 3


@pytest.mark.skipif(gpu_available(), reason="checks the behaviour where no device exists")
def test_without_a_device_create_fails_loudly(native):
    h = C.c_void_p()
    status = native.lib().ath_raster_create(C.byref(h))
    assert status == 6 and not h.value   # DeviceFailure, no handle
    assert len(native.lib().ath_last_error_message()) > 0


def test_the_package_exports_what_bench_and_tests_use():
    import athenea_b200 as A
    for name in A.__all__:
        assert hasattr(A, name), name
    for name in ("BatchTrainer", "MixedParams", "Params", "TileRasterizer", "l2_loss", "pinhole_for_vertical_fov"):
        assert name in A.__all__, name
