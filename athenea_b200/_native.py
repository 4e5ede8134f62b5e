"""ctypes binding of libathenea_b200.so (include/athenea_raster.h).

The structs below mirror the header field for field. Loading fails loudly when
the library is missing: there is no fallback path.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libathenea_b200.so")

OK = 0
STATUS_NAMES = {0: "OK", 1: "Unknown", 2: "NotFound", 3: "InvalidArgument", 4: "Unsupported", 5: "IoFailure",
                6: "DeviceFailure", 7: "ShaderFailure", 8: "PluginFailure", 9: "OutOfMemory", 10: "Cancelled",
                11: "InternalError", 12: "Timeout", 13: "Capacity"}
STATUS_CODES = {name: code for code, name in STATUS_NAMES.items()}


class AtheneaError(RuntimeError):
    """A failure the library reported: `code` is its ath_status (core/Error.h's ErrorCode order, plus 0 = OK)."""

    def __init__(self, code: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {message}")
        self.code = code
        self.name = STATUS_NAMES.get(code, str(code))


class Camera(C.Structure):
    _fields_ = [("camera_to_world", C.c_double * 16), ("orthographic", C.c_int32), ("focal", C.c_double),
                ("haperture", C.c_double), ("near_z", C.c_double), ("far_z", C.c_double),
                ("window_translate", C.c_double * 2), ("window_scale", C.c_double * 2), ("window_roll", C.c_double)]


class Projection(C.Structure):
    _fields_ = [("world_to_view", C.c_double * 16), ("focal_x", C.c_double), ("focal_y", C.c_double),
                ("centre_x", C.c_double), ("centre_y", C.c_double), ("near_z", C.c_double), ("far_z", C.c_double),
                ("orthographic", C.c_int32), ("eye_world", C.c_double * 3)]


class Edit(C.Structure):
    _fields_ = [("active", C.c_int32), ("shape", C.c_uint32), ("mode", C.c_uint32), ("invert", C.c_int32),
                ("centre", C.c_float * 3), ("size", C.c_float * 3), ("tint", C.c_float * 3),
                ("saturation", C.c_float), ("brightness", C.c_float), ("opacity", C.c_float),
                ("min_opacity", C.c_float), ("max_scale", C.c_float)]


class Instance(C.Structure):
    _fields_ = [("positions", C.c_void_p), ("shape", C.c_void_p), ("sh", C.c_void_p), ("count", C.c_uint32),
                ("rest_per_colour", C.c_uint32), ("sh_words", C.c_uint32), ("linear", C.c_int32),
                ("antialiased", C.c_int32), ("object_to_world", C.c_double * 16), ("edit", Edit)]


class Settings(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("antialias", C.c_int32),
                ("antialias_override", C.c_int32), ("made_spread", C.c_float), ("surfels", C.c_int32),
                ("max_sh_degree", C.c_uint32), ("background", C.c_float * 4), ("depth_mode", C.c_uint32),
                ("depth_threshold", C.c_float), ("time_stages", C.c_int32), ("count_splats", C.c_int32),
                ("counters_tag", C.c_uint64), ("contribution_mode", C.c_uint32), ("contribution", C.c_void_p),
                ("final_colour", C.c_void_p), ("crypto_ids", C.c_void_p), ("crypto", C.c_void_p),
                ("under_crypto", C.c_void_p), ("lift_mask", C.c_void_p), ("matte_lift", C.c_void_p),
                ("matte", C.c_void_p), ("matte_hard", C.c_int32), ("matte_threshold", C.c_float),
                ("trace", C.c_void_p)]


class Targets(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("colour", C.c_void_p), ("depth", C.c_void_p),
                ("position", C.c_void_p)]


class FrameStats(C.Structure):
    _fields_ = [("splats", C.c_uint32), ("visible", C.c_uint32), ("pairs", C.c_uint32),
                ("project_ms", C.c_double), ("counts_ms", C.c_double), ("depth_sort_ms", C.c_double),
                ("emit_ms", C.c_double), ("tile_sort_ms", C.c_double), ("blend_ms", C.c_double),
                ("total_ms", C.c_double)]


class CloudCounts(C.Structure):
    _fields_ = [("visible", C.c_uint32), ("pairs", C.c_uint32)]


class SplatCounters(C.Structure):
    _fields_ = [("tag", C.c_uint64), ("slots", C.c_uint32), ("visible", C.c_uint32), ("pairs", C.c_uint32),
                ("max_tiles", C.c_uint32), ("culled", C.c_uint32 * 7), ("cloud_count", C.c_uint32),
                ("clouds", CloudCounts * 64)]


class FrameBuffers(C.Structure):
    _fields_ = [("slots", C.c_uint32), ("pairs", C.c_uint32), ("tiles", C.c_uint32), ("records", C.c_void_p),
                ("rects", C.c_void_p), ("keys", C.c_void_p), ("offsets", C.c_void_p), ("pair_keys", C.c_void_p),
                ("pair_splats", C.c_void_p), ("ranges", C.c_void_p), ("grads", C.c_void_p)]


class Params(C.Structure):
    _fields_ = [("means", C.c_void_p), ("scales", C.c_void_p), ("quats", C.c_void_p), ("sh", C.c_void_p),
                ("count", C.c_uint32), ("sh_degree", C.c_uint32), ("sh_stride", C.c_uint32), ("linear", C.c_int32),
                ("object_to_world", C.c_double * 16)]


class ParamGrads(C.Structure):
    _fields_ = [("means", C.c_void_p), ("scales", C.c_void_p), ("quats", C.c_void_p), ("sh", C.c_void_p)]


class MixedParams(C.Structure):
    _fields_ = [("means", C.c_void_p), ("scales", C.c_void_p), ("quats", C.c_void_p), ("sh_low", C.c_void_p),
                ("sh_high", C.c_void_p), ("sh_scale", C.c_void_p), ("count", C.c_uint32), ("sh_degree", C.c_uint32),
                ("linear", C.c_int32), ("object_to_world", C.c_double * 16)]


class View(C.Structure):
    _fields_ = [("projection", Projection), ("width", C.c_uint32), ("height", C.c_uint32)]


class BatchStats(C.Structure):
    _fields_ = [("pairs", C.c_uint64), ("capacity", C.c_uint64), ("kept", C.c_uint32), ("tile", C.c_uint32),
                ("block_batch", C.c_uint32), ("ms_per_step", C.c_float), ("degenerate", C.c_uint32),
                ("evaluated", C.c_uint64), ("blended", C.c_uint64), ("adjoint_visited", C.c_uint64),
                ("adjoint_live", C.c_uint64), ("warp_visits_forward", C.c_uint64),
                ("warp_visits_adjoint", C.c_uint64), ("warp_visits_adjoint_summed", C.c_uint64),
                ("records_staged", C.c_uint64)]


class BatchBuffers(C.Structure):
    _fields_ = [("pairs", C.c_uint64), ("key_shift", C.c_uint32), ("slot_bits", C.c_uint32),
                ("total_tiles", C.c_uint32), ("views", C.c_uint32), ("sorted_pairs", C.c_void_p),
                ("ranges", C.c_void_p), ("sorted_values", C.c_void_p), ("tile_bases", C.POINTER(C.c_uint32)),
                ("depth_bits", C.c_uint32), ("exp_base", C.c_uint32)]


class Encoding(C.Structure):
    _fields_ = [(n, C.c_uint32) for n in ("stride", "x", "y", "z", "opacity", "scale0", "scale1", "scale2", "rot_w",
                                          "rot_x", "rot_y", "rot_z", "dc0", "dc1", "dc2", "rest_base",
                                          "file_per_colour", "keep_per_colour")]


# Every symbol include/athenea_raster.h declares, with its ctypes signature.
_P = C.c_void_p
SIGNATURES = {
    "ath_camera_looking_at": (C.c_int32, [_P, _P, _P, C.POINTER(Camera)]),
    "ath_camera_default": (C.c_int32, [C.POINTER(Camera)]),
    "ath_projection_for": (C.c_int32, [C.POINTER(Camera), C.c_uint32, C.c_uint32, C.POINTER(Projection)]),
    "ath_settings_default": (C.c_int32, [C.POINTER(Settings)]),
    "ath_raster_create": (C.c_int32, [C.POINTER(C.c_void_p)]),
    "ath_raster_destroy": (None, [_P]),
    "ath_raster_release_scratch": (C.c_int32, [_P]),
    "ath_raster_render": (C.c_int32, [_P, C.POINTER(Projection), _P, C.c_uint32, C.POINTER(Settings),
                                      C.POINTER(Targets), C.POINTER(FrameStats), _P]),
    "ath_raster_latest_counters": (C.c_int32, [_P, C.POINTER(SplatCounters)]),
    "ath_raster_check": (C.c_int32, [_P, C.POINTER(FrameStats)]),
    "ath_raster_render_over": (C.c_int32, [_P, C.POINTER(Projection), _P, C.c_uint32, C.POINTER(Settings),
                                           C.POINTER(Targets), C.POINTER(Targets), C.POINTER(FrameStats), _P]),
    "ath_raster_render_params": (C.c_int32, [_P, C.POINTER(Projection), C.POINTER(Params), C.POINTER(Settings),
                                             C.POINTER(Targets), C.POINTER(FrameStats), _P]),
    "ath_raster_backward": (C.c_int32, [_P, _P, _P, C.POINTER(ParamGrads), _P]),
    "ath_l2_loss": (C.c_int32, [_P, _P, C.c_uint32, _P, _P, _P]),
    "ath_params_to_mixed": (C.c_int32, [C.POINTER(Params), _P, _P, _P, _P]),
    "ath_batch_create": (C.c_int32, [C.POINTER(C.c_void_p)]),
    "ath_batch_destroy": (None, [_P]),
    "ath_batch_set_views": (C.c_int32, [_P, _P, C.c_uint32, C.POINTER(Settings)]),
    "ath_batch_set_tuning": (C.c_int32, [_P, C.c_uint32, C.c_uint32]),
    "ath_batch_pixels": (C.c_int32, [_P, C.POINTER(C.c_uint32)]),
    "ath_batch_train_step": (C.c_int32, [_P, C.POINTER(MixedParams), _P, _P, _P, C.POINTER(ParamGrads), _P]),
    "ath_batch_train_step_after": (C.c_int32, [_P, C.POINTER(MixedParams), _P, _P, _P, _P, C.POINTER(ParamGrads),
                                               _P]),
    "ath_batch_render": (C.c_int32, [_P, C.POINTER(MixedParams), _P, _P, _P]),
    "ath_batch_check": (C.c_int32, [_P, C.POINTER(BatchStats), _P]),
    "ath_batch_buffers_of": (C.c_int32, [_P, C.POINTER(BatchBuffers), _P]),
    "ath_batch_set_key_mode": (C.c_int32, [_P, C.c_uint32]),
    "ath_batch_set_buckets": (C.c_int32, [_P, C.c_uint32, C.c_uint32, _P, _P]),
    "ath_gradient_bucket": (C.c_int32, [C.c_uint32, C.c_uint32, C.c_uint32, C.POINTER(C.c_uint32),
                                        C.POINTER(C.c_uint32)]),
    "ath_set_memory_budget": (C.c_int32, [C.c_uint64]),
    "ath_memory_held": (C.c_int32, [C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    "ath_check_bounded_wait": (C.c_int32, [C.c_uint32, C.c_uint32, C.POINTER(C.c_uint32), _P]),
    "ath_measure_peaks": (C.c_int32, [C.c_uint32, C.POINTER(C.c_double), C.POINTER(C.c_double), _P]),
    "ath_ply_read_header": (C.c_int32, [C.c_char_p, C.POINTER(C.c_uint32), C.POINTER(Encoding)]),
    "ath_ply_read": (C.c_int32, [C.c_char_p, _P, C.c_uint64, C.POINTER(C.c_uint32), C.POINTER(Encoding)]),
    "ath_batch_time_stages": (C.c_int32, [_P, C.POINTER(MixedParams), _P, _P, _P, C.POINTER(ParamGrads),
                                          C.POINTER(C.c_float), _P]),
    "ath_batch_tune": (C.c_int32, [_P, C.POINTER(MixedParams), _P, _P, _P, C.POINTER(ParamGrads), C.c_uint32,
                                   C.POINTER(BatchStats), _P]),
    "ath_raster_frame_buffers": (C.c_int32, [_P, C.POINTER(FrameBuffers)]),
    "ath_sorter_create": (C.c_int32, [C.POINTER(C.c_void_p)]),
    "ath_sorter_destroy": (None, [_P]),
    "ath_sorter_sort": (C.c_int32, [_P, _P, _P, _P, _P, C.c_uint32, C.c_uint32, _P]),
    "ath_sorter_check": (C.c_int32, [_P]),
    "ath_sort_pairs_static": (C.c_int32, [_P, _P, _P, _P, C.c_uint32, C.c_uint32, _P]),
    "ath_sort_pairs_static_status": (C.c_int32, [_P]),
    "ath_decode_records": (C.c_int32, [_P, C.c_uint32, C.POINTER(Encoding), _P, _P, _P, C.POINTER(C.c_uint32), _P]),
    "ath_last_error_message": (C.c_char_p, []),
    "ath_version": (C.c_char_p, []),
}

_lib = None


def lib():
    """The loaded library; raises when it was not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m athenea_b200._build` "
                              "(or __graft_entry__.build()); there is no CPU fallback")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status: int) -> None:
    if status != OK:
        raise AtheneaError(status, lib().ath_last_error_message().decode())
