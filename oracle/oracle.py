"""ORACLE -- TEST INFRASTRUCTURE ONLY.

ctypes access to the CPU restatement of athenea's splat raster path
(oracle.cpp, oracle_f64.cpp). Imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, never by the product package.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")


def build() -> str:
    """Compiles liboracle.so with the committed Makefile (returns its path)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


class Edit(C.Structure):
    _fields_ = [("active", C.c_uint32), ("shape", C.c_uint32), ("mode", C.c_uint32), ("invert", C.c_uint32),
                ("centre", C.c_float * 3), ("size", C.c_float * 3), ("tint", C.c_float * 3),
                ("saturation", C.c_float), ("brightness", C.c_float), ("opacity", C.c_float),
                ("minOpacity", C.c_float), ("maxScale", C.c_float)]


class Frame(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("tilesX", C.c_uint32), ("tilesY", C.c_uint32),
                ("focalX", C.c_float), ("focalY", C.c_float), ("centreX", C.c_float), ("centreY", C.c_float),
                ("nearZ", C.c_float), ("farZ", C.c_float), ("orthographic", C.c_uint32), ("antialias", C.c_uint32),
                ("paidAt", C.c_float), ("surfels", C.c_uint32), ("m", C.c_float * 12), ("eye", C.c_float * 3),
                ("restPerColour", C.c_uint32), ("shWords", C.c_uint32), ("shLimit", C.c_uint32),
                ("linearCloud", C.c_uint32), ("depthMode", C.c_uint32), ("depthThreshold", C.c_float),
                ("bg", C.c_float * 4), ("edit", Edit), ("tile", C.c_uint32)]


class Encoding(C.Structure):
    _fields_ = [(n, C.c_uint32) for n in ("stride", "x", "y", "z", "opacity", "scale0", "scale1", "scale2", "rotW",
                                          "rotX", "rotY", "rotZ", "dc0", "dc1", "dc2", "restBase", "filePerColour",
                                          "keepPerColour")]


class Camera(C.Structure):
    _fields_ = [("cameraToWorld", C.c_double * 16), ("orthographic", C.c_uint32), ("focal", C.c_double),
                ("haperture", C.c_double), ("nearZ", C.c_double), ("farZ", C.c_double),
                ("windowTranslate", C.c_double * 2), ("windowScale", C.c_double * 2), ("windowRoll", C.c_double)]


class Projection(C.Structure):
    _fields_ = [("worldToView", C.c_double * 16), ("focalX", C.c_double), ("focalY", C.c_double),
                ("centreX", C.c_double), ("centreY", C.c_double), ("nearZ", C.c_double), ("farZ", C.c_double),
                ("orthographic", C.c_uint32), ("eyeWorld", C.c_double * 3)]


class Frame64(C.Structure):
    _fields_ = [("focalX", C.c_double), ("focalY", C.c_double), ("centreX", C.c_double), ("centreY", C.c_double),
                ("nearZ", C.c_double), ("farZ", C.c_double), ("width", C.c_uint32), ("height", C.c_uint32),
                ("orthographic", C.c_uint32), ("antialias", C.c_uint32), ("paidAt", C.c_double),
                ("m", C.c_double * 12), ("eye", C.c_double * 3), ("restPerColour", C.c_uint32),
                ("shWords", C.c_uint32), ("shLimit", C.c_uint32), ("linearCloud", C.c_uint32),
                ("bg", C.c_double * 4)]


_P = C.c_void_p
_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        L.orc_exp.restype = C.c_float
        L.orc_exp.argtypes = [C.c_float]
        L.orc_log.restype = C.c_float
        L.orc_log.argtypes = [C.c_float]
        L.orc_pow.restype = C.c_float
        L.orc_pow.argtypes = [C.c_float, C.c_float]
        L.orc_f32_to_f16.restype = C.c_uint16
        L.orc_f32_to_f16.argtypes = [C.c_float]
        L.orc_f16_to_f32.restype = C.c_float
        L.orc_f16_to_f32.argtypes = [C.c_uint16]
        L.orc_encode_quaternion.restype = C.c_uint32
        L.orc_encode_quaternion.argtypes = [_P]
        L.orc_decode_quaternion.argtypes = [C.c_uint32, _P]
        L.orc_decode.restype = C.c_uint32
        L.orc_decode.argtypes = [_P, C.c_uint32, C.POINTER(Encoding), _P, _P, _P, _P]
        L.orc_camera_looking_at.argtypes = [_P, _P, _P, C.POINTER(Camera)]
        L.orc_projection_for.argtypes = [C.POINTER(Camera), C.c_uint32, C.c_uint32, C.POINTER(Projection)]
        L.orc_frame_for.argtypes = [C.POINTER(Projection), _P, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int32,
                                    C.c_float, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, _P,
                                    C.c_uint32, C.c_float, C.POINTER(Edit), C.POINTER(Frame)]
        L.orc_project.argtypes = [C.POINTER(Frame), C.c_uint32, C.c_uint32, _P, _P, _P, _P, _P, _P, _P, _P, C.c_int]
        L.orc_project_params.argtypes = [C.POINTER(Frame), C.c_uint32, C.c_uint32, _P, _P, _P, _P, C.c_uint32,
                                         _P, _P, _P, _P, _P, C.c_int]
        L.orc_colour_gradient_exact.argtypes = [C.POINTER(Frame), _P, _P, _P, _P, _P]
        L.orc_fd_gradients_f64.argtypes = [C.POINTER(Frame64), C.c_uint32, _P, _P, _P, _P, _P, C.c_uint32, _P, _P,
                                           C.c_uint32, C.c_double, _P, C.POINTER(C.c_double), C.c_int]
        L.orc_bin.restype = C.c_uint64
        L.orc_bin.argtypes = [C.POINTER(Frame), C.c_uint32, _P, _P, _P, _P, _P, _P, _P, _P, _P]
        L.orc_bin_sampled.restype = C.c_uint64
        L.orc_bin_sampled.argtypes = [C.POINTER(Frame), C.c_uint32, _P, _P, _P, _P, _P, _P, _P, _P, C.c_uint32,
                                      C.c_uint32]
        L.orc_frame_set_tile.argtypes = [C.POINTER(Frame), C.c_uint32]
        L.orc_blend.restype = C.c_uint64
        L.orc_blend.argtypes = [C.POINTER(Frame), _P, _P, _P, _P, _P, _P, _P, C.c_int]
        L.orc_colour_gradient.argtypes = [C.POINTER(Frame), _P, _P, _P, _P, _P]
        L.orc_contribution_weight.argtypes = [C.POINTER(Frame), _P, _P, _P, _P]
        L.orc_contribution_change.argtypes = [C.POINTER(Frame), _P, _P, _P, _P, _P]
        L.orc_contribution_lift.argtypes = [C.POINTER(Frame), _P, _P, _P, _P, _P]
        L.orc_matte_lift.argtypes = [C.POINTER(Frame), _P, _P, _P, _P, C.c_uint32, C.c_float, _P]
        L.orc_trace.argtypes = [C.POINTER(Frame), _P, _P, _P, _P]
        L.orc_position.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, C.c_float, C.c_float, C.c_float, C.c_float,
                                   _P, _P, _P]
        L.orc_frame64_from.argtypes = [C.POINTER(Projection), _P, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                       C.c_uint32, C.c_uint32, C.c_uint32, _P, C.POINTER(Frame64)]
        L.orc_render_f64.argtypes = [C.POINTER(Frame64), C.c_uint32, _P, _P, _P, _P, _P, _P, C.c_double,
                                     C.c_uint32, C.c_uint32, C.c_int]
        L.orc_render_params_f64.argtypes = [C.POINTER(Frame64), C.c_uint32, _P, _P, _P, _P, _P, C.c_uint32,
                                            _P, _P, C.c_int]
        L.orc_blend_over.argtypes = [C.POINTER(Frame), _P, _P, _P, _P, _P, _P, _P, C.c_int]
        L.orc_blend_matte.argtypes = [C.POINTER(Frame), _P, _P, _P, _P, _P, _P, _P, C.c_int]
        L.orc_render_params_sampled_f64.argtypes = [C.POINTER(Frame64), C.c_uint32, _P, _P, _P, _P, C.c_uint32,
                                                    C.c_uint32, _P, _P, _P, C.c_double, C.c_uint32, C.c_uint32,
                                                    C.c_int]
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"], "oracle buffers must be contiguous"
    return a.ctypes.data_as(C.c_void_p)


def _mat16(m) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(m, dtype=np.float64).reshape(16))


# ---- scalar helpers --------------------------------------------------------
def exp(x: float) -> float:
    return lib().orc_exp(float(x))


def log(x: float) -> float:
    return lib().orc_log(float(x))


def pow_(x: float, y: float) -> float:
    return lib().orc_pow(float(x), float(y))


def f32_to_f16(v: float) -> int:
    return lib().orc_f32_to_f16(float(v))


def f16_to_f32(h: int) -> float:
    return lib().orc_f16_to_f32(int(h))


def encode_quaternion(q_xyzw) -> int:
    q = np.ascontiguousarray(np.asarray(q_xyzw, dtype=np.float32))
    return lib().orc_encode_quaternion(_ptr(q))


def decode_quaternion(word: int) -> np.ndarray:
    q = np.zeros(4, dtype=np.float32)
    lib().orc_decode_quaternion(int(word), _ptr(q))
    return q


# ---- decode ----------------------------------------------------------------
def decode(records: np.ndarray, enc: dict, keep_per_colour: int):
    """3DGS float records -> packed (positions, shape, sh, origin), valid ones only."""
    records = np.ascontiguousarray(records, dtype=np.float32)
    stride = enc["stride"]
    count = records.size // stride
    e = Encoding(stride=stride, keepPerColour=keep_per_colour,
                 **{k: enc[k] for k in ("x", "y", "z", "opacity", "scale0", "scale1", "scale2", "rotW", "rotX",
                                        "rotY", "rotZ", "dc0", "dc1", "dc2", "restBase", "filePerColour")})
    sh_words = 1 if keep_per_colour == 0 else (keep_per_colour * 3 + 1) // 2
    positions = np.zeros((max(count, 1), 4), np.float32)
    shape = np.zeros((max(count, 1), 4), np.uint32)
    sh = np.zeros((max(count, 1), sh_words), np.uint32)
    origin = np.zeros(max(count, 1), np.uint32)
    kept = lib().orc_decode(_ptr(records), count, C.byref(e), _ptr(positions), _ptr(shape), _ptr(sh), _ptr(origin))
    return positions[:kept].copy(), shape[:kept].copy(), sh[:kept].copy(), origin[:kept].copy(), sh_words


# ---- camera ----------------------------------------------------------------
def looking_at(eye, target, up=(0.0, 1.0, 0.0)) -> Camera:
    cam = Camera()
    e = np.asarray(eye, np.float64)
    t = np.asarray(target, np.float64)
    u = np.asarray(up, np.float64)
    lib().orc_camera_looking_at(_ptr(e), _ptr(t), _ptr(u), C.byref(cam))
    return cam


def default_camera() -> Camera:
    cam = Camera()
    for i in range(4):
        cam.cameraToWorld[i * 5] = 1.0
    cam.focal, cam.haperture, cam.nearZ, cam.farZ = 50.0, 24.576, 0.1, 10000.0
    cam.windowScale[0] = cam.windowScale[1] = 1.0
    return cam


def projection_for(cam: Camera, width: int, height: int) -> Projection:
    p = Projection()
    lib().orc_projection_for(C.byref(cam), width, height, C.byref(p))
    return p


def frame_for(proj: Projection, object_to_world, width, height, *, antialias=1, antialiased=-1, made_spread=0.0,
              surfels=1, max_sh_degree=3, rest_per_colour=15, sh_words=23, linear=0, bg=(0, 0, 0, 0),
              depth_mode=0, depth_threshold=0.5, edit: Edit | None = None) -> Frame:
    f = Frame()
    bgv = np.asarray(bg, np.float32)
    lib().orc_frame_for(C.byref(proj), _ptr(_mat16(object_to_world)), width, height, antialias, antialiased,
                        made_spread, surfels, max_sh_degree, rest_per_colour, sh_words, linear, _ptr(bgv),
                        depth_mode, depth_threshold, C.byref(edit) if edit is not None else None, C.byref(f))
    return f


# ---- the frame -------------------------------------------------------------
def project(f: Frame, positions, shape, sh, slots=None, base=0, out=None, threads=0):
    n = positions.shape[0]
    slots = slots or (base + n)
    if out is None:
        out = dict(records=np.zeros((slots, 12), np.float32), rects=np.zeros((slots, 4), np.uint32),
                   touched=np.zeros(slots, np.uint32), keys=np.zeros(slots, np.uint32),
                   visible=np.zeros(slots, np.uint32))
    if n:
        lib().orc_project(C.byref(f), n, base, _ptr(np.ascontiguousarray(positions, np.float32)),
                          _ptr(np.ascontiguousarray(shape, np.uint32)), _ptr(np.ascontiguousarray(sh, np.uint32)),
                          _ptr(out["records"]), _ptr(out["rects"]), _ptr(out["touched"]), _ptr(out["keys"]),
                          _ptr(out["visible"]), threads)
    return out


def project_params(f: Frame, means, scales, quats, sh, sh_stride, out=None, base=0, threads=0):
    """The projection from FP32 training parameters (float4 means/scales/quats, sh rows)."""
    n = means.shape[0]
    slots = base + n
    if out is None:
        out = dict(records=np.zeros((slots, 12), np.float32), rects=np.zeros((slots, 4), np.uint32),
                   touched=np.zeros(slots, np.uint32), keys=np.zeros(slots, np.uint32),
                   visible=np.zeros(slots, np.uint32))
    if n:
        lib().orc_project_params(C.byref(f), n, base, _ptr(np.ascontiguousarray(means, np.float32)),
                                 _ptr(np.ascontiguousarray(scales, np.float32)),
                                 _ptr(np.ascontiguousarray(quats, np.float32)),
                                 _ptr(np.ascontiguousarray(sh, np.float32)), sh_stride, _ptr(out["records"]),
                                 _ptr(out["rects"]), _ptr(out["touched"]), _ptr(out["keys"]), _ptr(out["visible"]),
                                 threads)
    return out


def colour_gradient_exact(f: Frame, binned: dict, proj: dict, dl_dpixel: np.ndarray) -> np.ndarray:
    """Per slot, sum over pixels of weight * dL/dpixel (rgb), in double."""
    slots = proj["touched"].shape[0]
    out = np.zeros((slots, 3), np.float64)
    ps = binned["pair_splats"] if binned["pairs"] else np.zeros(1, np.uint32)
    lib().orc_colour_gradient_exact(C.byref(f), _ptr(binned["ranges"]), _ptr(ps), _ptr(proj["records"]),
                                    _ptr(np.ascontiguousarray(dl_dpixel, np.float32)), _ptr(out))
    return out


def fd_gradients_f64(f64: Frame64, means, log_scales, quats, logits, shs, sh_degree, target, which, eps,
                     threads=0):
    """FP64 central differences of the mean-L2 loss (decisions frozen at the base), 59 a Gaussian:
    means xyz, logit, log scales xyz, quat wxyz, sh[48]. Returns (grads (K, 59), loss)."""
    which = np.ascontiguousarray(which, np.uint32)
    out = np.zeros((which.shape[0], 59), np.float64)
    loss = C.c_double(0.0)
    lib().orc_fd_gradients_f64(C.byref(f64), means.shape[0], _ptr(np.ascontiguousarray(means, np.float64)),
                               _ptr(np.ascontiguousarray(log_scales, np.float64)),
                               _ptr(np.ascontiguousarray(quats, np.float64)),
                               _ptr(np.ascontiguousarray(logits, np.float64)),
                               _ptr(np.ascontiguousarray(shs, np.float64)), sh_degree,
                               _ptr(np.ascontiguousarray(target, np.float32)), _ptr(which), which.shape[0], eps,
                               _ptr(out), C.byref(loss), threads)
    return out, loss.value


def bin_(f: Frame, proj: dict):
    slots = proj["touched"].shape[0]
    pairs = int(proj["touched"].astype(np.uint64).sum())
    tiles = f.tilesX * f.tilesY
    pair_tiles = np.zeros(max(pairs, 1), np.uint32)
    pair_splats = np.zeros(max(pairs, 1), np.uint32)
    ranges = np.zeros(2 * tiles, np.uint32)
    visible = C.c_uint32(0)
    n = lib().orc_bin(C.byref(f), slots, _ptr(proj["records"]), _ptr(proj["rects"]), _ptr(proj["touched"]),
                      _ptr(proj["keys"]), _ptr(proj["visible"]), _ptr(pair_tiles), _ptr(pair_splats), _ptr(ranges),
                      C.byref(visible))
    assert n == pairs
    return dict(pair_tiles=pair_tiles[:pairs], pair_splats=pair_splats[:pairs], ranges=ranges, pairs=pairs,
                visible=visible.value)


def set_tile(f: Frame, tile: int) -> Frame:
    """The frame at tile size `tile` (orc_frame_set_tile): rects, the tile test and tiles follow it."""
    lib().orc_frame_set_tile(C.byref(f), tile)
    return f


def bin_sampled(f: Frame, proj: dict, tile_stride: int, tile_offset: int = 0):
    """bin_ keeping only the pairs of tiles t with t % tile_stride == tile_offset."""
    slots = proj["touched"].shape[0]
    tiles = f.tilesX * f.tilesY
    args = (C.byref(f), slots, _ptr(proj["records"]), _ptr(proj["rects"]), _ptr(proj["touched"]), _ptr(proj["keys"]),
            _ptr(proj["visible"]))
    pairs = lib().orc_bin_sampled(*args, None, None, None, tile_stride, tile_offset)
    pair_tiles = np.zeros(max(pairs, 1), np.uint32)
    pair_splats = np.zeros(max(pairs, 1), np.uint32)
    ranges = np.zeros(2 * tiles, np.uint32)
    n = lib().orc_bin_sampled(*args, _ptr(pair_tiles), _ptr(pair_splats), _ptr(ranges), tile_stride, tile_offset)
    assert n == pairs
    return dict(pair_tiles=pair_tiles[:pairs], pair_splats=pair_splats[:pairs], ranges=ranges, pairs=pairs)


def blend(f: Frame, binned: dict, proj: dict, threads=0):
    w, h = f.width, f.height
    colour = np.zeros((h * w, 4), np.float32)
    depth = np.zeros(h * w, np.float32)
    final_t = np.zeros(h * w, np.float32)
    last = np.zeros(h * w, np.uint32)
    ps = binned["pair_splats"] if binned["pairs"] else np.zeros(1, np.uint32)
    ev = lib().orc_blend(C.byref(f), _ptr(binned["ranges"]), _ptr(ps), _ptr(proj["records"]), _ptr(colour),
                         _ptr(depth), _ptr(final_t), _ptr(last), threads)
    return dict(colour=colour, depth=depth, final_t=final_t, last=last, evaluated=int(ev))


def blend_over(f: Frame, binned: dict, proj: dict, under_colour: np.ndarray, under_depth: np.ndarray, threads=0):
    """The blend over an opaque under layer (float4 colour, float depth a pixel; depth 0 = none)."""
    w, h = f.width, f.height
    colour = np.zeros((h * w, 4), np.float32)
    depth = np.zeros(h * w, np.float32)
    ps = binned["pair_splats"] if binned["pairs"] else np.zeros(1, np.uint32)
    lib().orc_blend_over(C.byref(f), _ptr(binned["ranges"]), _ptr(ps), _ptr(proj["records"]),
                         _ptr(np.ascontiguousarray(under_colour, np.float32)),
                         _ptr(np.ascontiguousarray(under_depth, np.float32)), _ptr(colour), _ptr(depth), threads)
    return dict(colour=colour, depth=depth)


def blend_matte(f: Frame, binned: dict, proj: dict, crypto_ids: np.ndarray, under_depth=None, under_crypto=None,
                threads=0) -> np.ndarray:
    """The Cryptomatte layers: (3, pixels, 4) float32 (id bits, coverage, id bits, coverage)."""
    pixels = f.width * f.height
    out = np.zeros((3, pixels, 4), np.float32)
    ps = binned["pair_splats"] if binned["pairs"] else np.zeros(1, np.uint32)
    ud = None if under_depth is None else np.ascontiguousarray(under_depth, np.float32)
    uc = None if under_crypto is None else np.ascontiguousarray(under_crypto, np.uint32)
    lib().orc_blend_matte(C.byref(f), _ptr(binned["ranges"]), _ptr(ps), _ptr(proj["records"]),
                          _ptr(np.ascontiguousarray(crypto_ids, np.uint32)), _ptr(ud) if ud is not None else None,
                          _ptr(uc) if uc is not None else None, _ptr(out), threads)
    return out


def colour_gradient(f: Frame, binned: dict, proj: dict, dl_dpixel: np.ndarray) -> np.ndarray:
    slots = proj["touched"].shape[0]
    out = np.zeros((slots, 4), np.int32)
    d = np.ascontiguousarray(dl_dpixel, np.float32)
    ps = binned["pair_splats"] if binned["pairs"] else np.zeros(1, np.uint32)
    lib().orc_colour_gradient(C.byref(f), _ptr(binned["ranges"]), _ptr(ps), _ptr(proj["records"]), _ptr(d),
                              _ptr(out))
    return out


def contribution_weight(f: Frame, binned: dict, proj: dict) -> np.ndarray:
    slots = proj["touched"].shape[0]
    out = np.zeros(slots, np.uint32)
    ps = binned["pair_splats"] if binned["pairs"] else np.zeros(1, np.uint32)
    lib().orc_contribution_weight(C.byref(f), _ptr(binned["ranges"]), _ptr(ps), _ptr(proj["records"]), _ptr(out))
    return out


def contribution_change(f: Frame, binned: dict, proj: dict, whole: np.ndarray) -> np.ndarray:
    """contributionMode 2: (slots, 2) uint32 words, the low and high word of each slot's 64-bit sum."""
    slots = proj["touched"].shape[0]
    out = np.zeros((slots, 2), np.uint32)
    w = np.ascontiguousarray(whole, np.float32)
    ps = binned["pair_splats"] if binned["pairs"] else np.zeros(1, np.uint32)
    lib().orc_contribution_change(C.byref(f), _ptr(binned["ranges"]), _ptr(ps), _ptr(proj["records"]), _ptr(w),
                                  _ptr(out))
    return out


def contribution_lift(f: Frame, binned: dict, proj: dict, mask: np.ndarray) -> np.ndarray:
    """contributionMode 3: (slots, 2) uint32 words, the weight times the mask and the weight, in 1/1024."""
    slots = proj["touched"].shape[0]
    out = np.zeros((slots, 2), np.uint32)
    m = np.ascontiguousarray(mask, np.float32)
    ps = binned["pair_splats"] if binned["pairs"] else np.zeros(1, np.uint32)
    lib().orc_contribution_lift(C.byref(f), _ptr(binned["ranges"]), _ptr(ps), _ptr(proj["records"]), _ptr(m),
                                _ptr(out))
    return out


def matte_lift(f: Frame, binned: dict, proj: dict, lift: np.ndarray, hard: bool = False,
               threshold: float = 0.5) -> np.ndarray:
    """The matte a lift's sums (two uint32 a slot) give each pixel of this frame."""
    out = np.zeros(f.width * f.height, np.float32)
    sums = np.ascontiguousarray(lift, np.uint32)
    ps = binned["pair_splats"] if binned["pairs"] else np.zeros(1, np.uint32)
    lib().orc_matte_lift(C.byref(f), _ptr(binned["ranges"]), _ptr(ps), _ptr(proj["records"]), _ptr(sums),
                         1 if hard else 0, threshold, _ptr(out))
    return out


def trace(f: Frame, binned: dict, proj: dict) -> np.ndarray:
    """The trace's 11 planes (uint32, (11, width * height)); words the product leaves unwritten are 0 here."""
    out = np.zeros((11, f.width * f.height), np.uint32)
    ps = binned["pair_splats"] if binned["pairs"] else np.zeros(1, np.uint32)
    lib().orc_trace(C.byref(f), _ptr(binned["ranges"]), _ptr(ps), _ptr(proj["records"]), _ptr(out))
    return out


def position(f: Frame, proj_: Projection, depth: np.ndarray) -> np.ndarray:
    w, h = f.width, f.height
    inv = np.linalg.inv(np.asarray(proj_.worldToView[:], np.float64).reshape(4, 4))
    rows = np.ascontiguousarray(inv[:3].reshape(12).astype(np.float32))
    out = np.zeros((h * w, 4), np.float32)
    lib().orc_position(w, h, f.orthographic, f.focalX, f.focalY, f.centreX, f.centreY, _ptr(rows),
                       _ptr(np.ascontiguousarray(depth, np.float32)), _ptr(out))
    return out


def render(instances, proj_: Projection, width, height, *, threads=0, **settings):
    """A whole frame, the way TileRasterizer::render draws one (TileRasterizer.cpp:296-1295).

    instances: list of (positions, shape, sh, rest_per_colour, sh_words, object_to_world, linear).
    Returns the dict of every intermediate and output.
    """
    slots = sum(int(i[0].shape[0]) for i in instances)
    out = dict(records=np.zeros((max(slots, 1), 12), np.float32), rects=np.zeros((max(slots, 1), 4), np.uint32),
               touched=np.zeros(max(slots, 1), np.uint32), keys=np.zeros(max(slots, 1), np.uint32),
               visible=np.zeros(max(slots, 1), np.uint32))
    base = 0
    frames = []
    for (pos, shape, sh, rpc, shw, o2w, linear) in instances:
        f = frame_for(proj_, o2w, width, height, rest_per_colour=rpc, sh_words=shw, linear=linear, **settings)
        frames.append(f)
        project(f, pos, shape, sh, base=base, out=out, threads=threads)
        base += pos.shape[0]
    if not frames:
        frames.append(frame_for(proj_, np.eye(4), width, height, **settings))
    f0 = frames[0]
    if slots == 0:
        for k in out:
            out[k] = out[k][:0]
    binned = bin_(f0, out)
    blended = blend(f0, binned, out, threads=threads)
    return dict(frame=f0, proj=out, binned=binned, **blended)


# ---- FP64 ------------------------------------------------------------------
def frame64(proj_: Projection, object_to_world, width, height, *, antialias=1, max_sh_degree=3, rest_per_colour=15,
            sh_words=23, linear=0, bg=(0, 0, 0, 0)) -> Frame64:
    f = Frame64()
    lib().orc_frame64_from(C.byref(proj_), _ptr(_mat16(object_to_world)), width, height, antialias, max_sh_degree,
                           rest_per_colour, sh_words, linear, _ptr(np.asarray(bg, np.float64)), C.byref(f))
    return f


def render_f64(f: Frame64, positions, shape, sh, *, margin=1e-5, tile_stride=1, tile_offset=0, threads=0):
    w, h = f.width, f.height
    colour = np.full((h * w, 4), np.nan, np.float64)
    depth = np.full(h * w, np.nan, np.float64)
    near = np.zeros(h * w, np.uint8)
    n = positions.shape[0]
    lib().orc_render_f64(C.byref(f), n, _ptr(np.ascontiguousarray(positions, np.float32)),
                         _ptr(np.ascontiguousarray(shape, np.uint32)), _ptr(np.ascontiguousarray(sh, np.uint32)),
                         _ptr(colour), _ptr(depth), _ptr(near), margin, tile_stride, tile_offset, threads)
    return dict(colour=colour, depth=depth, near=near)


def render_params_sampled_f64(f: Frame64, means, scales, quats, sh, sh_degree, *, margin=1e-5, tile_stride=1,
                              tile_offset=0, threads=0):
    """FP32 training parameters ((N,4) means+logit, (N,4) log scales, (N,4) wxyz,
    (N,stride) SH) rendered in FP64; pixels of unsampled tiles stay NaN."""
    w, h = f.width, f.height
    colour = np.full((h * w, 4), np.nan, np.float64)
    depth = np.full(h * w, np.nan, np.float64)
    near = np.zeros(h * w, np.uint8)
    sh = np.ascontiguousarray(sh, np.float32)
    lib().orc_render_params_sampled_f64(
        C.byref(f), means.shape[0], _ptr(np.ascontiguousarray(means, np.float32)),
        _ptr(np.ascontiguousarray(scales, np.float32)), _ptr(np.ascontiguousarray(quats, np.float32)), _ptr(sh),
        sh.shape[1], sh_degree, _ptr(colour), _ptr(depth), _ptr(near), margin, tile_stride, tile_offset, threads)
    return dict(colour=colour, depth=depth, near=near)
