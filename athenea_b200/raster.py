"""The reference's rasteriser interface, over the C ABI.

Mirrors render::TileRasterizer (modules/render/include/athenea/render/
TileRasterizer.h:452-487), its settings and targets (:248-450), the camera
(Camera.h) and scene::CloudLoader::upload's decode (scene/GpuClouds.h:366), with
the same names, argument meaning and errors (failures raise AtheneaError
carrying the ErrorCode the reference would return). Device memory is torch's:
clouds and targets are CUDA tensors the caller owns.
"""
from __future__ import annotations

import ctypes as C
import math
import os
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _native as N
from ._native import AtheneaError, check


def _ptr(t: torch.Tensor | None):
    if t is None:
        return None
    if not t.is_cuda:
        raise AtheneaError(3, "device memory expected: pass CUDA tensors")
    if not t.is_contiguous():
        raise AtheneaError(3, "contiguous tensors expected")
    return C.c_void_p(t.data_ptr())


def _mat(m) -> np.ndarray:
    return np.asarray(m, dtype=np.float64).reshape(4, 4)


# ---- camera (Camera.h / Camera.cpp) ----------------------------------------
@dataclass
class Lens:
    """Camera.h:89-117."""
    orthographic: bool = False
    focal: float = 50.0
    haperture: float = 24.576
    vaperture: float = 18.672
    near_z: float = 0.1
    far_z: float = 10000.0
    window_translate: tuple = (0.0, 0.0)
    window_scale: tuple = (1.0, 1.0)
    window_roll: float = 0.0


@dataclass
class Camera:
    """Camera.h:119-126: camera_to_world is row-major, acting on column vectors."""
    camera_to_world: np.ndarray = field(default_factory=lambda: np.eye(4))
    lens: Lens = field(default_factory=Lens)

    @staticmethod
    def looking_at(eye, target, up=(0.0, 1.0, 0.0)) -> "Camera":
        """Camera::lookingAt (Camera.cpp:9-25)."""
        c = N.Camera()
        check(N.lib().ath_camera_looking_at(np.asarray(eye, np.float64).ctypes.data_as(C.c_void_p),
                                            np.asarray(target, np.float64).ctypes.data_as(C.c_void_p),
                                            np.asarray(up, np.float64).ctypes.data_as(C.c_void_p), C.byref(c)))
        cam = Camera(np.array(c.camera_to_world[:]).reshape(4, 4))
        cam.lens.near_z = c.near_z
        return cam

    def _native(self) -> N.Camera:
        c = N.Camera()
        c.camera_to_world[:] = list(_mat(self.camera_to_world).reshape(16))
        c.orthographic = 1 if self.lens.orthographic else 0
        c.focal, c.haperture = self.lens.focal, self.lens.haperture
        c.near_z, c.far_z = self.lens.near_z, self.lens.far_z
        c.window_translate[:] = list(self.lens.window_translate)
        c.window_scale[:] = list(self.lens.window_scale)
        c.window_roll = self.lens.window_roll
        return c

    def projection_for(self, width: int, height: int) -> N.Projection:
        """projectionFor (Camera.cpp:32-64)."""
        p = N.Projection()
        check(N.lib().ath_projection_for(C.byref(self._native()), width, height, C.byref(p)))
        return p


def pinhole_for_vertical_fov(eye, target, width, height, vfov_degrees, up=(0.0, 1.0, 0.0)) -> Camera:
    """A lookingAt camera whose focal length gives `vfov_degrees` vertically over `height`
    pixels (square pixels: focal_px = (height / 2) / tan(vfov / 2))."""
    cam = Camera.looking_at(eye, target, up)
    focal_px = (height * 0.5) / math.tan(math.radians(vfov_degrees) * 0.5)
    cam.lens.focal = cam.lens.haperture * focal_px / width
    return cam


# ---- the cloud (scene/GpuClouds.h) -----------------------------------------
@dataclass
class GpuSplats:
    """scene::GpuSplats (GpuClouds.h:44-52): the packed layout of common/packing.slang."""
    positions: torch.Tensor          # (count, 4) float32
    shape: torch.Tensor              # (count, 4) int32 (uint32 bits)
    sh: torch.Tensor                 # (count, sh_words) int32 (uint32 bits)
    count: int
    rest_per_colour: int
    sh_words: int
    linear: bool = False
    antialiased: int = -1            # what the file said: -1 nothing

    def degree(self) -> int:
        r = self.rest_per_colour
        return 3 if r >= 15 else 2 if r >= 8 else 1 if r >= 3 else 0


# 3DGS record layouts (io::SplatEncoding) the decode reads.
def encoding_3dgs(rest_per_colour: int, stride: int | None = None, **fields) -> dict:
    """The field layout of a 3DGS PLY record: x y z nx ny nz f_dc(3) f_rest(3 r) opacity scale(3) rot(4)."""
    rest = 3 * rest_per_colour
    e = dict(x=0, y=1, z=2, dc0=6, dc1=7, dc2=8, rest_base=9, file_per_colour=rest_per_colour,
             opacity=9 + rest, scale0=10 + rest, scale1=11 + rest, scale2=12 + rest, rot_w=13 + rest,
             rot_x=14 + rest, rot_y=15 + rest, rot_z=16 + rest)
    e["stride"] = stride if stride is not None else 17 + rest
    e.update(fields)
    return e


PER_DEGREE = (0, 3, 8, 15)


def read_splat_ply(path: str) -> tuple[np.ndarray, dict]:
    """ath_ply_read (readSplatPly, modules/io/src/SplatReaders.cpp:50-200): a 3DGS
    PLY's vertex records as an (N, stride) float32 array and their encoding, for
    CloudLoader.upload(torch.from_numpy(records).cuda(), encoding)."""
    count = C.c_uint32()
    e = N.Encoding()
    raw = os.fsencode(path)
    check(N.lib().ath_ply_read_header(raw, C.byref(count), C.byref(e)))
    records = np.zeros((count.value, e.stride), np.float32)
    check(N.lib().ath_ply_read(raw, records.ctypes.data_as(C.c_void_p), records.size, C.byref(count), C.byref(e)))
    encoding = {k: int(getattr(e, k)) for k, _ in N.Encoding._fields_}
    return records, encoding


class CloudLoader:
    """scene::CloudLoader::upload (GpuClouds.h:366): records -> packed splats, on the GPU."""

    @staticmethod
    def upload(records: torch.Tensor, encoding: dict, max_degree: int = 3, linear: bool = False,
               stream: torch.cuda.Stream | None = None) -> GpuSplats:
        if records.dtype != torch.float32 or not records.is_cuda:
            raise AtheneaError(3, "records must be a CUDA float32 tensor")
        stride = encoding["stride"]
        count = records.numel() // stride
        keep = min(encoding["file_per_colour"], PER_DEGREE[min(max_degree, 3)])
        sh_words = 1 if keep == 0 else (keep * 3 + 1) // 2
        dev = records.device
        positions = torch.empty((max(count, 1), 4), dtype=torch.float32, device=dev)
        shape = torch.empty((max(count, 1), 4), dtype=torch.int32, device=dev)
        sh = torch.zeros((max(count, 1), sh_words), dtype=torch.int32, device=dev)
        e = N.Encoding(keep_per_colour=keep, **{k: encoding[k] for k in (
            "stride", "x", "y", "z", "opacity", "scale0", "scale1", "scale2", "rot_w", "rot_x", "rot_y", "rot_z",
            "dc0", "dc1", "dc2", "rest_base", "file_per_colour")})
        kept = C.c_uint32(0)
        s = stream if stream is not None else torch.cuda.current_stream(dev)
        check(N.lib().ath_decode_records(_ptr(records.contiguous()), count, C.byref(e), _ptr(positions),
                                         _ptr(shape), _ptr(sh), C.byref(kept), C.c_void_p(s.cuda_stream)))
        n = kept.value
        return GpuSplats(positions[:max(n, 1)], shape[:max(n, 1)], sh[:max(n, 1)], n, keep, sh_words, linear)


# ---- settings, instances, targets (TileRasterizer.h) -----------------------
@dataclass
class SplatEdit:
    """TileRasterizer.h:38-60."""
    active: bool = False
    shape: int = 0
    mode: int = 2
    centre: tuple = (0.0, 0.0, 0.0)
    size: tuple = (1.0, 1.0, 1.0)
    tint: tuple = (1.0, 1.0, 1.0)
    saturation: float = 1.0
    brightness: float = 1.0
    opacity: float = 1.0
    min_opacity: float = 0.0
    max_scale: float = 0.0
    invert: bool = False


@dataclass
class SplatInstance:
    """TileRasterizer.h:85-172 (its plain-path fields)."""
    splats: GpuSplats | None
    object_to_world: np.ndarray = field(default_factory=lambda: np.eye(4))
    edit: SplatEdit = field(default_factory=SplatEdit)


@dataclass
class RenderSettings:
    """TileRasterizer.h:248-371 (its plain-path fields)."""
    width: int = 1920
    height: int = 1080
    antialias: bool = True
    antialias_override: bool | None = None
    made_spread: float = 0.0
    surfels: bool = True
    max_sh_degree: int = 3
    background: tuple = (0.0, 0.0, 0.0, 0.0)
    depth_mode: int = 0           # 0 Mean, 1 Threshold
    depth_threshold: float = 0.5
    time_stages: bool = False
    count_splats: bool = False
    counters_tag: int = 0
    contribution_mode: int = 0    # 1 weights, 2 squared change, 3 lifted mask, 4 colour gradients (TileRasterizer.h:351-371)
    contribution: torch.Tensor | None = None    # int32: a word a slot (mode 1), two (modes 2, 3) or four (mode 4)
    final_colour: torch.Tensor | None = None    # float4 a pixel: the whole frame (mode 2) or dL/dpixel (mode 4)
    crypto_ids: torch.Tensor | None = None      # int32 a slot: the Cryptomatte id (0 names nothing)
    crypto: torch.Tensor | None = None          # (3, height * width, 4) float32: the matte's layers
    under_crypto: torch.Tensor | None = None    # int32 a pixel: the under layer's id
    lift_mask: torch.Tensor | None = None       # float a pixel, 0 to 1: mode 3's mask
    matte_lift: torch.Tensor | None = None      # int32, two a slot: what mode 3 lifted (weight x mask, weight)
    matte: torch.Tensor | None = None           # float a pixel: the matte those sums give
    matte_hard: bool = False
    matte_threshold: float = 0.5
    trace: torch.Tensor | None = None           # int32 (11, height * width): the splats each pixel is made of

    def _native(self) -> N.Settings:
        s = N.Settings()
        s.width, s.height = self.width, self.height
        s.antialias = 1 if self.antialias else 0
        s.antialias_override = -1 if self.antialias_override is None else int(bool(self.antialias_override))
        s.made_spread = self.made_spread
        s.surfels = 1 if self.surfels else 0
        s.max_sh_degree = self.max_sh_degree
        s.background[:] = list(self.background)
        s.depth_mode = self.depth_mode
        s.depth_threshold = self.depth_threshold
        s.time_stages = 1 if self.time_stages else 0
        s.count_splats = 1 if self.count_splats else 0
        s.counters_tag = self.counters_tag
        s.contribution_mode = self.contribution_mode
        s.contribution = _ptr(self.contribution) if self.contribution is not None else None
        s.final_colour = _ptr(self.final_colour) if self.final_colour is not None else None
        s.crypto_ids = _ptr(self.crypto_ids) if self.crypto_ids is not None else None
        s.crypto = _ptr(self.crypto) if self.crypto is not None else None
        s.under_crypto = _ptr(self.under_crypto) if self.under_crypto is not None else None
        s.lift_mask = _ptr(self.lift_mask) if self.lift_mask is not None else None
        s.matte_lift = _ptr(self.matte_lift) if self.matte_lift is not None else None
        s.matte = _ptr(self.matte) if self.matte is not None else None
        s.matte_hard = 1 if self.matte_hard else 0
        s.matte_threshold = self.matte_threshold
        s.trace = _ptr(self.trace) if self.trace is not None else None
        return s


@dataclass
class RenderTargets:
    """TileRasterizer.h:421-450 plus P: CUDA tensors, bottom row first."""
    width: int = 0
    height: int = 0
    colour: torch.Tensor | None = None     # (h*w, 4) float32, premultiplied linear
    depth: torch.Tensor | None = None      # (h*w,) float32, view z
    position: torch.Tensor | None = None   # (h*w, 4) float32, world xyz (optional)

    @staticmethod
    def make(width: int, height: int, position: bool = False, device="cuda") -> "RenderTargets":
        n = width * height
        return RenderTargets(width, height, torch.empty((n, 4), dtype=torch.float32, device=device),
                             torch.empty(n, dtype=torch.float32, device=device),
                             torch.empty((n, 4), dtype=torch.float32, device=device) if position else None)


def _instances(instances) -> tuple:
    arr = (N.Instance * max(len(instances), 1))()
    for k, inst in enumerate(instances):
        s = inst.splats
        a = arr[k]
        if s is not None and s.count:
            a.positions = _ptr(s.positions)
            a.shape = _ptr(s.shape)
            a.sh = _ptr(s.sh)
            a.count = s.count
            a.rest_per_colour = s.rest_per_colour
            a.sh_words = s.sh_words
            a.linear = 1 if s.linear else 0
            a.antialiased = s.antialiased
        a.object_to_world[:] = list(_mat(inst.object_to_world).reshape(16))
        e = inst.edit
        a.edit.active = 1 if e.active else 0
        a.edit.shape, a.edit.mode, a.edit.invert = e.shape, e.mode, 1 if e.invert else 0
        a.edit.centre[:], a.edit.size[:], a.edit.tint[:] = list(e.centre), list(e.size), list(e.tint)
        a.edit.saturation, a.edit.brightness, a.edit.opacity = e.saturation, e.brightness, e.opacity
        a.edit.min_opacity, a.edit.max_scale = e.min_opacity, e.max_scale
    return arr, len(instances)


@dataclass
class FrameStats:
    """TileRasterizer.h:408-419."""
    splats: int = 0
    visible: int = 0
    pairs: int = 0
    project_ms: float = 0.0
    counts_ms: float = 0.0
    depth_sort_ms: float = 0.0
    emit_ms: float = 0.0
    tile_sort_ms: float = 0.0
    blend_ms: float = 0.0
    total_ms: float = 0.0


@dataclass
class CloudCounts:
    """SplatCounters::Cloud (TileRasterizer.h:396-399)."""
    visible: int
    pairs: int


@dataclass
class SplatCounters:
    """TileRasterizer.h:373-401."""
    tag: int
    slots: int
    visible: int
    pairs: int
    max_tiles: int
    culled: list
    clouds: list


class TileRasterizer:
    """render::TileRasterizer (TileRasterizer.h:452-487)."""

    def __init__(self, handle):
        self._h = handle
        self._destroy = N.lib().ath_raster_destroy

    @staticmethod
    def create() -> "TileRasterizer":
        h = C.c_void_p()
        check(N.lib().ath_raster_create(C.byref(h)))
        return TileRasterizer(h)

    def __del__(self):
        # the destroy function is held by the instance: at interpreter exit the
        # module's globals may already be gone
        h = getattr(self, "_h", None)
        destroy = getattr(self, "_destroy", None)
        if h is not None and h.value and destroy is not None:
            destroy(h)
            self._h = None

    def render(self, camera, instances, settings: RenderSettings, targets: RenderTargets,
               stream: torch.cuda.Stream | None = None, under: "RenderTargets | None" = None,
               do_check: bool = True) -> FrameStats:
        """render(const Camera&/const Projection&, ..., const RenderTargets* under) -> FrameStats
        (TileRasterizer.cpp:287-1295); `under`, when given, is an opaque layer the splats are
        composited over (ath_raster_render_over). The native frame neither reads back nor
        waits; with `do_check` (the default, as the reference's render returns its totals and
        errors) this waits for the frame through ath_raster_check, raising its status (an
        overflow of the pairs is ATH_E_CAPACITY) and filling visible and pairs. do_check=False
        returns at once, the totals 0 unless the frame read them."""
        proj = camera.projection_for(settings.width, settings.height) if isinstance(camera, Camera) else camera
        arr, n = _instances(instances)
        t = N.Targets(targets.width, targets.height, _ptr(targets.colour), _ptr(targets.depth),
                      _ptr(targets.position))
        dev = targets.colour.device if targets.colour is not None else torch.device("cuda")
        s = stream if stream is not None else torch.cuda.current_stream(dev)
        native = settings._native()
        u = None if under is None else N.Targets(under.width, under.height, _ptr(under.colour), _ptr(under.depth),
                                                 None)

        def draw():
            stats = N.FrameStats()
            if u is None:
                check(N.lib().ath_raster_render(self._h, C.byref(proj), arr, n, C.byref(native), C.byref(t),
                                                C.byref(stats), C.c_void_p(s.cuda_stream)))
            else:
                check(N.lib().ath_raster_render_over(self._h, C.byref(proj), arr, n, C.byref(native), C.byref(t),
                                                     C.byref(u), C.byref(stats), C.c_void_p(s.cuda_stream)))
            return stats

        stats = self._drawn(draw, do_check)
        return FrameStats(*[getattr(stats, f) for f, _ in N.FrameStats._fields_])

    def _drawn(self, draw, do_check: bool):
        """Draws, and with do_check waits for the frame: a frame whose pairs outgrew the
        handle's capacity (ATH_E_CAPACITY) is drawn once more, the capacity grown from it, so
        that the frame returned is whole, as the reference's render always returns one."""
        stats = draw()
        if not do_check:
            return stats
        totals = N.FrameStats()
        status = N.lib().ath_raster_check(self._h, C.byref(totals))
        if status == N.STATUS_CODES["Capacity"]:
            stats = draw()
            status = N.lib().ath_raster_check(self._h, C.byref(totals))
        check(status)
        stats.visible, stats.pairs = totals.visible, totals.pairs
        return stats

    def check(self) -> FrameStats:
        """ath_raster_check: waits for the last frame (and its backward) and returns its totals;
        raises its status (ATH_E_CAPACITY when its pairs outgrew the buffers)."""
        totals = N.FrameStats()
        check(N.lib().ath_raster_check(self._h, C.byref(totals)))
        return FrameStats(*[getattr(totals, f) for f, _ in N.FrameStats._fields_])

    def latest_counters(self) -> SplatCounters | None:
        """latestCounters (TileRasterizer.h:478): the newest counted frame the device has
        finished, never waiting; None until one has."""
        c = N.SplatCounters()
        status = N.lib().ath_raster_latest_counters(self._h, C.byref(c))
        if status == 2:
            return None
        check(status)
        return SplatCounters(c.tag, c.slots, c.visible, c.pairs, c.max_tiles, list(c.culled),
                             [CloudCounts(c.clouds[k].visible, c.clouds[k].pairs) for k in range(c.cloud_count)])

    def release_scratch(self) -> None:
        """releaseScratch (TileRasterizer.h:482)."""
        check(N.lib().ath_raster_release_scratch(self._h))


def measure_peaks(repeats: int = 5, stream: torch.cuda.Stream | None = None) -> dict:
    """ath_measure_peaks: the current device's FP32 FMA rate (TFLOP/s) and hardware base-2
    exponential rate (G results/s), measured."""
    fma, ex2 = C.c_double(), C.c_double()
    s = stream if stream is not None else torch.cuda.current_stream()
    check(N.lib().ath_measure_peaks(repeats, C.byref(fma), C.byref(ex2), C.c_void_p(s.cuda_stream)))
    return {"fp32_tflops": fma.value, "ex2_gops": ex2.value}


def set_memory_budget(nbytes: int) -> None:
    """A cap on this library's device memory, in bytes (0: none), as the reference's
    ATHENEA_GPU_BUDGET (modules/gpu/src/Device.cpp:434-449): a frame whose scratch would
    pass it raises AtheneaError OutOfMemory (9); release_scratch gives memory back."""
    check(N.lib().ath_set_memory_budget(C.c_uint64(int(nbytes))))


def memory_held() -> tuple[int, int]:
    """(bytes this library's device buffers hold now, the budget; 0 = none)."""
    held, budget = C.c_uint64(), C.c_uint64()
    check(N.lib().ath_memory_held(C.byref(held), C.byref(budget)))
    return held.value, budget.value


def check_bounded_wait(preset: int, limit: int, stream: torch.cuda.Stream | None = None) -> int:
    """Run the library's bounded device-side wait on a flag set to `preset` (0: never set),
    giving up after `limit` spins; returns the spins taken, or raises AtheneaError Timeout (12)
    when it gave up. The context stays usable either way."""
    spins = C.c_uint32()
    s = stream if stream is not None else torch.cuda.current_stream()
    check(N.lib().ath_check_bounded_wait(C.c_uint32(preset), C.c_uint32(limit), C.byref(spins),
                                         C.c_void_p(s.cuda_stream)))
    return spins.value


# ---- differentiation -----------------------------------------------------------
@dataclass
class Params:
    """A cloud as FP32 training parameters (ath_params): CUDA tensors, one Gaussian a row.

    means (N, 4): x y z, opacity logit; scales (N, 4): log scales (4th unused);
    quats (N, 4): w x y z; sh (N, stride): DC rgb, then the rest rgb per basis.
    """
    means: torch.Tensor
    scales: torch.Tensor
    quats: torch.Tensor
    sh: torch.Tensor
    sh_degree: int = 3
    linear: bool = False
    object_to_world: np.ndarray = field(default_factory=lambda: np.eye(4))

    @property
    def count(self) -> int:
        return int(self.means.shape[0])

    def zeros_like(self) -> "Params":
        return Params(torch.zeros_like(self.means), torch.zeros_like(self.scales), torch.zeros_like(self.quats),
                      torch.zeros_like(self.sh), self.sh_degree, self.linear, self.object_to_world)

    def _native(self) -> N.Params:
        p = N.Params()
        p.means, p.scales, p.quats, p.sh = _ptr(self.means), _ptr(self.scales), _ptr(self.quats), _ptr(self.sh)
        p.count = self.count
        p.sh_degree = self.sh_degree
        p.sh_stride = int(self.sh.shape[1])
        p.linear = 1 if self.linear else 0
        p.object_to_world[:] = list(_mat(self.object_to_world).reshape(16))
        return p


def _render_params(self, camera, params: Params, settings: RenderSettings, targets: RenderTargets,
                   stream: torch.cuda.Stream | None = None, do_check: bool = True) -> FrameStats:
    """A differentiable frame (ath_raster_render_params): render() for one cloud of training
    parameters, keeping what backward() needs. do_check as for render()."""
    proj = camera.projection_for(settings.width, settings.height) if isinstance(camera, Camera) else camera
    t = N.Targets(targets.width, targets.height, _ptr(targets.colour), _ptr(targets.depth), _ptr(targets.position))
    s = stream if stream is not None else torch.cuda.current_stream(targets.colour.device)
    self._params_keep = params   # the backward reads them again
    native_params, native = params._native(), settings._native()

    def draw():
        st = N.FrameStats()
        check(N.lib().ath_raster_render_params(self._h, C.byref(proj), C.byref(native_params), C.byref(native),
                                               C.byref(t), C.byref(st), C.c_void_p(s.cuda_stream)))
        return st

    stats = self._drawn(draw, do_check)
    return FrameStats(*[getattr(stats, f) for f, _ in N.FrameStats._fields_])


def _backward(self, dl_dcolour: torch.Tensor, grads: Params, dl_ddepth: torch.Tensor | None = None,
              stream: torch.cuda.Stream | None = None) -> None:
    """ath_raster_backward: adds dL/dparameters of the last render_params frame into `grads`."""
    g = N.ParamGrads(_ptr(grads.means), _ptr(grads.scales), _ptr(grads.quats), _ptr(grads.sh))
    s = stream if stream is not None else torch.cuda.current_stream(dl_dcolour.device)
    check(N.lib().ath_raster_backward(self._h, _ptr(dl_dcolour), _ptr(dl_ddepth), C.byref(g),
                                      C.c_void_p(s.cuda_stream)))


TileRasterizer.render_params = _render_params
TileRasterizer.backward = _backward


def l2_loss(colour: torch.Tensor, target: torch.Tensor, dl_dcolour: torch.Tensor, loss: torch.Tensor,
            stream: torch.cuda.Stream | None = None) -> None:
    """ath_l2_loss: mean over pixels and rgb of (colour - target)^2 added into `loss` (a 1-element
    CUDA tensor); dL/dcolour written (float4 a pixel, alpha 0)."""
    s = stream if stream is not None else torch.cuda.current_stream(colour.device)
    check(N.lib().ath_l2_loss(_ptr(colour), _ptr(target), int(colour.shape[0]), _ptr(dl_dcolour), _ptr(loss),
                              C.c_void_p(s.cuda_stream)))


# ---- the batched, mixed-precision training step ---------------------------------
@dataclass
class MixedParams:
    """ath_mixed_params: geometry FP32 (as Params), SH DC and band 1 in BF16 (N, 12),
    bands 2-3 in FP8 e4m3 (N, 36) times a per-Gaussian scale (N,)."""
    means: torch.Tensor
    scales: torch.Tensor
    quats: torch.Tensor
    sh_low: torch.Tensor      # (N, 12) bfloat16
    sh_high: torch.Tensor     # (N, 36) uint8 (e4m3 bits)
    sh_scale: torch.Tensor    # (N,) float32
    sh_degree: int = 3
    linear: bool = False
    object_to_world: np.ndarray = field(default_factory=lambda: np.eye(4))

    @property
    def count(self) -> int:
        return int(self.means.shape[0])

    @staticmethod
    def from_params(P: "Params", stream: torch.cuda.Stream | None = None) -> "MixedParams":
        """ath_params_to_mixed: the SH to BF16 / FP8; the geometry tensors are shared."""
        n = P.count
        dev = P.means.device
        low = torch.empty((n, 12), dtype=torch.bfloat16, device=dev)
        high = torch.empty((n, 36), dtype=torch.uint8, device=dev)
        scale = torch.empty(n, dtype=torch.float32, device=dev)
        s = stream if stream is not None else torch.cuda.current_stream(dev)
        check(N.lib().ath_params_to_mixed(C.byref(P._native()), _ptr(low), _ptr(high), _ptr(scale),
                                          C.c_void_p(s.cuda_stream)))
        return MixedParams(P.means, P.scales, P.quats, low, high, scale, P.sh_degree, P.linear, P.object_to_world)

    def dequantized_sh(self) -> torch.Tensor:
        """The SH as the mixed layout holds them, back in FP32 (N, 48)."""
        n = self.count
        out = torch.zeros((n, 48), dtype=torch.float32, device=self.means.device)
        out[:, :12] = self.sh_low.float()
        e4m3 = self.sh_high.view(torch.float8_e4m3fn).float()
        out[:, 12:] = e4m3 * self.sh_scale[:, None]
        return out

    def _native(self) -> N.MixedParams:
        p = N.MixedParams()
        p.means, p.scales, p.quats = _ptr(self.means), _ptr(self.scales), _ptr(self.quats)
        p.sh_low, p.sh_high, p.sh_scale = _ptr(self.sh_low), _ptr(self.sh_high), _ptr(self.sh_scale)
        p.count = self.count
        p.sh_degree = self.sh_degree
        p.linear = 1 if self.linear else 0
        p.object_to_world[:] = list(_mat(self.object_to_world).reshape(16))
        return p


class BatchTrainer:
    """ath_batch: many views of one cloud, forward + loss + backward a step, each
    stage one launch over every view, the step captured in a CUDA graph."""

    def __init__(self):
        h = C.c_void_p()
        check(N.lib().ath_batch_create(C.byref(h)))
        self._h = h
        self._destroy = N.lib().ath_batch_destroy
        self.pixels = 0
        self.views = []

    def __del__(self):
        # the destroy function is held by the instance: at interpreter exit the
        # module's globals may already be gone
        h = getattr(self, "_h", None)
        destroy = getattr(self, "_destroy", None)
        if h is not None and h.value and destroy is not None:
            destroy(h)
            self._h = None

    def set_views(self, views, settings: RenderSettings | None = None) -> None:
        """views: [(projection, width, height)]; images concatenated in this order."""
        arr = (N.View * len(views))()
        for k, (proj, w, h) in enumerate(views):
            arr[k].projection = proj
            arr[k].width, arr[k].height = w, h
        s = (settings or RenderSettings())._native()
        check(N.lib().ath_batch_set_views(self._h, arr, len(views), C.byref(s)))
        px = C.c_uint32()
        check(N.lib().ath_batch_pixels(self._h, C.byref(px)))
        self.pixels = px.value
        self.views = [(w, h) for _, w, h in views]

    def set_tuning(self, tile: int, block_batch: int) -> None:
        check(N.lib().ath_batch_set_tuning(self._h, tile, block_batch))

    def set_buckets(self, buckets, events=None) -> None:
        """ath_batch_set_buckets: the step's gradients bucket by bucket into `buckets` (a
        parallel.BucketedGradients), recording events[k] (torch.cuda.Event) after bucket k;
        None: back to one gradient set a step."""
        if buckets is None:
            check(N.lib().ath_batch_set_buckets(self._h, 0, 0, None, None))
            self._buckets = None
            return
        arr = buckets.native()
        ev = None
        if events is not None:
            for e in events:
                if e.cuda_event == 0:          # torch makes the event on its first record
                    e.record()
            ev = (C.c_void_p * len(events))(*[e.cuda_event for e in events])
        self._buckets = (buckets, arr, events, ev)
        check(N.lib().ath_batch_set_buckets(self._h, buckets.count, len(buckets.params), arr, ev))

    def set_key_mode(self, mode: int) -> None:
        """ath_batch_set_key_mode: 0 automatic, 1 packed, 2 wide, 3 packed with the depth exponent renumbered."""
        check(N.lib().ath_batch_set_key_mode(self._h, mode))

    def step(self, params: MixedParams, target: torch.Tensor, colour: torch.Tensor, loss: torch.Tensor,
             grads: "Params | None", stream: torch.cuda.Stream | None = None,
             target_ready: torch.cuda.Event | None = None) -> None:
        """ath_batch_train_step; `grads` None when gradient buckets are set. With `target_ready`
        (ath_batch_train_step_after), only the blends wait for that event: the target's upload
        overlaps the projection and the sort."""
        g = N.ParamGrads(None, None, None, None) if grads is None else \
            N.ParamGrads(_ptr(grads.means), _ptr(grads.scales), _ptr(grads.quats), _ptr(grads.sh))
        s = stream if stream is not None else torch.cuda.current_stream(colour.device)
        self._keep = (params, target, colour, loss, grads, target_ready)
        if target_ready is not None and target_ready.cuda_event == 0:
            target_ready.record(s)   # torch makes the event on its first record
        ready = C.c_void_p(target_ready.cuda_event if target_ready is not None else None)
        check(N.lib().ath_batch_train_step_after(self._h, C.byref(params._native()), _ptr(target), ready,
                                                 _ptr(colour), _ptr(loss), C.byref(g), C.c_void_p(s.cuda_stream)))

    def render(self, params: MixedParams, colour: torch.Tensor, depth: torch.Tensor | None = None,
               stream: torch.cuda.Stream | None = None) -> None:
        """ath_batch_render: every view's colour (float4 a pixel, views concatenated) and, when given, depth
        (float a pixel), no loss or backward."""
        s = stream if stream is not None else torch.cuda.current_stream(colour.device)
        self._keep_render = (params, colour, depth)
        check(N.lib().ath_batch_render(self._h, C.byref(params._native()), _ptr(colour), _ptr(depth),
                                       C.c_void_p(s.cuda_stream)))

    def check(self, stream: torch.cuda.Stream | None = None) -> dict:
        st = N.BatchStats()
        s = stream if stream is not None else torch.cuda.current_stream()
        check(N.lib().ath_batch_check(self._h, C.byref(st), C.c_void_p(s.cuda_stream)))
        return dict(pairs=st.pairs, capacity=st.capacity, kept=st.kept, tile=st.tile, block_batch=st.block_batch,
                    degenerate=st.degenerate, evaluated=st.evaluated, blended=st.blended,
                    adjoint_visited=st.adjoint_visited, adjoint_live=st.adjoint_live,
                    warp_visits_forward=st.warp_visits_forward, warp_visits_adjoint=st.warp_visits_adjoint,
                    warp_visits_adjoint_summed=st.warp_visits_adjoint_summed, records_staged=st.records_staged)

    def tune(self, params: MixedParams, target, colour, loss, grads: "Params", repeats: int = 3,
             stream: torch.cuda.Stream | None = None) -> dict:
        g = N.ParamGrads(_ptr(grads.means), _ptr(grads.scales), _ptr(grads.quats), _ptr(grads.sh))
        st = N.BatchStats()
        s = stream if stream is not None else torch.cuda.current_stream(colour.device)
        self._keep = (params, target, colour, loss, grads)
        check(N.lib().ath_batch_tune(self._h, C.byref(params._native()), _ptr(target), _ptr(colour), _ptr(loss),
                                     C.byref(g), repeats, C.byref(st), C.c_void_p(s.cuda_stream)))
        return dict(pairs=st.pairs, tile=st.tile, block_batch=st.block_batch, ms_per_step=st.ms_per_step)

    def time_stages(self, params: MixedParams, target, colour, loss, grads: "Params | None",
                    stream: torch.cuda.Stream | None = None) -> dict:
        """ath_batch_time_stages: one step, not captured, with events between its stages (ms);
        `grads` None when gradient buckets are set."""
        g = N.ParamGrads(None, None, None, None) if grads is None else \
            N.ParamGrads(_ptr(grads.means), _ptr(grads.scales), _ptr(grads.quats), _ptr(grads.sh))
        ms = (C.c_float * 5)()
        s = stream if stream is not None else torch.cuda.current_stream(colour.device)
        self._keep = (params, target, colour, loss, grads)
        check(N.lib().ath_batch_time_stages(self._h, C.byref(params._native()), _ptr(target), _ptr(colour),
                                            _ptr(loss), C.byref(g), ms, C.c_void_p(s.cuda_stream)))
        names = ("project_emit", "sort", "ranges", "blends", "project_adjoint")
        return {n: float(v) for n, v in zip(names, ms)}

    def buffers(self) -> dict:
        b = N.BatchBuffers()
        check(N.lib().ath_batch_buffers_of(self._h, C.byref(b), C.c_void_p(torch.cuda.current_stream().cuda_stream)))
        return dict(pairs=b.pairs, key_shift=b.key_shift, slot_bits=b.slot_bits, total_tiles=b.total_tiles,
                    sorted_pairs=b.sorted_pairs, ranges=b.ranges, sorted_values=b.sorted_values,
                    tile_bases=[b.tile_bases[k] for k in range(b.views)], depth_bits=b.depth_bits,
                    exp_base=b.exp_base)
