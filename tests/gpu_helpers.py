"""Shared by the GPU tests: drive the product through its C ABI with torch
device memory, and the oracle on the same packed inputs."""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

import athenea_b200 as A
from athenea_b200 import _native as N


class _DeviceView:
    """A device buffer the library owns, as torch sees one (__cuda_array_interface__)."""

    def __init__(self, ptr: int, shape, typestr: str):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 3, "strides": None}


def fetch(ptr, shape, dtype) -> np.ndarray:
    n = int(np.prod(shape))
    if n == 0 or not ptr:
        return np.zeros(shape, dtype)
    typestr = {np.float32: "<f4", np.uint32: "<u4", np.uint64: "<u8", np.int32: "<i4"}[dtype]
    t = torch.as_tensor(_DeviceView(ptr, shape, typestr), device="cuda")
    torch.cuda.synchronize()
    return t.cpu().numpy().astype(dtype, copy=False).copy()


def upload(packed) -> A.GpuSplats:
    pos, shape, sh, rpc, shw = packed
    n = pos.shape[0]
    return A.GpuSplats(torch.from_numpy(np.ascontiguousarray(pos, np.float32)).cuda(),
                       torch.from_numpy(np.ascontiguousarray(shape, np.uint32).view(np.int32)).cuda(),
                       torch.from_numpy(np.ascontiguousarray(sh, np.uint32).view(np.int32)).cuda(),
                       n, rpc, shw)


def frame_buffers(raster: A.TileRasterizer) -> dict:
    fb = N.FrameBuffers()
    N.check(N.lib().ath_raster_frame_buffers(raster._h, C.byref(fb)))
    s, p, t = fb.slots, fb.pairs, fb.tiles
    return dict(slots=s, pairs=p, tiles=t,
                records=fetch(fb.records, (s, 12), np.float32),
                rects=fetch(fb.rects, (s, 2), np.uint32),
                keys=fetch(fb.keys, (s,), np.uint32),
                offsets=fetch(fb.offsets, (s,), np.uint32),
                pair_keys=fetch(fb.pair_keys, (p,), np.uint64),
                pair_splats=fetch(fb.pair_splats, (p,), np.uint32),
                ranges=fetch(fb.ranges, (t, 2), np.uint32))


def render_product(raster, proj, splats_list, o2w_list, settings: A.RenderSettings, position=False):
    targets = A.RenderTargets.make(settings.width, settings.height, position=position)
    inst = [A.SplatInstance(s, o) for s, o in zip(splats_list, o2w_list)]
    stats = raster.render(proj, inst, settings, targets)
    torch.cuda.synchronize()
    out = dict(stats=stats, colour=targets.colour.cpu().numpy(), depth=targets.depth.cpu().numpy())
    if position:
        out["position"] = targets.position.cpu().numpy()
    out.update(frame_buffers(raster))
    return out


def oracle_projection(O, proj: N.Projection):
    """The product's projection, as the oracle's struct (one projection, both sides)."""
    p = O.Projection()
    p.worldToView[:] = proj.world_to_view[:]
    p.focalX, p.focalY, p.centreX, p.centreY = proj.focal_x, proj.focal_y, proj.centre_x, proj.centre_y
    p.nearZ, p.farZ, p.orthographic = proj.near_z, proj.far_z, proj.orthographic
    p.eyeWorld[:] = proj.eye_world[:]
    return p


def touched_of(out) -> np.ndarray:
    offs = out["offsets"].astype(np.int64)
    nxt = np.append(offs[1:], out["pairs"])
    t = nxt - offs
    t[out["keys"] >= 0xFF000000] = 0
    return t
