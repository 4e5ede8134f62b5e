// Stage (a): per-Gaussian projection -- splat/splat_project.slang:497-785 and
// :1080-1129 (projectSplat<0>, the plain entry splatProjectPlain) -- with the
// exclusive scan of the tiles each splat touches fused in (the reference runs
// PrefixSum::apply over them afterwards, TileRasterizer.cpp:1088-1089).
// Stage (b): the pairs, as 64-bit (tile << 24 | depth key) keys in slot order
// (splat/splat_emit.slang:17-50 applied to slot order), and the tiles' ranges
// (splat/splat_ranges.slang:11-25).
//
// Built with --fmad=false: see splat_math.cuh.
#include <algorithm>

#include <cuda_runtime.h>

#include "gauss.cuh"
#include "kernels.h"
#include "raster_types.cuh"
#include "splat_math.cuh"

namespace ath {
namespace {

struct Fate {
    bool removed, graded;
    float opacity;
};

// common/edit.slang:46-78
__device__ Fate editFate(const EditConst& e, float px, float py, float pz, float opacity, const float s[3]) {
    Fate fate{false, false, opacity};
    if (e.active == 0) return fate;
    if (e.minOpacity > 0.0f && opacity < e.minOpacity) {
        fate.removed = true;
        return fate;
    }
    if (e.maxScale > 0.0f && fmaxf(fmaxf(fabsf(s[0]), fabsf(s[1])), fabsf(s[2])) > e.maxScale) {
        fate.removed = true;
        return fate;
    }
    const float rx = px - e.centre[0], ry = py - e.centre[1], rz = pz - e.centre[2];
    bool inside = e.shape == 1 ? ((rx * rx + ry * ry) + rz * rz) <= e.size[0] * e.size[0]
                               : (fabsf(rx) <= e.size[0] && fabsf(ry) <= e.size[1] && fabsf(rz) <= e.size[2]);
    if (e.invert != 0) inside = !inside;
    if ((e.mode == 0 && !inside) || (e.mode == 1 && inside)) {
        fate.removed = true;
        return fate;
    }
    if (inside) {
        fate.graded = true;
        fate.opacity = opacity * e.opacity;
        fate.removed = !(fate.opacity >= kFaint);
    }
    return fate;
}

// common/edit.slang:86-90
__device__ void editGrade(const EditConst& e, float c[3]) {
    float g[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) g[k] = (c[k] * e.tint[k]) * e.brightness;
    const float luma = (g[0] * 0.2126f + g[1] * 0.7152f) + g[2] * 0.0722f;
#pragma unroll
    for (int k = 0; k < 3; ++k) c[k] = fmaxf(luma + (g[k] - luma) * e.saturation, 0.0f);
}

// common/sh.slang:25-51, the view-dependent part of the colour, channel by channel.
template <uint32_t L>
__device__ void evaluateRest(const InstanceConst& I, uint32_t i, uint32_t degree, float x, float y, float z,
                             float out[3]) {
    const float kC1 = 0.4886025119029199f;
#pragma unroll
    for (int ch = 0; ch < 3; ++ch) out[ch] = 0.0f;
    if (degree == 0) return;
#pragma unroll
    for (int ch = 0; ch < 3; ++ch) {
        const uint32_t c = (uint32_t)ch;
        auto B = [&](uint32_t k) { return restAt<L>(I, i, k * 3 + c); };
        float r = (((-kC1) * y) * B(0) + (kC1 * z) * B(1)) - (kC1 * x) * B(2);
        if (degree >= 2) {
            const float xx = x * x, yy = y * y, zz = z * z;
            const float xy = x * y, yz = y * z, xz = x * z;
            const float t = (((((1.0925484305920792f * xy) * B(3) + (-1.0925484305920792f * yz) * B(4)) +
                               (0.31539156525252005f * ((2.0f * zz - xx) - yy)) * B(5)) +
                              (-1.0925484305920792f * xz) * B(6)) +
                             (0.5462742152960396f * (xx - yy)) * B(7));
            r = r + t;
            if (degree >= 3) {
                const float u = ((((((((-0.5900435899266435f * y) * (3.0f * xx - yy)) * B(8) +
                                     ((2.890611442640554f * xy) * z) * B(9)) +
                                    ((-0.4570457994644658f * y) * ((4.0f * zz - xx) - yy)) * B(10)) +
                                   ((0.3731763325901154f * z) * ((2.0f * zz - 3.0f * xx) - 3.0f * yy)) * B(11)) +
                                  ((-0.4570457994644658f * x) * ((4.0f * zz - xx) - yy)) * B(12)) +
                                 ((1.445305721320277f * z) * (xx - yy)) * B(13)) +
                                ((-0.5900435899266435f * x) * (xx - 3.0f * yy)) * B(14));
                r = r + u;
            }
        }
        out[ch] = r;
    }
}

struct Projected {
    uint32_t touched;
    uint32_t key;   // depth key, or kCulledKey | reason
};

// One splat: projectSplat<0>. Writes the record and the rect of a splat that
// is kept; a culled one writes nothing here (its key says why).
template <uint32_t L>
__device__ Projected projectSlot(const FrameConst& F, const InstanceConst& I, uint32_t i, uint32_t slot,
                                 float4* __restrict__ recs, uint2* __restrict__ rects) {
    const Gauss g = loadGauss<L>(I, i);
    const Fate fate = editFate(I.edit, g.px, g.py, g.pz, g.opacity, g.scale);
    if (fate.removed) return {0, kCulledKey | kCullEdit};
    const Geometry G = projectGeometry(F, I, g, fate.opacity);
    if (G.cull) return {0, kCulledKey | G.cull};
    uint32_t rx0, ry0, rx1, ry1;
    if (!tileRectOf(F, G, rx0, ry0, rx1, ry1)) return {0, kCulledKey | kCullOffscreen};
    uint32_t touched = 0;
    for (uint32_t ty = ry0; ty <= ry1; ++ty)
        for (uint32_t tx = rx0; tx <= rx1; ++tx)
            touched += tileTouched(F.width, F.height, G.cx, G.cy, G.ca, G.cb, G.cc, G.cutoff, tx, ty) ? 1u : 0u;
    if (touched == 0) return {0, kCulledKey | kCullNoTile};

    const uint32_t degree = min(degreeOf(I.restPerColour), F.shLimit);
    const float dx = g.px - I.eye[0], dy = g.py - I.eye[1], dz = g.pz - I.eye[2];
    const float len = sqrtf((dx * dx + dy * dy) + dz * dz);
    float rest[3];
    evaluateRest<L>(I, i, degree, dx / len, dy / len, dz / len, rest);
    float colour[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float v = g.base[k] + rest[k];
        colour[k] = I.linear != 0 ? fmaxf(v, 0.0f) : srgbToLinear(v);
    }
    if (fate.graded) editGrade(I.edit, colour);

    recs[(size_t)slot * 3 + 0] = make_float4(G.cx, G.cy, G.tz, G.cutoff);
    recs[(size_t)slot * 3 + 1] = make_float4(G.ca, G.cb, G.cc, G.alpha);
    recs[(size_t)slot * 3 + 2] = make_float4(colour[0], colour[1], colour[2], 0.0f);
    rects[slot] = make_uint2(rx0 | (ry0 << 16), rx1 | (ry1 << 16));
    return {touched, __float_as_uint(G.tz) >> 7};
}

constexpr uint32_t kProjectThreads = 256;

template <uint32_t L>
__global__ void __launch_bounds__(kProjectThreads)
    projectKernel(const FrameConst F, const InstanceConst* __restrict__ inst, uint32_t nInst, uint32_t slots,
                  uint32_t countCulls, float4* __restrict__ recs, uint2* __restrict__ rects,
                  uint32_t* __restrict__ keys, uint32_t* __restrict__ offsets, uint64_t* __restrict__ flags,
                  uint32_t* __restrict__ words) {
    __shared__ uint32_t sTicket;
    __shared__ uint32_t sWarp[kProjectThreads / 32];
    __shared__ uint64_t sPrefix;
    __shared__ uint32_t sCulled[8];
    __shared__ uint32_t sCloud[2 * kMaxClouds];   // count_splats: (visible, pairs) a cloud, this block's share
    if (threadIdx.x == 0) sTicket = atomicAdd(&words[kWordTicket], 1u);
    if (threadIdx.x < 8) sCulled[threadIdx.x] = 0;
    if (countCulls && threadIdx.x < 2 * kMaxClouds) sCloud[threadIdx.x] = 0;
    __syncthreads();
    const uint32_t b = sTicket;
    const uint32_t slot = b * kProjectThreads + threadIdx.x;
    uint32_t touched = 0;
    bool kept = false;
    if (slot < slots) {
        uint32_t k = 0;
        while (k + 1 < nInst && slot >= inst[k + 1].base) ++k;
        const Projected p = projectSlot<L>(F, inst[k], slot - inst[k].base, slot, recs, rects);
        keys[slot] = p.key;
        touched = p.touched;
        kept = p.key < kCulledKey;
        if (countCulls && !kept) atomicAdd(&sCulled[p.key & 7u], 1u);
        // splatCountersCloud's rows (TileRasterizer.cpp:1335-1346): the first 64 clouds one by one
        if (countCulls && kept && k < kMaxClouds) {
            atomicAdd(&sCloud[2 * k], 1u);
            atomicAdd(&sCloud[2 * k + 1], touched);
        }
    }
    // block-wide exclusive scan of `touched`
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    uint32_t incl = touched;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= (uint32_t)o) incl += v;
    }
    if (lane == 31) sWarp[warp] = incl;
    const uint32_t keptCount = __syncthreads_count(kept);
    uint32_t warpBase = 0, blockTotal = 0;
#pragma unroll
    for (uint32_t w = 0; w < kProjectThreads / 32; ++w) {
        const uint32_t v = sWarp[w];
        warpBase += w < warp ? v : 0u;
        blockTotal += v;
    }
    if (warp == 0) {
        const uint64_t prefix = lookbackExclusive(flags, b, blockTotal, &words[kWordStatus]);
        if (lane == 0) {
            sPrefix = prefix;
            if (keptCount) atomicAdd(&words[kWordVisible], keptCount);
            if (b == gridDim.x - 1) {
                const uint64_t total = prefix + blockTotal;
                words[kWordPairsLo] = (uint32_t)total;
                words[kWordPairsHi] = (uint32_t)(total >> 32);
            }
        }
    }
    if (countCulls) {
        uint32_t most = touched;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) most = max(most, __shfl_xor_sync(0xFFFFFFFFu, most, o));
        if (lane == 0 && most) atomicMax(&words[kWordMaxTiles], most);
    }
    __syncthreads();
    if (countCulls && threadIdx.x < 7 && sCulled[threadIdx.x]) atomicAdd(&words[kWordCulled + threadIdx.x], sCulled[threadIdx.x]);
    if (countCulls && threadIdx.x < 2 * kMaxClouds && sCloud[threadIdx.x])
        atomicAdd(&words[kWordClouds + threadIdx.x], sCloud[threadIdx.x]);
    if (slot < slots) offsets[slot] = (uint32_t)(sPrefix + (incl - touched) + warpBase);
}

// splat_emit.slang:17-50, for the slots in slot order: one 64-bit key
// (tile << 24 | depth key) and one value (the slot) per touched tile, row-major
// over the rect, with the same test as the projection. A stable sort of these
// keys gives each tile its splats in (depth key, slot) order -- the order the
// reference's depth sort followed by its stable tile sort gives
// (splat/frame.slang:17-20).
__global__ void __launch_bounds__(256)
    emitKernel(uint32_t width, uint32_t height, uint32_t tilesX, uint32_t slots, const float4* __restrict__ recs,
               const uint2* __restrict__ rects, const uint32_t* __restrict__ keys,
               const uint32_t* __restrict__ offsets, uint32_t* __restrict__ words, uint64_t capacity,
               uint64_t* __restrict__ pairKeys, uint32_t* __restrict__ pairValues) {
    const uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t total = (uint64_t)words[kWordPairsLo] | ((uint64_t)words[kWordPairsHi] << 32);
    if (slot == 0) {
        // what the sort, the ranges and the blends take: the pairs the buffers hold
        words[kWordPairsKept] = (uint32_t)min(total, capacity);
        if (total > capacity) atomicOr(&words[kWordSticky], kStatusPairOverflow);
    }
    if (slot >= slots) return;
    const uint32_t key = keys[slot];
    if (key >= kCulledKey) return;
    const uint32_t first = offsets[slot];
    const uint32_t expected = (slot + 1 < slots ? offsets[slot + 1] : (uint32_t)total) - first;
    const float4 s = recs[(size_t)slot * 3 + 0];
    const float4 k = recs[(size_t)slot * 3 + 1];
    const uint2 r = rects[slot];
    const uint32_t rx0 = r.x & 0xFFFFu, ry0 = r.x >> 16, rx1 = r.y & 0xFFFFu, ry1 = r.y >> 16;
    uint32_t written = 0;
    for (uint32_t ty = ry0; ty <= ry1 && written < expected; ++ty) {
        for (uint32_t tx = rx0; tx <= rx1 && written < expected; ++tx) {
            if (!tileTouched(width, height, s.x, s.y, k.x, k.y, k.z, s.w, tx, ty)) continue;
            const uint64_t at = (uint64_t)first + written;
            if (at < capacity) {
                pairKeys[at] = ((uint64_t)(ty * tilesX + tx) << 24) | key;
                pairValues[at] = slot;
            }
            written += 1;
        }
    }
}

// splat_ranges.slang:11-25 over the sorted keys; ranges were cleared first
// (splat_tiles_clear.slang).
// `pairsDevice`, when given, holds the pair count (at most `pairs`, the grid's bound).
__global__ void __launch_bounds__(256)
    rangesKernel(uint32_t pairs, const uint32_t* __restrict__ pairsDevice, uint32_t tiles,
                 const uint64_t* __restrict__ pairKeys, uint2* __restrict__ ranges, uint32_t* __restrict__ status) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (pairsDevice) pairs = min(pairs, *pairsDevice);
    if (i >= pairs) return;
    const uint32_t t = (uint32_t)(pairKeys[i] >> 24);
    if (t >= tiles) {
        atomicOr(status, kStatusIndexRange);
        return;
    }
    if (i == 0 || (uint32_t)(pairKeys[i - 1] >> 24) != t) ranges[t].x = i;
    if (i + 1 == pairs || (uint32_t)(pairKeys[i + 1] >> 24) != t) ranges[t].y = i + 1;
}

}   // namespace

cudaError_t launchProject(const FrameConst& F, const InstanceConst* inst, uint32_t nInst, uint32_t slots,
                          uint32_t layout, bool countCulls, float4* recs, uint2* rects, uint32_t* keys,
                          uint32_t* offsets, uint64_t* flags, uint32_t* words, cudaStream_t stream) {
    if (slots == 0) return cudaSuccess;
    const uint32_t blocks = (slots + kProjectThreads - 1) / kProjectThreads;
    const uint32_t cc = countCulls ? 1u : 0u;
    if (layout == kLayoutPacked)
        projectKernel<kLayoutPacked><<<blocks, kProjectThreads, 0, stream>>>(F, inst, nInst, slots, cc, recs, rects,
                                                                            keys, offsets, flags, words);
    else if (layout == kLayoutParams)
        projectKernel<kLayoutParams><<<blocks, kProjectThreads, 0, stream>>>(F, inst, nInst, slots, cc, recs, rects,
                                                                            keys, offsets, flags, words);
    else
        projectKernel<kLayoutMixed><<<blocks, kProjectThreads, 0, stream>>>(F, inst, nInst, slots, cc, recs, rects,
                                                                           keys, offsets, flags, words);
    return cudaGetLastError();
}

uint32_t projectBlocks(uint32_t slots) { return (slots + kProjectThreads - 1) / kProjectThreads; }

cudaError_t launchEmit(const FrameConst& F, uint32_t slots, const float4* recs, const uint2* rects,
                       const uint32_t* keys, const uint32_t* offsets, uint32_t* words, uint64_t capacity,
                       uint64_t* pairKeys, uint32_t* pairValues, cudaStream_t stream) {
    emitKernel<<<std::max(1u, (slots + 255) / 256), 256, 0, stream>>>(F.width, F.height, F.tilesX, slots, recs, rects, keys,
                                                        offsets, words, capacity, pairKeys, pairValues);
    return cudaGetLastError();
}

cudaError_t launchRanges(uint32_t pairs, const uint32_t* pairsDevice, uint32_t tiles, const uint64_t* pairKeys,
                         uint2* ranges, uint32_t* status, cudaStream_t stream) {
    if (pairs == 0) return cudaSuccess;
    rangesKernel<<<(pairs + 255) / 256, 256, 0, stream>>>(pairs, pairsDevice, tiles, pairKeys, ranges, status);
    return cudaGetLastError();
}

}   // namespace ath
