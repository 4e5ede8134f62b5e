// The batched, mixed-precision training step: every view of a batch through
// each stage in one launch, with nothing read back between stages, so the
// whole step (forward, loss, backward) is captured once in a CUDA graph and
// replayed.
//
//   projectEmit   one block = 256 Gaussians x one view (blocks of the same
//                 Gaussians for every view run back to back, so the cloud is
//                 read from DRAM once and from L2 after): the exact projection
//                 geometry and the record, then the tiles touched, tested by a
//                 warp over its 32 footprints' candidate tiles as one list, the
//                 scan over every view's pairs by an epoch-tagged look-back, and
//                 the pairs; it also clears the records' gradient words.
//   sort          one onesweep sort of every view's pairs, packed into one
//                 64-bit word (global tile | 24-bit depth key | Gaussian), on
//                 the tile and depth bits only: stability keeps each tile's
//                 ties in Gaussian order, the reference's (frame.slang:17-20).
//   ranges        each tile's [start, end) in the sorted pairs.
//   blends        one persistent kernel over every view's tiles (a tile queue;
//                 tile size 8, 16 or 32 and a record batch of 64, 128, 256 or
//                 512): for each tile the forward blend, the loss of its pixels
//                 (each view's mean L2 against its target, summed over views)
//                 and the blend's adjoint (batch_blend.cu).
//   projectAdjoint one thread a Gaussian over every view, its gradient kept in
//                 registers and written once.
//
// The geometry that decides footprints, tiles and depth keys is the plain
// path's to the bit (this file builds with --fmad=false and calls the same
// projectGeometry): pairs, their order and the tile ranges are the reference's,
// except for near-degenerate footprints (det < 1e-6 trace^2 of the dilated 2D
// covariance), whose determinants and inverse come from FP64 (gauss.cuh
// wideCovariance) and whose tile test evaluates the conic in factored form;
// ath_batch_stats.degenerate counts them. Records carry the factored conic
// (ca, fr, fs): power = ca (dx + fr dy)^2 + fs dy^2, which has no cancellation
// and one operation fewer than the expanded form. Colour (SH in BF16/FP8 from
// the mixed layout), the blend's exponential and its divisions use the fast
// hardware paths; the image error that costs is measured against an FP64 oracle.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <vector>

#include <cuda_bf16.h>
#include <cuda_fp8.h>
#include <cuda_runtime.h>

#include "../../include/athenea_raster.h"
#include "adjoint.cuh"
#include "batch_kernels.cuh"
#include "host_util.h"
#include "kernels.h"

namespace ath {
namespace {

constexpr uint32_t kProjThreads = 256;

// ---- the step's first kernel: a new epoch, the step's counters cleared ------
__global__ void beginStepKernel(uint32_t* words) {
    words[kBatchEpoch] = (words[kBatchEpoch] + 1u) & 0x3FFFFFFFu;
    words[kBatchTicket] = 0;
    words[kBatchPairsLo] = 0;
    words[kBatchPairsHi] = 0;
    words[kBatchBlendTicket] = 0;
    words[kBatchKept] = 0;
    for (int p = 0; p < 8; ++p) words[kBatchSortTickets + p] = 0;
    words[kBatchDegenerate] = 0;
    words[kBatchExpMin] = 0xFFu;
    words[kBatchExpMax] = 0u;
}

// Block b's word of an epoch-tagged look-back: its aggregate (its inclusive
// sum for block 0), stored ahead of lookbackEpoch so that the block can do
// other work before it waits.
__device__ __forceinline__ void publishEpoch(uint64_t* flags, uint32_t b, uint32_t aggregate, uint32_t epoch) {
    if ((threadIdx.x & 31u) == 0) storeRelaxed(flags + b, tagged(epoch, b == 0 ? 2 : 1, aggregate));
}

// The decoupled look-back of lookbackExclusive with epoch-tagged 32-bit values.
// `published`: block b's word was stored already (publishEpoch).
__device__ uint32_t lookbackEpoch(uint64_t* flags, uint32_t b, uint32_t aggregate, uint32_t epoch, uint32_t* status,
                                  bool published = false) {
    const uint32_t lane = threadIdx.x & 31u;
    if (b == 0) {
        if (lane == 0 && !published) storeRelaxed(flags, tagged(epoch, 2, aggregate));
        return 0;
    }
    if (lane == 0 && !published) storeRelaxed(flags + b, tagged(epoch, 1, aggregate));
    uint64_t exclusive = 0;
    int64_t window = (int64_t)b - 1;
    uint32_t spins = 0;
    while (true) {
        const int64_t idx = window - (int64_t)lane;
        const uint64_t v = idx >= 0 ? loadRelaxed(flags + idx) : tagged(epoch, 2, 0);
        const uint32_t st = (uint32_t)(v >> 34) == (epoch & 0x3FFFFFFFu) ? (uint32_t)(v >> 32) & 3u : 0u;
        const uint32_t notReady = __ballot_sync(0xFFFFFFFFu, st == 0);
        const uint32_t inclusive = __ballot_sync(0xFFFFFFFFu, st == 2);
        const uint32_t first = inclusive ? (uint32_t)(__ffs(inclusive) - 1) : 32u;
        const uint32_t need = first >= 31 ? 0xFFFFFFFFu : ((2u << first) - 1u);
        if (notReady & need) {
            if (++spins > kSpinLimit || ((spins & 255u) == 0 && gaveUp(status))) {
                if (lane == 0) atomicOr(status, kStatusLookbackTimeout);
                break;
            }
            __nanosleep(32);
            continue;
        }
        exclusive += warpSum64(lane <= first ? (v & 0xFFFFFFFFull) : 0ull);
        if (first < 32) break;
        window -= 32;
    }
    if (exclusive + aggregate > 0xFFFFFFFFull) atomicOr(status, kStatusPairOverflow);
    if (lane == 0) storeRelaxed(flags + b, tagged(epoch, 2, (uint32_t)(exclusive + aggregate)));
    return (uint32_t)exclusive;
}

// The SH basis after the constant term (common/sh.slang:25-51) at direction (x, y, z).
__device__ __forceinline__ void shBasisFast(float x, float y, float z, float Y[15]) {
    const float C1 = 0.4886025119029199f;
    Y[0] = -C1 * y; Y[1] = C1 * z; Y[2] = -C1 * x;
    const float xx = x * x, yy = y * y, zz = z * z, xy = x * y, yz = y * z, xz = x * z;
    Y[3] = 1.0925484305920792f * xy; Y[4] = -1.0925484305920792f * yz;
    Y[5] = 0.31539156525252005f * (2.0f * zz - xx - yy); Y[6] = -1.0925484305920792f * xz;
    Y[7] = 0.5462742152960396f * (xx - yy);
    Y[8] = -0.5900435899266435f * y * (3.0f * xx - yy); Y[9] = 2.890611442640554f * xy * z;
    Y[10] = -0.4570457994644658f * y * (4.0f * zz - xx - yy);
    Y[11] = 0.3731763325901154f * z * (2.0f * zz - 3.0f * xx - 3.0f * yy);
    Y[12] = -0.4570457994644658f * x * (4.0f * zz - xx - yy); Y[13] = 1.445305721320277f * z * (xx - yy);
    Y[14] = -0.5900435899266435f * x * (xx - 3.0f * yy);
}

// The gradient of basis function k of shBasisFast with respect to (x, y, z).
__device__ __forceinline__ void shBasisGrad(uint32_t k, float x, float y, float z, float g[3]) {
    const float C1 = 0.4886025119029199f, C20 = 1.0925484305920792f, C22 = 0.31539156525252005f,
                C24 = 0.5462742152960396f, C30 = -0.5900435899266435f, C31 = 2.890611442640554f,
                C32 = -0.4570457994644658f, C33 = 0.3731763325901154f, C35 = 1.445305721320277f;
    const float xx = x * x, yy = y * y, zz = z * z;
    g[0] = g[1] = g[2] = 0.0f;
    switch (k) {
        case 0: g[1] = -C1; break;
        case 1: g[2] = C1; break;
        case 2: g[0] = -C1; break;
        case 3: g[0] = C20 * y; g[1] = C20 * x; break;
        case 4: g[1] = -C20 * z; g[2] = -C20 * y; break;
        case 5: g[0] = -2.0f * C22 * x; g[1] = -2.0f * C22 * y; g[2] = 4.0f * C22 * z; break;
        case 6: g[0] = -C20 * z; g[2] = -C20 * x; break;
        case 7: g[0] = 2.0f * C24 * x; g[1] = -2.0f * C24 * y; break;
        case 8: g[0] = C30 * 6.0f * x * y; g[1] = C30 * (3.0f * xx - 3.0f * yy); break;
        case 9: g[0] = C31 * y * z; g[1] = C31 * x * z; g[2] = C31 * x * y; break;
        case 10: g[0] = C32 * (-2.0f * x * y); g[1] = C32 * (4.0f * zz - xx - 3.0f * yy); g[2] = C32 * 8.0f * y * z; break;
        case 11: g[0] = C33 * (-6.0f * x * z); g[1] = C33 * (-6.0f * y * z); g[2] = C33 * (6.0f * zz - 3.0f * xx - 3.0f * yy); break;
        case 12: g[0] = C32 * (4.0f * zz - 3.0f * xx - yy); g[1] = C32 * (-2.0f * x * y); g[2] = C32 * 8.0f * x * z; break;
        case 13: g[0] = C35 * 2.0f * x * z; g[1] = C35 * (-2.0f * y * z); g[2] = C35 * (xx - yy); break;
        default: g[0] = C30 * (3.0f * xx - 3.0f * yy); g[1] = C30 * (-6.0f * x * y); break;
    }
}

__device__ __forceinline__ uint32_t basesOf(uint32_t degree) {
    return degree == 3 ? 15 : degree == 2 ? 8 : degree == 1 ? 3 : 0;
}

// The colour (linear, clamped at 0) of a Gaussian seen along (dx, dy, dz) from
// the eye, from the mixed layout's SH held in registers.
__device__ __forceinline__ void colourFast(const MixedSh& sh, const Gauss& g, uint32_t degree, uint32_t linear,
                                           float dx, float dy, float dz, float colour[3]) {
    const float len = sqrtf((dx * dx + dy * dy) + dz * dz);
    const float inv = fastRcp(len);
    float Y[15];
    shBasisFast(dx * inv, dy * inv, dz * inv, Y);
    const uint32_t bases = basesOf(degree);
#pragma unroll
    for (int ch = 0; ch < 3; ++ch) {
        float v = g.base[ch];
#pragma unroll
        for (uint32_t k = 0; k < 15; ++k)
            if (k < bases) v = __fmaf_rn(Y[k], sh.rest(k * 3 + (uint32_t)ch), v);
        if (linear) {
            colour[ch] = fmaxf(v, 0.0f);
        } else {
            const float c = fmaxf(v, 0.0f);
            colour[ch] = c <= 0.04045f ? c * (1.0f / 12.92f) : __powf((c + 0.055f) * (1.0f / 1.055f), 2.4f);
        }
    }
}

// colourFast's adjoint: dL/dcolour `gc` -> dL/dSH (added into dSh, the DC
// first) and dL/dposition through the view direction (added into dp).
__device__ __forceinline__ void colourAdjointFast(const MixedSh& sh, const Gauss& g, uint32_t degree, uint32_t linear,
                                                  const float eye[3], const float gc[3], float dSh[48], float dp[3]) {
    const float ex = g.px - eye[0], ey = g.py - eye[1], ez = g.pz - eye[2];
    const float len = sqrtf((ex * ex + ey * ey) + ez * ez);
    const float inv = fastRcp(len);
    const float x = ex * inv, y = ey * inv, z = ez * inv;
    float Y[15];
    shBasisFast(x, y, z, Y);
    const uint32_t bases = basesOf(degree);
    float dv[3];
#pragma unroll
    for (int ch = 0; ch < 3; ++ch) {
        float v = g.base[ch];
#pragma unroll
        for (uint32_t k = 0; k < 15; ++k)
            if (k < bases) v = __fmaf_rn(Y[k], sh.rest(k * 3 + (uint32_t)ch), v);
        float dcdv;
        if (linear) {
            dcdv = v > 0.0f ? 1.0f : 0.0f;
        } else {
            dcdv = v <= 0.0f      ? 0.0f
                   : v <= 0.04045f ? 1.0f / 12.92f
                                   : (2.4f / 1.055f) * __powf((v + 0.055f) * (1.0f / 1.055f), 1.4f);
        }
        dv[ch] = gc[ch] * dcdv;
        dSh[ch] += kSH0 * dv[ch];
    }
    float dDir[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
    for (uint32_t k = 0; k < 15; ++k) {
        if (k >= bases) continue;
        float w = 0.0f;
#pragma unroll
        for (int ch = 0; ch < 3; ++ch) {
            dSh[3 + k * 3 + ch] += Y[k] * dv[ch];
            w = __fmaf_rn(sh.rest(k * 3 + (uint32_t)ch), dv[ch], w);
        }
        float gk[3];
        shBasisGrad(k, x, y, z, gk);
        dDir[0] = __fmaf_rn(gk[0], w, dDir[0]);
        dDir[1] = __fmaf_rn(gk[1], w, dDir[1]);
        dDir[2] = __fmaf_rn(gk[2], w, dDir[2]);
    }
    // dir = e / |e|
    const float dd = (dDir[0] * x + dDir[1] * y) + dDir[2] * z;
    dp[0] += (dDir[0] - x * dd) * inv;
    dp[1] += (dDir[1] - y * dd) * inv;
    dp[2] += (dDir[2] - z * dd) * inv;
}

// A tile of the rect (rx0, ry0, cols) at row-major index `local`: the row from a
// float quotient corrected to the exact one.
__device__ __forceinline__ void rectTile(uint32_t local, uint32_t cols, float invCols, uint32_t& c, uint32_t& r) {
    r = (uint32_t)(((float)local + 0.5f) * invCols);
    if (r * cols > local) --r;
    else if ((r + 1) * cols <= local) ++r;
    c = local - r * cols;
}

// frame.slang:374-379 for tile size T: does tile (tx, ty) hold a pixel centre
// inside the footprint? The factored form for a near-degenerate footprint.
__device__ __forceinline__ bool footprintTouches(float4 fa, float4 fb, bool wide, uint32_t tx, uint32_t ty,
                                                 uint32_t T, uint32_t width, uint32_t height) {
    const float lx = ((float)(tx * T) + 0.5f) - fa.x, ly = ((float)(ty * T) + 0.5f) - fa.y;
    const float hx = ((float)(min((tx + 1) * T, width) - 1) + 0.5f) - fa.x;
    const float hy = ((float)(min((ty + 1) * T, height) - 1) + 0.5f) - fa.y;
    const float best = wide ? minPowerOverBoxFactored(fa.z, fa.w, fb.x, fb.z, fb.w, lx, ly, hx, hy)
                            : minPowerOverBox(fa.z, fa.w, fb.x, lx, ly, hx, hy);
    return best <= fb.y;
}

// The least lane k whose inclusive sum `incl` passes q (q below the warp's total).
__device__ __forceinline__ uint32_t ownerOf(uint32_t incl, uint32_t q) {
    uint32_t lo = 0;
#pragma unroll
    for (uint32_t step = 16; step >= 1; step >>= 1) {
        const uint32_t probe = __shfl_sync(0xFFFFFFFFu, incl, lo + step - 1u);
        if (probe <= q) lo += step;
    }
    return lo;
}

// ---- the batched projection and pair emission: one thread a (view, Gaussian) ----
// A block projects kProjThreads Gaussians for one view and writes their records.
// The tiles are tested and the pairs written by warps: the candidate tiles of a
// warp's 32 footprints (each footprint's screen rect, row-major) are one list,
// lane l taking entry 32 c + l, so a warp's work is the sum of its rects, not 32
// times the largest. A first walk counts the pairs (its ballots kept in shared
// memory), the block's total is published for the epoch look-back, the records'
// SH colours are computed while the blocks before finish theirs, the block's
// place among the pairs is read back, and a second walk writes the pairs in list order: a footprint's pairs in its rect's
// row-major order, footprints in thread order (splat_emit.slang:37-49).
constexpr uint32_t kBallotCache = 16;   // chunks of 32 candidates whose ballots a warp keeps

template <uint32_t L>
__global__ void __launch_bounds__(kProjThreads, 5)   // five blocks an SM: the kernel is latency-bound
    projectEmitKernel(const BatchConst B, const BatchView* __restrict__ views, float4* __restrict__ recs,
                      uint64_t* __restrict__ pairs, uint32_t* __restrict__ values, uint64_t* __restrict__ flags,
                      uint32_t* __restrict__ words, float* __restrict__ grads, uint32_t gaussBlocks) {
    constexpr uint32_t kWarps = kProjThreads / 32;
    __shared__ uint32_t sTicket;
    __shared__ uint32_t sWarp[kWarps];
    __shared__ uint32_t sPrefix;
    __shared__ BatchView sView;
    __shared__ FrameConst sF;
    __shared__ float4 sFa[kProjThreads];   // cx cy ca cb
    __shared__ float4 sFb[kProjThreads];   // cc cutoff fr fs
    __shared__ uint4 sRect[kProjThreads];  // rx0 ry0 cols, (depth key, 1 << 31 if wide)
    __shared__ float sInvCols[kProjThreads];
    __shared__ uint32_t sHit[kProjThreads];
    __shared__ uint32_t sBallot[kWarps][kBallotCache];
    if (threadIdx.x == 0) sTicket = atomicAdd(&words[kBatchTicket], 1u);
    __syncthreads();
    const uint32_t t = sTicket;
    const uint32_t gb = t / B.views, v = t % B.views;
    if (threadIdx.x == 0) {
        sView = views[v];
        FrameConst F{};
        F.width = sView.width; F.height = sView.height; F.tilesX = sView.tilesX; F.tilesY = sView.tilesY;
        F.focalX = sView.focalX; F.focalY = sView.focalY; F.centreX = sView.centreX; F.centreY = sView.centreY;
        F.nearZ = sView.nearZ; F.farZ = sView.farZ; F.orthographic = sView.orthographic; F.shLimit = B.shLimit;
        sF = F;
    }
    __syncthreads();
    const uint32_t epoch = words[kBatchEpoch];
    const FrameConst& F = sF;
    const uint32_t T = B.tile;
    const uint32_t i = gb * kProjThreads + threadIdx.x;
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    uint32_t area = 0;
    uint32_t expByte = 0;   // the record's depth exponent byte, when its rect is on screen
    sHit[threadIdx.x] = 0u;
    if (i < B.count && gb < gaussBlocks) {
        // the record's gradient words, which the blend adjoint sums into, start at zero (a training step's)
        if (grads) {
            float2* zero = reinterpret_cast<float2*>(grads + ((size_t)v * B.count + i) * kGradWords);
#pragma unroll
            for (uint32_t k = 0; k < kGradWords / 2; ++k) zero[k] = make_float2(0.0f, 0.0f);
        }
        InstanceConst I = B.inst;
#pragma unroll
        for (int k = 0; k < 12; ++k) I.m[k] = sView.m[k];
        I.eye[0] = sView.eye[0]; I.eye[1] = sView.eye[1]; I.eye[2] = sView.eye[2];
        const Gauss g = loadGauss<L>(I, i);
        const Geometry G = projectGeometry<true>(F, I, g, g.opacity);
        if (!G.cull) {
            // frame.slang:383-402 for tile size T; a near-degenerate footprint's
            // extents from its covariance's diagonal, which cc / det(conic) and
            // ca / det(conic) equal, without the cancelling determinant
            float ex, ey;
            if (G.wide) {
                ex = sqrtf(G.cutoff * (G.a + 0.3f));
                ey = sqrtf(G.cutoff * (G.c + 0.3f));
            } else {
                const float det2 = G.ca * G.cc - G.cb * G.cb;
                const float inv = det2 > 1e-20f ? 1.0f / det2 : 0.0f;
                ex = sqrtf(fmaxf((G.cutoff * G.cc) * inv, 0.0f));
                ey = sqrtf(fmaxf((G.cutoff * G.ca) * inv, 0.0f));
            }
            const float x1 = G.cx - ex, y1 = G.cy - ey, x2 = G.cx + ex, y2 = G.cy + ey;
            if (!(x2 < 0.0f || y2 < 0.0f || x1 >= (float)F.width || y1 >= (float)F.height)) {
                const uint32_t rx0 = (uint32_t)fmaxf(x1, 0.0f) / T;
                const uint32_t ry0 = (uint32_t)fmaxf(y1, 0.0f) / T;
                const uint32_t rx1 = (uint32_t)fminf(x2, (float)F.width - 1.0f) / T;
                const uint32_t ry1 = (uint32_t)fminf(y2, (float)F.height - 1.0f) / T;
                const uint32_t cols = rx1 - rx0 + 1;
                area = cols * (ry1 - ry0 + 1);
                sFa[threadIdx.x] = make_float4(G.cx, G.cy, G.ca, G.cb);
                sFb[threadIdx.x] = make_float4(G.cc, G.cutoff, G.fr, G.fs);
                // the depth field: the 24-bit depth key (exponent byte, 16 mantissa bits; z > 0),
                // or with the exponent renumbered from the step's planned base, which keeps the
                // order while every exponent lies in the plan's range
                const uint32_t depthKey = __float_as_uint(G.tz) >> 7;
                expByte = depthKey >> 16;
                uint32_t field = depthKey;
                if (B.depthBits < 24) {
                    const uint32_t span = 1u << (B.depthBits - 16);
                    uint32_t r = expByte - B.expBase;
                    if (expByte < B.expBase || r >= span) {
                        atomicOr(&words[kBatchStatus], kStatusDepthRange);
                        r = expByte < B.expBase ? 0u : span - 1u;
                    }
                    field = (r << 16) | (depthKey & 0xFFFFu);
                }
                sRect[threadIdx.x] = make_uint4(rx0, ry0, cols, field | (G.wide ? 1u << 31 : 0u));
                sInvCols[threadIdx.x] = 1.0f / (float)cols;
                // the record (read only through the pairs, so written for any rect on screen);
                // its colour once the block's pair count is published
                const size_t r = ((size_t)v * B.count + i) * 3;
                recs[r + 0] = make_float4(G.cx, G.cy, G.tz, G.cutoff);
                recs[r + 1] = make_float4(G.ca, G.fr, G.fs, G.alpha);
            }
        }
    }
    if (B.sizing) {
        // the depths' range of exponents, for planning the pairs' depth field (an atomic
        // only where this warp widens what the words already hold)
        const uint32_t lo = __reduce_min_sync(0xFFFFFFFFu, area ? expByte : 0xFFu);
        const uint32_t hi = __reduce_max_sync(0xFFFFFFFFu, area ? expByte : 0u);
        if (lane == 0 && lo <= hi) {
            if (lo < *reinterpret_cast<volatile uint32_t*>(&words[kBatchExpMin])) atomicMin(&words[kBatchExpMin], lo);
            if (hi > *reinterpret_cast<volatile uint32_t*>(&words[kBatchExpMax])) atomicMax(&words[kBatchExpMax], hi);
        }
    }
    // the warp's candidate list: lane k's rect at [incl - area, incl)
    uint32_t incl = area;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t u = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= (uint32_t)o) incl += u;
    }
    const uint32_t excl = incl - area;
    const uint32_t total = __shfl_sync(0xFFFFFFFFu, incl, 31);
    const uint32_t base = warp * 32;
    __syncwarp();
    uint32_t warpPairs = 0;
    for (uint32_t ch = 0, q0 = 0; q0 < total; ++ch, q0 += 32) {
        const uint32_t q = q0 + lane;
        const uint32_t owner = ownerOf(incl, min(q, total - 1u));
        const uint32_t start = __shfl_sync(0xFFFFFFFFu, excl, owner);
        bool hit = false;
        if (q < total) {
            const uint4 rect = sRect[base + owner];
            uint32_t c, r;
            rectTile(q - start, rect.z, sInvCols[base + owner], c, r);
            hit = footprintTouches(sFa[base + owner], sFb[base + owner], (rect.w >> 31) != 0u, rect.x + c, rect.y + r,
                                   T, F.width, F.height);
        }
        const uint32_t hits = __ballot_sync(0xFFFFFFFFu, hit);
        if (ch < kBallotCache && lane == 0) sBallot[warp][ch] = hits;
        warpPairs += __popc(hits);
        if (hit) sHit[base + owner] = 1u;
    }
    __syncwarp();
    const bool touched = sHit[threadIdx.x] != 0u;
    if (touched && (sRect[threadIdx.x].w >> 31)) atomicAdd(&words[kBatchDegenerate], 1u);
    // the scan of every view's pairs, in (Gaussian block, view, warp) order
    if (lane == 0) sWarp[warp] = warpPairs;
    const uint32_t kept = __syncthreads_count(touched);
    uint32_t warpBase = 0, blockTotal = 0;
#pragma unroll
    for (uint32_t w = 0; w < kWarps; ++w) {
        warpBase += w < warp ? sWarp[w] : 0u;
        blockTotal += sWarp[w];
    }
    if (warp == 0) publishEpoch(flags, t, blockTotal, epoch);
    // the record's colour (SH seen from the view's eye), which needs no place among the
    // pairs: computed while the blocks before this one finish their counts
    if (area > 0) {
        const InstanceConst& I = B.inst;
        const float4 m = __ldg(reinterpret_cast<const float4*>(I.means) + i);
        Gauss g;
        const __nv_bfloat16* bl = reinterpret_cast<const __nv_bfloat16*>(I.shLow) + (size_t)i * 12;
        g.base[0] = 0.5f + kSH0 * __bfloat162float(bl[0]);
        g.base[1] = 0.5f + kSH0 * __bfloat162float(bl[1]);
        g.base[2] = 0.5f + kSH0 * __bfloat162float(bl[2]);
        const uint32_t degree = min(degreeOf(I.restPerColour), F.shLimit);
        float colour[3];
        colourFast(loadMixedSh(I, i), g, degree, I.linear, m.x - sView.eye[0], m.y - sView.eye[1],
                   m.z - sView.eye[2], colour);
        recs[((size_t)v * B.count + i) * 3 + 2] = make_float4(colour[0], colour[1], colour[2], 0.0f);
    }
    if (warp == 0) {
        const uint32_t prefix = lookbackEpoch(flags, t, blockTotal, epoch, &words[kBatchStatus], true);
        if (lane == 0) {
            sPrefix = prefix;
            if (kept) atomicAdd(&words[kBatchKept], kept);
            if (t == gridDim.x - 1) {
                const uint64_t all = (uint64_t)prefix + blockTotal;
                words[kBatchPairsLo] = (uint32_t)all;
                words[kBatchPairsHi] = (uint32_t)(all >> 32);
                if (all > B.capacity) atomicOr(&words[kBatchStatus], kStatusPairOverflow);
            }
        }
    }
    __syncthreads();
    if (warpPairs == 0) return;
    // the pairs, in list order. packed: (global tile << keyShift) | (depth << slotBits) | Gaussian;
    // wide: (global tile << 24) | depth, the Gaussian beside it in `values`
    const uint32_t tileBase = sView.tileBase;
    const uint32_t below = (1u << lane) - 1u;
    uint64_t at = (uint64_t)sPrefix + warpBase;
    for (uint32_t ch = 0, q0 = 0; q0 < total; ++ch, q0 += 32) {
        const uint32_t q = q0 + lane;
        const uint32_t owner = ownerOf(incl, min(q, total - 1u));
        const uint32_t start = __shfl_sync(0xFFFFFFFFu, excl, owner);
        const uint4 rect = sRect[base + owner];
        uint32_t c = 0, r = 0;
        if (q < total) rectTile(q - start, rect.z, sInvCols[base + owner], c, r);
        const uint32_t tx = rect.x + c, ty = rect.y + r;
        uint32_t hits;
        if (ch < kBallotCache) {
            hits = sBallot[warp][ch];
        } else {
            const bool hit = q < total && footprintTouches(sFa[base + owner], sFb[base + owner], (rect.w >> 31) != 0u,
                                                           tx, ty, T, F.width, F.height);
            hits = __ballot_sync(0xFFFFFFFFu, hit);
        }
        if ((hits >> lane) & 1u) {
            const uint64_t pos = at + __popc(hits & below);
            const uint32_t gi = gb * kProjThreads + base + owner;
            if (pos < B.capacity) {
                const uint32_t tile = tileBase + ty * sView.tilesX + tx;
                pairs[pos] = ((uint64_t)tile << B.keyShift) | ((uint64_t)(rect.w & 0x7FFFFFFFu) << B.slotBits) |
                             (B.wide ? 0u : gi);
                if (B.wide) values[pos] = gi;
            }
        }
        at += __popc(hits);
    }
}

// The tiles in the order the blends take them: heaviest first (by the bit
// length of their pair count), so that the last tiles of the queue are light.
__global__ void __launch_bounds__(1024)
    tileOrderKernel(const uint2* __restrict__ ranges, uint32_t totalTiles, uint32_t* __restrict__ order) {
    __shared__ uint32_t sCount[33], sStart[33];
    if (threadIdx.x < 33) sCount[threadIdx.x] = 0;
    __syncthreads();
    for (uint32_t t = threadIdx.x; t < totalTiles; t += blockDim.x) {
        const uint2 r = ranges[t];
        atomicAdd(&sCount[32 - __clz(r.y - r.x)], 1u);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t s = 0;
        for (int k = 32; k >= 0; --k) {
            sStart[k] = s;
            s += sCount[k];
        }
    }
    __syncthreads();
    for (uint32_t t = threadIdx.x; t < totalTiles; t += blockDim.x) {
        const uint2 r = ranges[t];
        order[atomicAdd(&sStart[32 - __clz(r.y - r.x)], 1u)] = t;
    }
}

// Each tile's range in the sorted pairs: a thread takes a run of eight keys (four
// 16-byte loads) and the key before it, and writes a range's start and the
// previous range's end where the tile changes.
constexpr uint32_t kRangeRun = 8;

__global__ void __launch_bounds__(256)
    rangesBatchKernel(uint64_t capacity, const uint32_t* __restrict__ words, uint32_t keyShift, uint32_t totalTiles,
                      const uint64_t* __restrict__ pairs, uint2* __restrict__ ranges, uint32_t* __restrict__ status) {
    const uint64_t n = min((uint64_t)words[kBatchPairsLo] | ((uint64_t)words[kBatchPairsHi] << 32), capacity);
    for (uint64_t run = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; run * kRangeRun < n;
         run += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t i0 = run * kRangeRun;
        uint64_t key[kRangeRun];
        if (i0 + kRangeRun <= n) {
            const ulonglong2* at = reinterpret_cast<const ulonglong2*>(pairs + i0);
#pragma unroll
            for (uint32_t k = 0; k < kRangeRun / 2; ++k) {
                const ulonglong2 two = at[k];
                key[2 * k] = two.x;
                key[2 * k + 1] = two.y;
            }
        } else {
#pragma unroll
            for (uint32_t k = 0; k < kRangeRun; ++k) key[k] = i0 + k < n ? pairs[i0 + k] : 0ull;
        }
        uint32_t prev = i0 == 0 ? 0xFFFFFFFFu : (uint32_t)(pairs[i0 - 1] >> keyShift);
#pragma unroll
        for (uint32_t k = 0; k < kRangeRun; ++k) {
            const uint64_t i = i0 + k;
            if (i >= n) break;
            uint32_t t = (uint32_t)(key[k] >> keyShift);
            if (t >= totalTiles) {
                atomicOr(status, kStatusIndexRange);
                t = 0xFFFFFFFFu;
            }
            if (t != prev) {
                if (t != 0xFFFFFFFFu) ranges[t].x = (uint32_t)i;
                if (prev < totalTiles) ranges[prev].y = (uint32_t)i;
            }
            if (i + 1 == n && t != 0xFFFFFFFFu) ranges[t].y = (uint32_t)n;
            prev = t;
        }
    }
}


// ---- Gaussians grouped by the views whose records took a gradient ----------------
// The projection's adjoint runs a Gaussian a thread over every view and skips a view
// whose record got no gradient (on C1 most records lie behind the pixels' early stop
// and get none); a warp of Gaussians with different such views runs each view's work
// for a few lanes. The forward blend sets `seen[v count + i]` for every record (v, i)
// some pixel blends (the records the blend adjoint gives a gradient). Ordering the
// Gaussians [first, end) by their word of those views (bit v mod 64, folded to 8 bits:
// exactly the views for up to 8) lets whole warps skip a view. Within a group the
// Gaussians keep their order inside each block of 256; the blocks' runs follow in the
// order the blocks reserve them. The adjoint's results do not depend on the order
// (each Gaussian's gradient is its own thread's).

// Gaussian i's views whose record some pixel blended: bit v mod 64.
__device__ __forceinline__ uint64_t seenViews(const uint8_t* __restrict__ seen, uint32_t views, uint32_t count,
                                              uint32_t i) {
    uint64_t m = 0;
    for (uint32_t v = 0; v < views; ++v) m |= (uint64_t)(seen[(size_t)v * count + i] != 0u) << (v & 63u);
    return m;
}
__device__ __forceinline__ uint32_t groupOf(uint64_t m) {
    m ^= m >> 32;
    m ^= m >> 16;
    m ^= m >> 8;
    return (uint32_t)m & 255u;
}

__global__ void __launch_bounds__(256)
    groupCountKernel(const uint8_t* __restrict__ seen, uint32_t views, uint32_t count, uint32_t first, uint32_t end,
                     uint32_t* __restrict__ counts) {
    __shared__ uint32_t sCount[256];
    sCount[threadIdx.x] = 0;
    __syncthreads();
    const uint32_t i = first + blockIdx.x * 256 + threadIdx.x;
    if (i < end) atomicAdd(&sCount[groupOf(seenViews(seen, views, count, i))], 1u);
    __syncthreads();
    if (sCount[threadIdx.x]) atomicAdd(&counts[threadIdx.x], sCount[threadIdx.x]);
}

// order[first + k], k < end - first: the Gaussians of [first, end), group by group;
// viewsOf[first + k]: that Gaussian's seenViews word (the views the adjoint visits
// when there are at most 64).
__global__ void __launch_bounds__(256)
    groupPlaceKernel(const uint8_t* __restrict__ seen, uint32_t views, uint32_t count, uint32_t first, uint32_t end,
                     const uint32_t* __restrict__ counts, uint32_t* __restrict__ cursors, uint32_t* __restrict__ order,
                     uint64_t* __restrict__ viewsOf) {
    __shared__ uint32_t sWarpCount[8][256];   // a warp's Gaussians of each group, then their offsets
    __shared__ uint32_t sStart[256], sBase[256], sWarp[8];
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    for (uint32_t w = 0; w < 8; ++w) sWarpCount[w][tid] = 0;
    // where each group starts: the exclusive scan of the groups' sizes
    const uint32_t c = counts[tid];
    uint32_t incl = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t u = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= (uint32_t)o) incl += u;
    }
    if (lane == 31) sWarp[warp] = incl;
    __syncthreads();
    uint32_t before = 0;
#pragma unroll
    for (uint32_t w = 0; w < 8; ++w) before += w < warp ? sWarp[w] : 0u;
    sStart[tid] = before + incl - c;
    // a Gaussian's rank among the block's Gaussians of its group, in index order
    const uint32_t i = first + blockIdx.x * 256 + tid;
    const bool valid = i < end;
    const uint64_t m = valid ? seenViews(seen, views, count, i) : 0ull;
    const uint32_t h = valid ? groupOf(m) : 256u + lane;
    const uint32_t peers = __match_any_sync(0xFFFFFFFFu, h);
    const uint32_t inWarp = __popc(peers & ((1u << lane) - 1u));
    if (valid && inWarp == 0) sWarpCount[warp][h] = __popc(peers);
    __syncthreads();
    {
        // group tid: its warps' counts to offsets, the block's total reserved at once
        uint32_t sum = 0;
        for (uint32_t w = 0; w < 8; ++w) {
            const uint32_t k = sWarpCount[w][tid];
            sWarpCount[w][tid] = sum;
            sum += k;
        }
        if (sum) sBase[tid] = atomicAdd(&cursors[tid], sum);
    }
    __syncthreads();
    if (valid) {
        const uint32_t at = sStart[h] + sBase[h] + sWarpCount[warp][h] + inWarp;
        if (at < end - first) {
            order[first + at] = i;
            viewsOf[first + at] = m;
        }
    }
}

// ---- the projection's adjoint over every view: one thread a Gaussian ---------
// Two passes over the views, so that what is live across them stays small: the
// colour's adjoint (the SH gradient, 48 values, and the position's share through
// the view direction), then the geometry's (position and opacity a view; the
// covariance factor's gradient dL/dM summed over the views and taken to the
// scales and the rotation once). The cloud's loads and the SH (packed in
// registers) are read once.
// Gaussians [first, end) a launch (a gradient bucket, or the whole cloud), whose
// gradients go to g*[i - first]; thread k takes Gaussian order[first + k]
// (groupPlaceKernel's order).
__global__ void __launch_bounds__(128)
    projectAdjointBatchKernel(const BatchConst B, const BatchView* __restrict__ views, const float* __restrict__ grads,
                              float4* __restrict__ gMeans, float4* __restrict__ gScales, float4* __restrict__ gQuats,
                              float* __restrict__ gSh, uint32_t shStride, uint32_t first, uint32_t end,
                              const uint32_t* __restrict__ order, const uint64_t* __restrict__ viewsOf) {
    // a warp's SH gradient rows (stride 49: lane l's value k at bank (17 l + k) mod 32), written
    // out a row at a time so that each store covers whole sectors: the rows of a grouped
    // warp's Gaussians lie far apart, and a lane storing its own row touches a sector a value
    __shared__ float sSh[4][32 * 49];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t limit = min(end, B.count);
    const uint32_t slot = first + blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t picked = slot < limit ? (order ? order[slot] : slot) : first;
    const bool active = slot < limit && picked >= first && picked < limit;
    if (!__any_sync(0xFFFFFFFFu, active)) return;
    const uint32_t i = active ? picked : first;   // a permutation of [first, end), grouped
    const uint32_t o = i - first;   // the row in this launch's gradient arrays
    // the views whose record of this Gaussian took a gradient (up to 64 views; past 64,
    // every view, the zero records skipped by their value): the other views' records
    // are not even read
    const bool masked = order && B.views <= 64;
    const uint64_t seenMask = masked && active ? viewsOf[slot] : 0ull;
    auto nextView = [&](uint32_t from) -> uint32_t {   // the first such view >= from, or B.views
        if (!masked) return from;
        const uint64_t m = from < 64u ? seenMask >> from : 0ull;
        return m ? from + (uint32_t)__ffsll((long long)m) - 1u : B.views;
    };
    InstanceConst I = B.inst;
    const Gauss g = loadGauss<kLayoutMixed>(I, i);
    const uint32_t degree = min(degreeOf(I.restPerColour), B.shLimit);
    float dp[3] = {0.0f, 0.0f, 0.0f};
    if (active) {
        const MixedSh sh = loadMixedSh(I, i);
        float dSh[48];
#pragma unroll
        for (int k = 0; k < 48; ++k) dSh[k] = 0.0f;
        // each view's colour gradient loaded a view ahead, so its latency overlaps the work
        // words 6..8 of a record (8-byte aligned: a record is 40 bytes): a pair and one
        float2 nextRG = make_float2(0.0f, 0.0f);
        float nextB = 0.0f;
        uint32_t v = nextView(0);
        if (v < B.views) {
            const float* gr = grads + ((size_t)v * B.count + i) * kGradWords;
            nextRG = *reinterpret_cast<const float2*>(gr + kGradR);
            nextB = gr[kGradB];
        }
        while (v < B.views) {
            const float gc[3] = {nextRG.x, nextRG.y, nextB};
            const uint32_t vn = nextView(v + 1);
            if (vn < B.views) {
                const float* gr = grads + ((size_t)vn * B.count + i) * kGradWords;
                nextRG = *reinterpret_cast<const float2*>(gr + kGradR);
                nextB = gr[kGradB];
            }
            if (!(gc[0] == 0.0f && gc[1] == 0.0f && gc[2] == 0.0f))
                colourAdjointFast(sh, g, degree, I.linear, views[v].eye, gc, dSh, dp);
            v = vn;
        }
        float* mine = sSh[warp] + lane * 49;
#pragma unroll
        for (uint32_t k = 0; k < 48; ++k) mine[k] = dSh[k];
    }
    __syncwarp();
    {
        // row r is lane r's, for the active lanes
        const uint32_t cols = min(48u, shStride), lanes = __ballot_sync(0xFFFFFFFFu, active);
        for (uint32_t r = 0; r < 32; ++r) {
            const uint32_t orow = __shfl_sync(0xFFFFFFFFu, o, r);
            if (!((lanes >> r) & 1u)) continue;
            float* row = gSh + (size_t)orow * shStride;
            for (uint32_t c = lane; c < cols; c += 32) row[c] = sSh[warp][r * 49 + c];
        }
    }
    if (!active) return;
    ParamGrad acc;
    acc.dp[0] = acc.dp[1] = acc.dp[2] = 0.0f;
    acc.dLogit = 0.0f;
    acc.dLogScale[0] = acc.dLogScale[1] = acc.dLogScale[2] = 0.0f;
    acc.dQuat[0] = acc.dQuat[1] = acc.dQuat[2] = acc.dQuat[3] = 0.0f;
    float dMsum[3][3] = {{0.0f, 0.0f, 0.0f}, {0.0f, 0.0f, 0.0f}, {0.0f, 0.0f, 0.0f}};
    bool shaped = false;
    // words 0..5 of a record (the moments and dL/dalpha) as three 8-byte pairs, a view ahead
    float2 next[3] = {make_float2(0.0f, 0.0f), make_float2(0.0f, 0.0f), make_float2(0.0f, 0.0f)};
    uint32_t view = nextView(0);
    if (view < B.views) {
        const float2* gr = reinterpret_cast<const float2*>(grads + ((size_t)view * B.count + i) * kGradWords);
#pragma unroll
        for (int k = 0; k < 3; ++k) next[k] = gr[k];
    }
    for (uint32_t v = view, vn; v < B.views; v = vn) {
        float gw[kGradWords];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            gw[2 * k] = next[k].x;
            gw[2 * k + 1] = next[k].y;
        }
        gw[6] = gw[7] = gw[8] = gw[9] = 0.0f;
        bool any = false;
#pragma unroll
        for (int k = 0; k < 6; ++k) any |= gw[k] != 0.0f;
        vn = nextView(v + 1);
        if (vn < B.views) {
            const float2* gr = reinterpret_cast<const float2*>(grads + ((size_t)vn * B.count + i) * kGradWords);
#pragma unroll
            for (int k = 0; k < 3; ++k) next[k] = gr[k];
        }
        if (!any) continue;
        const BatchView& V = views[v];
        FrameConst F{};
        F.width = V.width; F.height = V.height; F.tilesX = V.tilesX; F.tilesY = V.tilesY;
        F.focalX = V.focalX; F.focalY = V.focalY; F.centreX = V.centreX; F.centreY = V.centreY;
        F.nearZ = V.nearZ; F.farZ = V.farZ; F.orthographic = V.orthographic; F.shLimit = B.shLimit;
#pragma unroll
        for (int k = 0; k < 12; ++k) I.m[k] = V.m[k];
        I.eye[0] = V.eye[0]; I.eye[1] = V.eye[1]; I.eye[2] = V.eye[2];
        const Geometry G = projectGeometry<true>(F, I, g, g.opacity);
        batchMomentsToRecordGrad(G.ca, G.fr, G.fs, gw);   // the blend's moments, to the record's terms
        gw[5] = gw[5] / G.alpha;   // the blend summed the opacity times dL/dopacity (alpha >= 1/255)
        float dpv[3] = {0.0f, 0.0f, 0.0f};
        float dM[3][3];
        geometryAdjointToM(F, I, g, G, gw, dpv, acc, dM);
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int col = 0; col < 3; ++col) dMsum[r][col] += dM[r][col];
        shaped = true;
    }
    // dL/dM summed over the views, to the scales and the quaternion once
    if (shaped) {
        float R[3][3];
        rotationOf(g, R);
        shapeAdjoint(I, i, g, R, dMsum, acc);
    }
    gMeans[o] = make_float4(acc.dp[0] + dp[0], acc.dp[1] + dp[1], acc.dp[2] + dp[2], acc.dLogit);
    gScales[o] = make_float4(acc.dLogScale[0], acc.dLogScale[1], acc.dLogScale[2], 0.0f);
    gQuats[o] = make_float4(acc.dQuat[0], acc.dQuat[1], acc.dQuat[2], acc.dQuat[3]);
}

// ---- FP32 SH -> the mixed layout ------------------------------------------------
// DC and band 1 (12 values) to BF16; bands 2-3 (36 values) to FP8 e4m3 over a
// per-Gaussian scale, the largest magnitude over e4m3's largest finite (448).
__global__ void __launch_bounds__(256)
    toMixedKernel(const float* __restrict__ sh, uint32_t count, uint32_t stride, uint32_t degree,
                  __nv_bfloat16* __restrict__ low, __nv_fp8_e4m3* __restrict__ high, float* __restrict__ scale) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const float* row = sh + (size_t)i * stride;
    const uint32_t rest = degree >= 3 ? 45 : degree == 2 ? 24 : degree == 1 ? 9 : 0;
#pragma unroll
    for (uint32_t k = 0; k < 12; ++k) low[(size_t)i * 12 + k] = __float2bfloat16_rn(k < 3 + rest ? row[k] : 0.0f);
    float most = 0.0f;
    for (uint32_t k = 9; k < rest; ++k) most = fmaxf(most, fabsf(row[3 + k]));
    const float s = most > 0.0f ? most / 448.0f : 1.0f;
    scale[i] = s;
    const float inv = 1.0f / s;
    for (uint32_t k = 0; k < 36; ++k) high[(size_t)i * 36 + k] = __nv_fp8_e4m3(9 + k < rest ? row[12 + k] * inv : 0.0f);
}

}   // namespace
}   // namespace ath

// ===========================================================================
// Host side
// ===========================================================================
using namespace ath;

struct ath_batch {
    int device = 0;
    int sms = 148;
    std::vector<BatchView> views;
    DeviceBuffer viewsDev;
    uint32_t totalTiles = 0, totalPixels = 0, tileBits = 0;
    uint32_t tile = 16, blockBatch = 256;
    float bg[4] = {0, 0, 0, 0};
    uint32_t shLimit = 3, antialias = 1;
    uint32_t depthMode = 0;
    float depthThreshold = 0.5f;
    std::vector<ath_projection> projections;
    std::vector<uint32_t> widths, heights, tileBases;
    uint32_t lastSorted = 0, lastSlotBits = 0;
    // scratch
    DeviceBuffer words, recs, grads, projFlags, pairs[2], values[2], sortHist, sortFlags, ranges, tileOrder, live;
    DeviceBuffer seen, adjointOrder, adjointViews, groupWords;   // the projection adjoint's grouping
    uint32_t keyMode = 0;      // 0 automatic; 1 packed; 2 wide; 3 packed, depth exponent renumbered
    bool lastWide = false;
    // the pairs' form, planned by each sizing from its depths' exponents
    bool planned = false, planWide = false;
    uint32_t depthBits = 24, expBase = 0, lastDepthBits = 24, lastExpBase = 0;
    uint32_t count = 0;
    uint64_t capacity = 0;
    bool resize = true;
    // the captured steps: a few, keyed by the arrays a step reads and writes, so that a
    // caller alternating input or output buffers (double-buffered targets) replays
    // without capturing again
    static constexpr int kGraphs = 4;
    cudaStream_t captureStream = nullptr;
    cudaGraphExec_t exec[kGraphs] = {};
    uintptr_t graphKey[kGraphs][14] = {};
    int nextGraph = 0;   // the slot the next capture replaces
    // the gradient buckets (ath_batch_set_buckets): each bucket's arrays, and the event
    // the step records after its projection adjoint; empty: the whole cloud into `grads`
    std::vector<ath_param_grads> bucketGrads;
    std::vector<cudaEvent_t> bucketEvents;
    uint32_t bucketCount = 0;   // the Gaussians the buckets were set for
};

namespace {

uint32_t bitsForValues(uint64_t values) {   // FrameParams.h:18-24
    uint32_t bits = 1;
    while (bits < 63 && (uint64_t{1} << bits) < values) ++bits;
    return bits;
}

void dropGraph(ath_batch* b) {
    for (int k = 0; k < ath_batch::kGraphs; ++k) {
        if (b->exec[k]) cudaGraphExecDestroy(b->exec[k]);
        b->exec[k] = nullptr;
    }
    b->nextGraph = 0;
}

ath_status buildViews(ath_batch* b) {
    const uint32_t T = b->tile;
    b->views.clear();
    uint32_t tileBase = 0, pixelBase = 0;
    ath_settings s{};
    ath_settings_default(&s);
    for (size_t v = 0; v < b->projections.size(); ++v) {
        const ath_projection& p = b->projections[v];
        BatchView V{};
        V.width = b->widths[v];
        V.height = b->heights[v];
        V.tilesX = (V.width + T - 1) / T;
        V.tilesY = (V.height + T - 1) / T;
        s.width = V.width;
        s.height = V.height;
        const FrameConst F = frameConstFor(p, s);
        V.focalX = F.focalX; V.focalY = F.focalY; V.centreX = F.centreX; V.centreY = F.centreY;
        V.nearZ = F.nearZ; V.farZ = F.farZ; V.orthographic = F.orthographic;
        V.tileBase = tileBase;
        V.pixelBase = pixelBase;
        V.lossScale = 1.0f / (3.0f * (float)V.width * (float)V.height);
        tileBase += V.tilesX * V.tilesY;
        pixelBase += V.width * V.height;
        b->views.push_back(V);
    }
    b->totalTiles = tileBase;
    b->totalPixels = pixelBase;
    b->tileBases.clear();
    for (const BatchView& V : b->views) b->tileBases.push_back(V.tileBase);
    b->tileBits = bitsForValues(tileBase);
    return ATH_OK;
}

// The per-view object -> view rows and eye for a cloud placed by `objectToWorld`.
void placeCloud(ath_batch* b, const double objectToWorld[16]) {
    ath_settings s{};
    ath_settings_default(&s);
    ath_instance in{};
    std::memcpy(in.object_to_world, objectToWorld, sizeof(in.object_to_world));
    for (size_t v = 0; v < b->views.size(); ++v) {
        const InstanceConst I = instanceConstFor(b->projections[v], s, in, 0);
        std::memcpy(b->views[v].m, I.m, sizeof(I.m));
        std::memcpy(b->views[v].eye, I.eye, sizeof(I.eye));
    }
}

// Whether a step's pairs take the wide form: a 64-bit (tile << 24 | depth) key
// and a 32-bit Gaussian index, sorted as key and value. The packed form (one
// 64-bit word) is used while tile, depth and Gaussian bits fit in 64.
bool wideKeys(const ath_batch* b, uint32_t count) {
    if (b->keyMode == 2) return true;
    if (b->keyMode == 1) return false;
    return 24 + bitsForValues(std::max<uint64_t>(count, 2)) + b->tileBits > 64;
}

BatchConst batchConst(const ath_batch* b, const ath_mixed_params& P) {
    BatchConst B{};
    B.views = (uint32_t)b->views.size();
    B.count = P.count;
    B.tile = b->tile;
    B.wide = (b->planned ? b->planWide : wideKeys(b, P.count)) ? 1u : 0u;
    B.slotBits = B.wide ? 0u : bitsForValues(std::max<uint64_t>(P.count, 2));
    B.depthBits = b->planned && !B.wide ? b->depthBits : 24u;
    B.expBase = B.depthBits < 24 ? b->expBase : 0u;
    B.keyShift = B.depthBits + B.slotBits;
    B.totalTiles = b->totalTiles;
    B.totalPixels = b->totalPixels;
    B.shLimit = b->shLimit;
    B.depthMode = b->depthMode;
    B.depthThreshold = b->depthThreshold;
    B.antialias = b->antialias;
    B.linear = P.linear ? 1u : 0u;
    B.restPerColour = P.sh_degree >= 3 ? 15 : P.sh_degree == 2 ? 8 : P.sh_degree == 1 ? 3 : 0;
    for (int k = 0; k < 4; ++k) B.bg[k] = b->bg[k];
    B.capacity = b->capacity;
    InstanceConst& I = B.inst;
    I = InstanceConst{};
    I.means = P.means;
    I.scales = P.scales;
    I.quats = P.quats;
    I.shLow = P.sh_low;
    I.shHigh = P.sh_high;
    I.shScale = P.sh_scale;
    I.count = P.count;
    I.restPerColour = B.restPerColour;
    I.linear = B.linear;
    I.antialias = b->antialias;
    return B;
}

template <typename K>
int residentBlocks(K kernel, int threads, int sms) {
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, threads, 0);
    return std::max(n, 1) * sms;
}

cudaError_t launchBlendsFor(const ath_batch* b, const BatchConst& B, uint32_t sorted, cudaStream_t stream,
                            float4* colour, const float* target, float* loss, float* grads, float* depth,
                            bool count) {
    BlendLaunch L{};
    L.views = static_cast<const BatchView*>(b->viewsDev.ptr);
    L.ranges = static_cast<const uint2*>(b->ranges.ptr);
    L.pairs = static_cast<const uint64_t*>(b->pairs[sorted].ptr);
    L.values = B.wide ? static_cast<const uint32_t*>(b->values[sorted].ptr) : nullptr;
    L.recs = static_cast<const float4*>(b->recs.ptr);
    L.words = static_cast<uint32_t*>(b->words.ptr);
    L.order = static_cast<const uint32_t*>(b->tileOrder.ptr);
    L.live = static_cast<uint32_t*>(b->live.ptr);
    L.seen = static_cast<uint8_t*>(b->seen.ptr);
    L.sms = b->sms;
    L.tile = b->tile;
    L.blockBatch = b->blockBatch;
    L.count = count;
    return launchBatchBlendStep(B, L, stream, colour, target, loss, grads, depth);
}

// One step, enqueued (captured or not). `countOnly`: the projection alone, to size the pairs.
// A null `target`: a render, the forward blend alone (no loss, no backward).
cudaError_t enqueueStep(ath_batch* b, const ath_mixed_params& P, const float* target, float4* colour, float* loss,
                        ath_param_grads& g, cudaStream_t stream, bool countOnly, cudaEvent_t* marks = nullptr,
                        float* depth = nullptr, cudaEvent_t targetReady = nullptr, bool countWork = false) {
    auto mark = [&](int k) { if (marks) cudaEventRecord(marks[k], stream); };
    mark(0);
    BatchConst B = batchConst(b, P);
    if (countOnly) {
        B.capacity = 0;
        B.sizing = 1;
    }
    uint32_t* words = static_cast<uint32_t*>(b->words.ptr);
    const uint32_t V = B.views;
    const uint32_t gaussBlocks = (P.count + kProjThreads - 1) / kProjThreads;
    beginStepKernel<<<1, 1, 0, stream>>>(words);
    cudaError_t err = cudaGetLastError();
    if (err == cudaSuccess && P.count)
        projectEmitKernel<kLayoutMixed><<<gaussBlocks * V, kProjThreads, 0, stream>>>(
            B, static_cast<const BatchView*>(b->viewsDev.ptr), static_cast<float4*>(b->recs.ptr),
            static_cast<uint64_t*>(b->pairs[0].ptr), static_cast<uint32_t*>(b->values[0].ptr),
            static_cast<uint64_t*>(b->projFlags.ptr), words, target ? static_cast<float*>(b->grads.ptr) : nullptr,
            gaussBlocks);
    if (err == cudaSuccess) err = cudaGetLastError();
    if (countOnly || err != cudaSuccess) return err;
    mark(1);
    uint64_t* keys[2] = {static_cast<uint64_t*>(b->pairs[0].ptr), static_cast<uint64_t*>(b->pairs[1].ptr)};
    uint32_t* vals[2] = {static_cast<uint32_t*>(b->values[0].ptr), static_cast<uint32_t*>(b->values[1].ptr)};
    const uint32_t bits = B.depthBits + b->tileBits;
    err = launchSortDevice(keys, B.wide ? vals : nullptr, (uint32_t)b->capacity, words + kBatchPairsLo,
                           words + kBatchEpoch, B.slotBits, bits, static_cast<uint32_t*>(b->sortHist.ptr),
                           static_cast<uint64_t*>(b->sortFlags.ptr), words + kBatchSortTickets, words + kBatchStatus,
                           stream);
    const uint32_t sorted = sortResultIndex(2, bits);
    mark(2);
    b->lastSorted = sorted;
    b->lastSlotBits = B.slotBits;
    b->lastWide = B.wide != 0;
    b->lastDepthBits = B.depthBits;
    b->lastExpBase = B.expBase;
    if (err == cudaSuccess) err = cudaMemsetAsync(b->ranges.ptr, 0, (size_t)b->totalTiles * 8, stream);
    if (err == cudaSuccess) {
        const uint32_t grid = std::max<uint32_t>(
            1, std::min<uint64_t>((b->capacity + 256 * kRangeRun - 1) / (256 * kRangeRun), (uint64_t)b->sms * 8));
        rangesBatchKernel<<<grid, 256, 0, stream>>>(b->capacity, words, B.keyShift, b->totalTiles, keys[sorted],
                                                    static_cast<uint2*>(b->ranges.ptr), words + kBatchStatus);
        err = cudaGetLastError();
    }
    if (err == cudaSuccess && b->totalTiles) {
        tileOrderKernel<<<1, 1024, 0, stream>>>(static_cast<const uint2*>(b->ranges.ptr), b->totalTiles,
                                               static_cast<uint32_t*>(b->tileOrder.ptr));
        err = cudaGetLastError();
    }
    mark(3);
    const bool train = target != nullptr;
    if (err == cudaSuccess && targetReady) {
        // the target's upload overlapped the stages before: only the blends read it
        cudaStreamCaptureStatus capturing = cudaStreamCaptureStatusNone;
        err = cudaStreamIsCapturing(stream, &capturing);
        if (err == cudaSuccess)
            err = cudaStreamWaitEvent(stream, targetReady,
                                      capturing == cudaStreamCaptureStatusActive ? cudaEventWaitExternal : 0);
    }
    if (err == cudaSuccess && train) err = cudaMemsetAsync(loss, 0, sizeof(float), stream);
    if (err == cudaSuccess && train && P.count)
        err = cudaMemsetAsync(b->seen.ptr, 0, (size_t)B.views * P.count, stream);
    // the forward blend, the loss and the blend adjoint (the record gradients were cleared by the projection)
    if (err == cudaSuccess)
        err = launchBlendsFor(b, B, sorted, stream, colour, target, loss, static_cast<float*>(b->grads.ptr), depth,
                              countWork);
    mark(4);
    if (err == cudaSuccess && train && P.count) {
        // the whole cloud into `g`, or bucket by bucket into each bucket's arrays, each
        // bucket's event recorded after it (a caller's exchange starts on it)
        const uint32_t buckets = b->bucketGrads.empty() ? 1u : (uint32_t)b->bucketGrads.size();
        for (uint32_t k = 0; k < buckets && err == cudaSuccess; ++k) {
            uint32_t first = 0, n = P.count;
            if (!b->bucketGrads.empty()) ath_gradient_bucket(P.count, buckets, k, &first, &n);
            const ath_param_grads& gk = b->bucketGrads.empty() ? g : b->bucketGrads[k];
            if (n) {
                // the bucket's Gaussians grouped by the views that gave them a gradient, then
                // the adjoint in that order
                const uint8_t* seen = static_cast<const uint8_t*>(b->seen.ptr);
                uint32_t* counts = static_cast<uint32_t*>(b->groupWords.ptr);
                uint32_t* order = static_cast<uint32_t*>(b->adjointOrder.ptr);
                uint64_t* viewsOf = static_cast<uint64_t*>(b->adjointViews.ptr);
                const uint32_t blocks = (n + 255) / 256;
                err = cudaMemsetAsync(counts, 0, 2 * 256 * 4, stream);
                if (err == cudaSuccess) {
                    groupCountKernel<<<blocks, 256, 0, stream>>>(seen, B.views, P.count, first, first + n, counts);
                    groupPlaceKernel<<<blocks, 256, 0, stream>>>(seen, B.views, P.count, first, first + n, counts,
                                                                 counts + 256, order, viewsOf);
                    projectAdjointBatchKernel<<<(n + 127) / 128, 128, 0, stream>>>(
                        B, static_cast<const BatchView*>(b->viewsDev.ptr), static_cast<const float*>(b->grads.ptr),
                        reinterpret_cast<float4*>(gk.means), reinterpret_cast<float4*>(gk.scales),
                        reinterpret_cast<float4*>(gk.quats), gk.sh, 48, first, first + n, order, viewsOf);
                    err = cudaGetLastError();
                }
            }
            if (err == cudaSuccess && !b->bucketEvents.empty() && b->bucketEvents[k]) {
                // in a captured step, an event record node of the graph (an external
                // event: a stream outside the graph may wait on it after each replay)
                cudaStreamCaptureStatus capturing = cudaStreamCaptureStatusNone;
                err = cudaStreamIsCapturing(stream, &capturing);
                if (err == cudaSuccess)
                    err = capturing == cudaStreamCaptureStatusActive
                              ? cudaEventRecordWithFlags(b->bucketEvents[k], stream, cudaEventRecordExternal)
                              : cudaEventRecord(b->bucketEvents[k], stream);
            }
        }
    }
    mark(5);
    return err;
}

ath_status reserveBatch(ath_batch* b, uint32_t count) {
    const uint32_t V = (uint32_t)b->views.size();
    const uint32_t gaussBlocks = (count + kProjThreads - 1) / kProjThreads;
    cudaError_t err = b->words.reserve(kBatchWords * sizeof(uint32_t));
    if (err == cudaSuccess && b->count == 0) err = cudaMemset(b->words.ptr, 0, kBatchWords * sizeof(uint32_t));
    if (err == cudaSuccess) err = b->recs.reserve((size_t)V * count * 48);
    if (err == cudaSuccess) err = b->grads.reserve((size_t)V * count * kGradWords * sizeof(float));
    if (err == cudaSuccess) err = b->projFlags.reserve((size_t)std::max(1u, gaussBlocks * V) * 8);
    if (err == cudaSuccess) err = b->ranges.reserve((size_t)std::max(1u, b->totalTiles) * 8);
    if (err == cudaSuccess) err = b->tileOrder.reserve((size_t)std::max(1u, b->totalTiles) * 4);
    if (err == cudaSuccess) err = b->sortHist.reserve(sortHistWords() * sizeof(uint32_t));
    if (err == cudaSuccess) err = b->viewsDev.reserve(std::max<size_t>(1, b->views.size()) * sizeof(BatchView));
    if (err == cudaSuccess) err = b->seen.reserve(std::max<size_t>(1, (size_t)V * count));
    if (err == cudaSuccess) err = b->adjointOrder.reserve((size_t)std::max(1u, count) * 4);
    if (err == cudaSuccess) err = b->adjointViews.reserve((size_t)std::max(1u, count) * 8);
    if (err == cudaSuccess) err = b->groupWords.reserve(2 * 256 * 4);
    if (err != cudaSuccess) return failCuda(err, "reserving the batch's scratch");
    b->count = count;
    return ATH_OK;
}

// Sizes the pairs: the projection alone, its total read back (the one host read,
// made before capture), and the pair buffers grown to 1.15 times it.
ath_status sizePairs(ath_batch* b, const ath_mixed_params& P, cudaStream_t stream) {
    ath_param_grads none{};
    // the projection's look-back words start "not ready": a buffer just allocated may
    // hold another batch's words, whose epoch tags the look-back would take as ready
    cudaError_t err = cudaMemsetAsync(b->projFlags.ptr, 0, b->projFlags.bytes, stream);
    if (err == cudaSuccess) err = enqueueStep(b, P, nullptr, nullptr, nullptr, none, stream, true);
    uint32_t w[kBatchWords];
    if (err == cudaSuccess) err = cudaMemcpyAsync(w, b->words.ptr, sizeof(w), cudaMemcpyDeviceToHost, stream);
    if (err == cudaSuccess) err = cudaStreamSynchronize(stream);
    if (err != cudaSuccess) return failCuda(err, "sizing the batch's pairs");
    if (w[kBatchStatus] & kStatusLookbackTimeout) return fail(ATH_E_TIMEOUT, "a look-back wait gave up while sizing");
    const uint64_t pairs = (uint64_t)w[kBatchPairsLo] | ((uint64_t)w[kBatchPairsHi] << 32);
    const uint64_t want = pairs + pairs / 7 + 65536;
    if (want > 0xFFFFFFFFull) return fail(ATH_E_UNSUPPORTED, "more than 2^32 pairs in one batched step");
    // The pairs' form: packed with the 24-bit depth key while tile, depth and Gaussian
    // bits fit in 64; else packed with the depth's exponent byte renumbered from a base
    // two below the least exponent seen here, in the fewest bits that hold two above
    // the greatest (a step whose depths leave that range reports it, and the next
    // step plans again); else wide.
    const uint32_t slot = bitsForValues(std::max<uint64_t>(b->count, 2));
    const uint32_t eLo = w[kBatchExpMin], eHi = w[kBatchExpMax];
    uint32_t depthBits = 24, expBase = 0;
    auto renumbered = [&]() {
        const uint32_t lo = eLo <= eHi && eLo > 2 ? eLo - 2 : 0;
        const uint32_t hi = eLo <= eHi ? std::min(255u, eHi + 2) : 0;
        const uint32_t e = bitsForValues(hi - lo + 1);
        if (16 + e + slot + b->tileBits > 64) return false;
        depthBits = 16 + e;
        expBase = lo;
        return true;
    };
    bool wide;
    if (b->keyMode == 2) {
        wide = true;
    } else if (b->keyMode == 1) {
        wide = false;
    } else if (b->keyMode == 3) {
        if (!renumbered())
            return fail(ATH_E_UNSUPPORTED, "tiles, the renumbered depth and the Gaussian index exceed 64 bits "
                                           "(packed keys asked for; the wide form has no such limit)");
        wide = false;
    } else {
        // packed with the 24-bit depth key while it fits, unless the renumbered depth
        // sorts in fewer passes (C1: 14 tile bits + 20 depth bits sort in four passes
        // of 9, 9, 8, 8 bits; with the 24-bit key, 38 bits take five); else renumbered; else wide
        const bool packedFits = 24 + slot + b->tileBits <= 64;
        if (renumbered() && (!packedFits || sortPasses(depthBits + b->tileBits) < sortPasses(24 + b->tileBits))) {
            wide = false;
        } else {
            wide = !packedFits;
            depthBits = 24;
            expBase = 0;
        }
    }
    b->planned = true;
    b->planWide = wide;
    b->depthBits = wide ? 24u : depthBits;
    b->expBase = wide ? 0u : expBase;
    if (want > b->capacity || !b->pairs[0].ptr || (wide && !b->values[0].ptr)) {
        const uint64_t room = std::max<uint64_t>(want, b->capacity);
        for (int k = 0; k < 2; ++k) {
            if ((err = b->pairs[k].reserve((size_t)room * 8)) != cudaSuccess) return failCuda(err, "reserving the pairs");
            if (wide && (err = b->values[k].reserve((size_t)room * 4)) != cudaSuccess)
                return failCuda(err, "reserving the pairs' Gaussians");
        }
        b->capacity = room;
    }
    const uint32_t bits = b->depthBits + b->tileBits;
    err = b->sortFlags.reserve(sortFlagWords((uint32_t)b->capacity, bits) * 8);
    if (err != cudaSuccess) return failCuda(err, "reserving the sort's look-back words");
    // the blends' live bits (written by the forward before the adjoint reads them; no clearing)
    err = b->live.reserve(liveWords(b->capacity, b->totalTiles, b->tile) * sizeof(uint32_t));
    if (err != cudaSuccess) return failCuda(err, "reserving the blends' live bits");
    // the look-back words carry epochs: start them all at "not ready"
    err = cudaMemsetAsync(b->sortFlags.ptr, 0, sortFlagWords((uint32_t)b->capacity, bits) * 8, stream);
    if (err == cudaSuccess) err = cudaMemsetAsync(b->words.ptr, 0, kBatchWords * sizeof(uint32_t), stream);
    if (err == cudaSuccess) err = cudaMemsetAsync(b->projFlags.ptr, 0, b->projFlags.bytes, stream);
    if (err != cudaSuccess) return failCuda(err, "clearing the batch's look-back words");
    b->resize = false;
    return ATH_OK;
}

}   // namespace

extern "C" ath_status ath_params_to_mixed(const ath_params* in, void* shLow, void* shHigh, float* shScale,
                                          void* stream) {
    if (!in || (in->count && (!in->sh || !shLow || !shHigh || !shScale)))
        return fail(ATH_E_INVALID_ARGUMENT, "ath_params_to_mixed: null argument");
    if (in->sh_degree > 3 || in->sh_stride < 3u + 3u * (in->sh_degree >= 3 ? 15u : in->sh_degree == 2 ? 8u : in->sh_degree == 1 ? 3u : 0u))
        return fail(ATH_E_INVALID_ARGUMENT, "ath_params_to_mixed: sh_degree / sh_stride");
    if (in->count == 0) return ATH_OK;
    toMixedKernel<<<(in->count + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        in->sh, in->count, in->sh_stride, in->sh_degree, static_cast<__nv_bfloat16*>(shLow),
        static_cast<__nv_fp8_e4m3*>(shHigh), shScale);
    const cudaError_t err = cudaGetLastError();
    return err == cudaSuccess ? ATH_OK : failCuda(err, "ath_params_to_mixed");
}

extern "C" ath_status ath_batch_create(ath_batch** out) {
    if (!out) return fail(ATH_E_INVALID_ARGUMENT, "ath_batch_create: null output");
    *out = nullptr;
    ath_batch* b = new (std::nothrow) ath_batch();
    if (!b) return fail(ATH_E_OUT_OF_MEMORY, "ath_batch_create: host allocation failed");
    cudaError_t err = cudaGetDevice(&b->device);
    if (err == cudaSuccess) err = cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, b->device);
    if (err == cudaSuccess) err = sortPrepare();
    if (err == cudaSuccess) err = cudaStreamCreateWithFlags(&b->captureStream, cudaStreamNonBlocking);
    if (err != cudaSuccess) {
        delete b;
        return failCuda(err, "ath_batch_create");
    }
    *out = b;
    return ATH_OK;
}

extern "C" void ath_batch_destroy(ath_batch* b) {
    if (!b) return;
    dropGraph(b);
    if (b->captureStream) cudaStreamDestroy(b->captureStream);
    delete b;
}

extern "C" ath_status ath_batch_set_views(ath_batch* b, const ath_view* views, uint32_t count,
                                          const ath_settings* settings) {
    if (!b || (count && !views)) return fail(ATH_E_INVALID_ARGUMENT, "ath_batch_set_views: null argument");
    if (count == 0 || count > kMaxBatchViews)
        return fail(ATH_E_INVALID_ARGUMENT, "ath_batch_set_views: 1 to 256 views a batch");
    uint64_t pixels = 0;
    for (uint32_t v = 0; v < count; ++v) {
        if (views[v].width == 0 || views[v].height == 0) return fail(ATH_E_INVALID_ARGUMENT, "a view needs a size");
        pixels += (uint64_t)views[v].width * views[v].height;
    }
    if (pixels > 0xFFFFFFFFull) return fail(ATH_E_UNSUPPORTED, "more than 2^32 pixels in one batch");
    b->projections.clear();
    b->widths.clear();
    b->heights.clear();
    for (uint32_t v = 0; v < count; ++v) {
        b->projections.push_back(views[v].projection);
        b->widths.push_back(views[v].width);
        b->heights.push_back(views[v].height);
    }
    if (settings) {
        for (int k = 0; k < 4; ++k) b->bg[k] = settings->background[k];
        b->shLimit = settings->max_sh_degree;
        b->antialias = settings->antialias_override >= 0 ? (uint32_t)(settings->antialias_override != 0)
                                                         : (uint32_t)(settings->antialias != 0);
        b->depthMode = settings->depth_mode;
        b->depthThreshold = settings->depth_threshold;
    }
    buildViews(b);
    b->resize = true;
    dropGraph(b);
    return ATH_OK;
}

extern "C" ath_status ath_batch_set_key_mode(ath_batch* b, uint32_t mode) {
    if (!b) return fail(ATH_E_INVALID_ARGUMENT, "ath_batch_set_key_mode: null batch");
    if (mode > 3) return fail(ATH_E_INVALID_ARGUMENT, "ath_batch_set_key_mode: mode must be 0, 1, 2 or 3");
    if (mode != b->keyMode) {
        b->keyMode = mode;
        b->resize = true;   // the next step sizes (and, for wide pairs, allocates) again
        dropGraph(b);
    }
    return ATH_OK;
}

extern "C" ath_status ath_batch_set_tuning(ath_batch* b, uint32_t tile, uint32_t blockBatch) {
    if (!b) return fail(ATH_E_INVALID_ARGUMENT, "ath_batch_set_tuning: null handle");
    if ((tile != 8 && tile != 16 && tile != 32) ||
        (blockBatch != 64 && blockBatch != 128 && blockBatch != 256 && blockBatch != 512))
        return fail(ATH_E_INVALID_ARGUMENT, "ath_batch_set_tuning: tile 8, 16 or 32; block batch 64, 128, 256 or 512");
    if (tile != b->tile || blockBatch != b->blockBatch) {
        b->tile = tile;
        b->blockBatch = blockBatch;
        if (!b->projections.empty()) buildViews(b);
        b->resize = true;
        dropGraph(b);
    }
    return ATH_OK;
}

extern "C" ath_status ath_batch_pixels(ath_batch* b, uint32_t* pixels) {
    if (!b || !pixels) return fail(ATH_E_INVALID_ARGUMENT, "ath_batch_pixels: null argument");
    *pixels = b->totalPixels;
    return ATH_OK;
}

namespace {

// A training step (target, loss and gradients given) or a render (all three
// null), checked, its buffers sized, captured once for its arrays and replayed.
ath_status runStep(ath_batch* b, const ath_mixed_params* params, const float* target, float* colour, float* loss,
                   ath_param_grads* grads, float* depth, void* streamPtr, const char* what,
                   cudaEvent_t targetReady = nullptr) {
    if (b->views.empty()) return fail(ATH_E_INVALID_ARGUMENT, std::string(what) + ": no views (ath_batch_set_views)");
    const ath_mixed_params& P = *params;
    if (P.count && (!P.means || !P.scales || !P.quats || !P.sh_low || !P.sh_high || !P.sh_scale))
        return fail(ATH_E_INVALID_ARGUMENT, std::string(what) + ": a cloud needs every array of the mixed layout");
    if (P.sh_degree > 3) return fail(ATH_E_INVALID_ARGUMENT, std::string(what) + ": sh_degree must be 0..3");
    if ((reinterpret_cast<uintptr_t>(P.sh_low) & 7u) || (reinterpret_cast<uintptr_t>(P.sh_high) & 3u) ||
        (reinterpret_cast<uintptr_t>(P.means) & 15u) || (reinterpret_cast<uintptr_t>(P.scales) & 15u) ||
        (reinterpret_cast<uintptr_t>(P.quats) & 15u))
        return fail(ATH_E_INVALID_ARGUMENT, std::string(what) + ": a cloud array is not aligned to its element");
    const uint32_t slotBits = bitsForValues(std::max<uint64_t>(P.count, 2));
    if (b->keyMode == 1 && 24 + slotBits + b->tileBits > 64)
        return fail(ATH_E_UNSUPPORTED, std::string(what) + ": tiles, depth key and Gaussian index exceed 64 bits "
                                       "(packed keys asked for; the wide form has no such limit)");
    if (b->keyMode == 3 && 17 + slotBits + b->tileBits > 64)
        return fail(ATH_E_UNSUPPORTED, std::string(what) + ": tiles, a renumbered depth and Gaussian index exceed "
                                       "64 bits (packed keys asked for; the wide form has no such limit)");
    if (24 + b->tileBits > 64)
        return fail(ATH_E_UNSUPPORTED, std::string(what) + ": more than 2^40 tiles");
    cudaStream_t stream = static_cast<cudaStream_t>(streamPtr);
    ath_status st = ATH_OK;
    // the buffers a view, a tile or a Gaussian holds: grown whenever the cloud, the
    // views or the tile size changed (set_views and set_tuning mark a resize)
    if (P.count != b->count || b->resize) {
        if ((st = reserveBatch(b, P.count)) != ATH_OK) return st;
        b->resize = true;
        dropGraph(b);
    }
    placeCloud(b, P.object_to_world);
    cudaError_t err = cudaMemcpyAsync(b->viewsDev.ptr, b->views.data(), b->views.size() * sizeof(BatchView),
                                      cudaMemcpyHostToDevice, stream);
    if (err != cudaSuccess) return failCuda(err, "ath_batch_train_step");
    if (b->resize) {
        if ((st = sizePairs(b, P, stream)) != ATH_OK) return st;
        dropGraph(b);
    }
    const uintptr_t key[14] = {(uintptr_t)P.means, (uintptr_t)P.scales, (uintptr_t)P.quats, (uintptr_t)P.sh_low,
                               (uintptr_t)P.sh_high, (uintptr_t)P.sh_scale, (uintptr_t)target, (uintptr_t)colour,
                               (uintptr_t)loss, (uintptr_t)(grads ? grads->means : nullptr),
                               (uintptr_t)(grads ? grads->sh : nullptr), (uintptr_t)P.count, (uintptr_t)depth,
                               (uintptr_t)targetReady};
    int slot = -1;
    for (int k = 0; k < ath_batch::kGraphs && slot < 0; ++k)
        if (b->exec[k] && std::memcmp(key, b->graphKey[k], sizeof(key)) == 0) slot = k;
    if (slot < 0) {
        slot = b->nextGraph;
        b->nextGraph = (b->nextGraph + 1) % ath_batch::kGraphs;
        if (b->exec[slot]) cudaGraphExecDestroy(b->exec[slot]);
        b->exec[slot] = nullptr;
        // Capture on the batch's own stream (the caller's may be the legacy one),
        // ordered after the caller's work so far.
        cudaEvent_t ready;
        err = cudaEventCreateWithFlags(&ready, cudaEventDisableTiming);
        if (err == cudaSuccess) err = cudaEventRecord(ready, stream);
        if (err == cudaSuccess) err = cudaStreamWaitEvent(b->captureStream, ready, 0);
        if (err == cudaSuccess) err = cudaStreamSynchronize(b->captureStream);
        cudaEventDestroy(ready);
        cudaGraph_t graph = nullptr;
        if (err == cudaSuccess) err = cudaStreamBeginCapture(b->captureStream, cudaStreamCaptureModeThreadLocal);
        if (err == cudaSuccess) {
            ath_param_grads g = grads ? *grads : ath_param_grads{};
            const cudaError_t enq =
                enqueueStep(b, P, target, reinterpret_cast<float4*>(colour), loss, g, b->captureStream, false,
                            nullptr, depth, targetReady);
            err = cudaStreamEndCapture(b->captureStream, &graph);
            if (enq != cudaSuccess) err = enq;
        }
        if (err == cudaSuccess) err = cudaGraphInstantiate(&b->exec[slot], graph, 0);
        if (graph) cudaGraphDestroy(graph);
        if (err != cudaSuccess) {
            b->exec[slot] = nullptr;
            return failCuda(err, "capturing the batched step");
        }
        std::memcpy(b->graphKey[slot], key, sizeof(key));
    }
    err = cudaGraphLaunch(b->exec[slot], stream);
    if (err != cudaSuccess) return failCuda(err, "launching the batched step");
    return ATH_OK;
}

}   // namespace

extern "C" ath_status ath_batch_train_step(ath_batch* b, const ath_mixed_params* params, const float* target,
                                           float* colour, float* loss, ath_param_grads* grads, void* streamPtr) {
    return ath_batch_train_step_after(b, params, target, nullptr, colour, loss, grads, streamPtr);
}

extern "C" ath_status ath_batch_train_step_after(ath_batch* b, const ath_mixed_params* params, const float* target,
                                                 void* targetReady, float* colour, float* loss, ath_param_grads* grads,
                                                 void* streamPtr) {
    if (!b || !params || !target || !colour || !loss)
        return fail(ATH_E_INVALID_ARGUMENT, "ath_batch_train_step: null argument");
    // with gradient buckets the buckets' arrays receive the gradients; an empty cloud
    // has no gradient rows, so its gradient arrays may be null
    if (b->bucketGrads.empty() &&
        (!grads || (params->count && (!grads->means || !grads->scales || !grads->quats || !grads->sh))))
        return fail(ATH_E_INVALID_ARGUMENT, "ath_batch_train_step: null gradient arrays");
    if (!b->bucketGrads.empty() && params->count != b->bucketCount)
        return fail(ATH_E_INVALID_ARGUMENT, "ath_batch_train_step: the gradient buckets were set for " +
                                                std::to_string(b->bucketCount) + " Gaussians, the cloud has " +
                                                std::to_string(params->count));
    return runStep(b, params, target, colour, loss, b->bucketGrads.empty() ? grads : nullptr, nullptr, streamPtr,
                   "ath_batch_train_step", static_cast<cudaEvent_t>(targetReady));
}

// Bucket k of `buckets` over `count` Gaussians: consecutive ranges in whole blocks
// of the projection adjoint (128 Gaussians), their sizes differing by at most one block.
extern "C" ath_status ath_gradient_bucket(uint32_t count, uint32_t buckets, uint32_t k, uint32_t* first,
                                          uint32_t* n) {
    if (!first || !n || buckets == 0 || k >= buckets)
        return fail(ATH_E_INVALID_ARGUMENT, "ath_gradient_bucket: bucket outside 0 .. buckets - 1");
    const uint64_t units = ((uint64_t)count + 127) / 128;
    const uint64_t base = units / buckets, extra = units % buckets;
    const uint64_t start = 128 * (k * base + std::min<uint64_t>(k, extra));
    const uint64_t end = std::min<uint64_t>(count, start + 128 * (base + (k < extra ? 1 : 0)));
    *first = (uint32_t)std::min<uint64_t>(start, count);
    *n = (uint32_t)(end > start ? end - start : 0);
    return ATH_OK;
}

extern "C" ath_status ath_batch_set_buckets(ath_batch* b, uint32_t count, uint32_t buckets,
                                            const ath_param_grads* grads, void* const* events) {
    if (!b) return fail(ATH_E_INVALID_ARGUMENT, "ath_batch_set_buckets: null handle");
    if (buckets && !grads) return fail(ATH_E_INVALID_ARGUMENT, "ath_batch_set_buckets: null bucket arrays");
    if (buckets > 1024) return fail(ATH_E_INVALID_ARGUMENT, "ath_batch_set_buckets: at most 1024 buckets");
    for (uint32_t k = 0; k < buckets; ++k) {
        uint32_t first = 0, n = 0;
        ath_gradient_bucket(count, buckets, k, &first, &n);
        if (n && (!grads[k].means || !grads[k].scales || !grads[k].quats || !grads[k].sh))
            return fail(ATH_E_INVALID_ARGUMENT, "ath_batch_set_buckets: bucket " + std::to_string(k) +
                                                    " needs its four gradient arrays");
    }
    b->bucketGrads.assign(grads, grads + buckets);
    b->bucketEvents.clear();
    if (buckets && events)
        for (uint32_t k = 0; k < buckets; ++k) b->bucketEvents.push_back(static_cast<cudaEvent_t>(events[k]));
    b->bucketCount = count;
    dropGraph(b);   // the arrays and events are part of the captured step
    return ATH_OK;
}

extern "C" ath_status ath_batch_render(ath_batch* b, const ath_mixed_params* params, float* colour, float* depth,
                                       void* streamPtr) {
    if (!b || !params || !colour) return fail(ATH_E_INVALID_ARGUMENT, "ath_batch_render: null argument");
    return runStep(b, params, nullptr, colour, nullptr, nullptr, depth, streamPtr, "ath_batch_render");
}

extern "C" ath_status ath_batch_check(ath_batch* b, ath_batch_stats* out, void* streamPtr) {
    if (!b || !out) return fail(ATH_E_INVALID_ARGUMENT, "ath_batch_check: null argument");
    if (!b->words.ptr) return fail(ATH_E_NOT_FOUND, "ath_batch_check: no step has run");
    cudaStream_t stream = static_cast<cudaStream_t>(streamPtr);
    uint32_t w[kBatchWords];
    cudaError_t err = cudaMemcpyAsync(w, b->words.ptr, sizeof(w), cudaMemcpyDeviceToHost, stream);
    if (err == cudaSuccess) err = cudaStreamSynchronize(stream);
    if (err != cudaSuccess) return failCuda(err, "ath_batch_check");
    out->pairs = (uint64_t)w[kBatchPairsLo] | ((uint64_t)w[kBatchPairsHi] << 32);
    out->kept = w[kBatchKept];
    auto word64 = [&](uint32_t k) { return (uint64_t)w[k] | ((uint64_t)w[k + 1] << 32); };
    out->evaluated = word64(kBatchEvaluated);
    out->blended = word64(kBatchBlended);
    out->adjoint_visited = word64(kBatchAdjVisited);
    out->adjoint_live = word64(kBatchAdjLive);
    out->warp_visits_forward = word64(kBatchFwdVisits);
    out->warp_visits_adjoint = word64(kBatchAdjVisits);
    out->warp_visits_adjoint_summed = word64(kBatchAdjSummed);
    out->records_staged = word64(kBatchStaged);
    out->degenerate = w[kBatchDegenerate];
    out->tile = b->tile;
    out->block_batch = b->blockBatch;
    out->capacity = b->capacity;
    if (w[kBatchStatus]) {
        const uint32_t bits = w[kBatchStatus];
        cudaMemsetAsync(static_cast<uint32_t*>(b->words.ptr) + kBatchStatus, 0, sizeof(uint32_t), stream);
        if (bits & kStatusPairOverflow) {
            b->resize = true;   // the next step sizes the pairs again
            return fail(ATH_E_CAPACITY, "a step had more pairs than its buffers; the next step grows them");
        }
        if (bits & kStatusDepthRange) {
            b->resize = true;   // the next step plans the pairs' depth field again
            return fail(ATH_E_CAPACITY, "a step's depths left the exponent range its pair keys were planned for "
                                        "(that step's order is not valid); the next step plans them again");
        }
        if (bits & kStatusLookbackTimeout) return fail(ATH_E_TIMEOUT, "a look-back wait of a batched step gave up");
        return fail(ATH_E_INTERNAL, "a batched step met an index outside its buffers");
    }
    return ATH_OK;
}

extern "C" ath_status ath_batch_time_stages(ath_batch* b, const ath_mixed_params* params, const float* target,
                                            float* colour, float* loss, ath_param_grads* grads, float ms[5],
                                            void* streamPtr) {
    // A step as ath_batch_train_step enqueues it, uncaptured, with events between
    // its stages, waited for: project+emit, sort, ranges, blends (forward, loss and
    // adjoint in one kernel), projection adjoint. The blends' work is counted in a step
    // run just before on the same inputs (the counting kernel is slower), so the timed
    // step runs the kernels a captured step runs.
    if (!b || !params || !grads || !ms) return fail(ATH_E_INVALID_ARGUMENT, "ath_batch_time_stages: null argument");
    ath_status st = ath_batch_train_step(b, params, target, colour, loss, grads, streamPtr);   // sized and placed
    if (st != ATH_OK) return st;
    cudaStream_t stream = static_cast<cudaStream_t>(streamPtr);
    cudaEvent_t marks[6];
    for (auto& e : marks) cudaEventCreate(&e);
    ath_param_grads g = *grads;
    // the blends' work counts start at zero for the counted step (the captured steps leave them)
    uint32_t* words = static_cast<uint32_t*>(b->words.ptr);
    cudaError_t err = cudaMemsetAsync(words + kBatchEvaluated, 0, 2 * sizeof(uint32_t), stream);
    if (err == cudaSuccess)
        err = cudaMemsetAsync(words + kBatchBlended, 0, (kBatchStaged + 2 - kBatchBlended) * sizeof(uint32_t),
                              stream);
    if (err == cudaSuccess)
        err = enqueueStep(b, *params, target, reinterpret_cast<float4*>(colour), loss, g, stream, false, nullptr,
                          nullptr, nullptr, true);
    if (err == cudaSuccess)
        err = enqueueStep(b, *params, target, reinterpret_cast<float4*>(colour), loss, g, stream, false, marks);
    if (err == cudaSuccess) err = cudaEventSynchronize(marks[5]);
    for (int k = 0; k < 5 && err == cudaSuccess; ++k) cudaEventElapsedTime(&ms[k], marks[k], marks[k + 1]);
    for (auto& e : marks) cudaEventDestroy(e);
    return err == cudaSuccess ? ATH_OK : failCuda(err, "ath_batch_time_stages");
}

extern "C" ath_status ath_batch_buffers_of(ath_batch* b, ath_batch_buffers* out, void* streamPtr) {
    if (!b || !out) return fail(ATH_E_INVALID_ARGUMENT, "ath_batch_buffers_of: null argument");
    if (!b->words.ptr || !b->pairs[0].ptr) return fail(ATH_E_NOT_FOUND, "ath_batch_buffers_of: no step has run");
    uint32_t w[kBatchWords];
    cudaError_t err = cudaMemcpyAsync(w, b->words.ptr, sizeof(w), cudaMemcpyDeviceToHost, static_cast<cudaStream_t>(streamPtr));
    if (err == cudaSuccess) err = cudaStreamSynchronize(static_cast<cudaStream_t>(streamPtr));
    if (err != cudaSuccess) return failCuda(err, "ath_batch_buffers_of");
    out->pairs = (uint64_t)w[kBatchPairsLo] | ((uint64_t)w[kBatchPairsHi] << 32);
    out->key_shift = b->lastDepthBits + b->lastSlotBits;
    out->depth_bits = b->lastDepthBits;
    out->exp_base = b->lastExpBase;
    out->slot_bits = b->lastSlotBits;
    out->sorted_values = b->lastWide ? static_cast<const uint32_t*>(b->values[b->lastSorted].ptr) : nullptr;
    out->total_tiles = b->totalTiles;
    out->views = (uint32_t)b->views.size();
    out->sorted_pairs = static_cast<const uint64_t*>(b->pairs[b->lastSorted].ptr);
    out->ranges = static_cast<const uint32_t*>(b->ranges.ptr);
    out->tile_bases = b->tileBases.data();
    return ATH_OK;
}

extern "C" ath_status ath_batch_tune(ath_batch* b, const ath_mixed_params* params, const float* target,
                                     float* colour, float* loss, ath_param_grads* grads, uint32_t repeats,
                                     ath_batch_stats* best, void* streamPtr) {
    if (!b || !params) return fail(ATH_E_INVALID_ARGUMENT, "ath_batch_tune: null argument");
    cudaStream_t stream = static_cast<cudaStream_t>(streamPtr);
    const uint32_t tiles[3] = {32, 16, 8}, batches[4] = {64, 128, 256, 512};
    float bestMs = 1e30f;
    uint32_t bestTile = b->tile, bestBatch = b->blockBatch;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    for (uint32_t t : tiles) {
        for (uint32_t nb : batches) {
            ath_status st = ath_batch_set_tuning(b, t, nb);
            if (st == ATH_OK) st = ath_batch_train_step(b, params, target, colour, loss, grads, streamPtr);
            // a setting that does not fit (too many tile bits for packed keys, or its pairs
            // past the memory) is skipped; any other failure ends the tuning
            if (st == ATH_E_UNSUPPORTED || st == ATH_E_OUT_OF_MEMORY) continue;
            if (st != ATH_OK) {
                cudaEventDestroy(e0);
                cudaEventDestroy(e1);
                return st;
            }
            cudaEventRecord(e0, stream);
            for (uint32_t r = 0; r < std::max(repeats, 1u); ++r)
                st = ath_batch_train_step(b, params, target, colour, loss, grads, streamPtr);
            cudaEventRecord(e1, stream);
            cudaEventSynchronize(e1);
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, e0, e1);
            ath_batch_stats s{};
            if (st == ATH_OK && ath_batch_check(b, &s, streamPtr) == ATH_OK && ms < bestMs) {
                bestMs = ms;
                bestTile = t;
                bestBatch = nb;
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    // the pair buffers grew to the setting with the most pairs; size them again for the one kept
    // (the sort's grid follows their capacity)
    cudaStreamSynchronize(stream);
    dropGraph(b);
    for (int k = 0; k < 2; ++k) {
        b->pairs[k].release();
        b->values[k].release();
    }
    b->capacity = 0;
    b->resize = true;
    ath_status st = ath_batch_set_tuning(b, bestTile, bestBatch);
    if (st == ATH_OK) st = ath_batch_train_step(b, params, target, colour, loss, grads, streamPtr);
    if (st == ATH_OK && best) st = ath_batch_check(b, best, streamPtr);
    if (best) best->ms_per_step = bestMs / (float)std::max(repeats, 1u);
    return st;
}
