// Stage (d): per-tile front-to-back blending -- splat/splat_blend.slang:236-578
// (splatBlend = blendPixel<composite=false, matte=false, traced=false>) -- with
// the P layer (usd/aov_position.slang:34-52) as its epilogue.
//
// One block a 16x16 tile, one thread a pixel. The tile's records are staged in
// shared memory 256 at a time (:287-312); a pixel stops at T < 1e-4 after
// accumulating (:501-505); the block stops loading once every pixel is done,
// counted with a block-wide ballot (__syncthreads_count). Per pixel the walk
// is sequential in the tile's (depth key, slot) order, so the result is the
// CPU restatement's to the bit (built with --fmad=false; see splat_math.cuh).
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "kernels.h"
#include "raster_types.cuh"
#include "splat_math.cuh"

namespace ath {
namespace {

constexpr uint32_t kBlendThreads = kTile * kTile;
constexpr float kColourGradScale = 256.0f;   // frame.slang:36
constexpr uint32_t kCryptoSlots = 6;         // splat_blend.slang:82

// A pixel's Cryptomatte ranks (splat_blend.slang:88-143): the ids that covered
// it most and their summed weights. Id 0 names nothing and is never kept; a full
// list gives its lightest slot up to a heavier id. Written ranked by weight,
// descending (a stable insertion sort), as 3 float4 (id bits, weight, id bits,
// weight).
// The trace's list (splat_trace.slang:33-128): the kTraceSlots heaviest splats
// of a pixel's walk by weight, the lightest rank kept so that a splat too light
// for the list costs one comparison, and everything the walk blended.
constexpr uint32_t kTraceSlots = 4;
constexpr uint32_t kTraceWords = kTraceSlots * 2 + kTraceSlots / 2 + 1;
constexpr uint32_t kTraceNone = 0xFFFFFFFFu, kTraceEmpty = 0xFFFFFFFEu;

__device__ __forceinline__ uint32_t halfBits(float v) { return (uint32_t)__half_as_ushort(__float2half_rn(v)); }

struct TraceList {
    uint32_t slots[kTraceSlots];
    float weights[kTraceSlots];
    float total, floor;
    uint32_t lightest;

    __device__ __forceinline__ void clear() {
#pragma unroll
        for (uint32_t k = 0; k < kTraceSlots; ++k) {
            slots[k] = kTraceNone;
            weights[k] = 0.0f;
        }
        total = floor = 0.0f;
        lightest = 0;
    }
    // a splat heavier than the lightest rank takes its place
    __device__ __forceinline__ void enter(uint32_t slot, float weight) {
#pragma unroll
        for (uint32_t k = 0; k < kTraceSlots; ++k)
            if (k == lightest) {
                slots[k] = slot;
                weights[k] = weight;
            }
        lightest = 0;
        float w = weights[0];
#pragma unroll
        for (uint32_t k = 1; k < kTraceSlots; ++k)
            if (weights[k] < w) {
                lightest = k;
                w = weights[k];
            }
        floor = w;
    }
    // planes of `pixels` words: the slots heaviest first, their view depths (as
    // the floats' bits), the weights as halves two a word, and (rest, under) as
    // halves; a pixel nothing reached writes kTraceEmpty in its first word alone
    __device__ void write(uint32_t* trace, uint32_t at, uint32_t pixels, float under,
                          const float4* __restrict__ recs) const {
        if (!(total > 0.0f) && !(under > 0.0f)) {
            trace[at] = kTraceEmpty;
            return;
        }
        uint32_t order[kTraceSlots];
#pragma unroll
        for (uint32_t k = 0; k < kTraceSlots; ++k) order[k] = k;
        for (uint32_t i = 1; i < kTraceSlots; ++i) {
            const uint32_t pick = order[i];
            uint32_t j = i;
            while (j > 0 && weights[order[j - 1]] < weights[pick]) {
                order[j] = order[j - 1];
                --j;
            }
            order[j] = pick;
        }
        float held = 0.0f;
        for (uint32_t k = 0; k < kTraceSlots; ++k) {
            const uint32_t from = order[k];
            const bool some = weights[from] > 0.0f;
            trace[k * pixels + at] = some ? slots[from] : kTraceNone;
            trace[(kTraceSlots + k) * pixels + at] = some ? __float_as_uint(recs[(size_t)slots[from] * 3].z) : 0u;
            held = held + weights[from];
        }
        for (uint32_t pair = 0; pair < kTraceSlots / 2; ++pair)
            trace[(kTraceSlots * 2 + pair) * pixels + at] =
                halfBits(weights[order[pair * 2]]) | (halfBits(weights[order[pair * 2 + 1]]) << 16);
        trace[(kTraceWords - 1) * pixels + at] = halfBits(fmaxf(total - held, 0.0f)) | (halfBits(fmaxf(under, 0.0f)) << 16);
    }
};

struct CryptoList {
    uint32_t ids[kCryptoSlots];
    float weights[kCryptoSlots];

    __device__ __forceinline__ void clear() {
#pragma unroll
        for (uint32_t k = 0; k < kCryptoSlots; ++k) {
            ids[k] = 0;
            weights[k] = 0.0f;
        }
    }
    __device__ __forceinline__ void add(uint32_t id, float weight) {
        if (weight <= 0.0f || id == 0) return;
        uint32_t lightest = 0;
        float lightestWeight = weights[0];
#pragma unroll
        for (uint32_t k = 0; k < kCryptoSlots; ++k) {
            if (ids[k] == id && weights[k] > 0.0f) {
                weights[k] += weight;
                return;
            }
            if (weights[k] < lightestWeight) {
                lightest = k;
                lightestWeight = weights[k];
            }
        }
#pragma unroll
        for (uint32_t k = 0; k < kCryptoSlots; ++k)
            if (k == lightest && weight > weights[k]) {
                ids[k] = id;
                weights[k] = weight;
            }
    }
    __device__ __forceinline__ void write(float4* out, uint32_t at, uint32_t pixels) const {
        uint32_t order[kCryptoSlots];
#pragma unroll
        for (uint32_t k = 0; k < kCryptoSlots; ++k) order[k] = k;
        for (uint32_t i = 1; i < kCryptoSlots; ++i) {
            const uint32_t pick = order[i];
            uint32_t j = i;
            while (j > 0 && weights[order[j - 1]] < weights[pick]) {
                order[j] = order[j - 1];
                --j;
            }
            order[j] = pick;
        }
        for (uint32_t layer = 0; layer < kCryptoSlots / 2; ++layer) {
            const uint32_t a = order[layer * 2], b = order[layer * 2 + 1];
            out[(size_t)layer * pixels + at] =
                make_float4(weights[a] > 0.0f ? __uint_as_float(ids[a]) : 0.0f, fmaxf(weights[a], 0.0f),
                            weights[b] > 0.0f ? __uint_as_float(ids[b]) : 0.0f, fmaxf(weights[b], 0.0f));
        }
    }
};

// kContribution: the contributionMode hooks of splat_blend.slang:364-407 (modes
// 1 to 4). kUnder: the composite over an opaque layer under the splats
// (:249-251,329-333,516-523,555-575): a pixel's walk stops at the first record
// at or behind the layer's depth, and the layer takes the rest of the pixel.
// The plain frame builds without either.
template <bool kContribution, bool kUnder, bool kMatte>
__global__ void __launch_bounds__(kBlendThreads)
    blendKernel(const FrameConst F, uint32_t pairs, uint32_t slots, const uint2* __restrict__ ranges,
                const uint32_t* __restrict__ pairValues, const float4* __restrict__ recs, float4* __restrict__ colour,
                float* __restrict__ depth, float4* __restrict__ position, float* __restrict__ finalT,
                uint32_t* __restrict__ lastContrib, uint32_t* __restrict__ status, Contribution contrib,
                Under under, Matte matte) {
    __shared__ float4 sScreen[kBlendThreads];
    __shared__ float4 sConic[kBlendThreads];
    __shared__ float4 sColour[kBlendThreads];
    __shared__ uint32_t sSlot[kContribution || kMatte ? kBlendThreads : 1];
    CryptoList list;
    if (kMatte) list.clear();
    TraceList trace;
    if (kMatte && matte.trace) trace.clear();

    const uint32_t tile = blockIdx.x;
    const uint32_t tx = tile % F.tilesX, ty = tile / F.tilesX;
    const uint32_t px = tx * kTile + (threadIdx.x % kTile);
    const uint32_t py = ty * kTile + (threadIdx.x / kTile);
    const bool inside = px < F.width && py < F.height;
    uint2 range = ranges[tile];
    if (range.y > pairs || range.x > range.y) {   // never, for ranges the sort wrote
        if (threadIdx.x == 0) atomicOr(status, kStatusIndexRange);
        range = make_uint2(0, 0);
    }
    const float pxc = (float)px + 0.5f, pyc = (float)py + 0.5f;
    const float underZ = kUnder && inside ? under.depth[py * F.width + px] : 0.0f;
    const bool underHit = kUnder && underZ > 0.0f;

    float r = 0.0f, g = 0.0f, bl = 0.0f;
    float T = 1.0f, depthSum = 0.0f, depthAt = -1.0f;
    float matteKnown = 0.0f, matteInside = 0.0f, matteUntold = 0.0f;   // the lifted matte's sums
    uint32_t last = 0;
    bool done = !inside;
    for (uint32_t first = range.x; first < range.y; first += kBlendThreads) {
        if (__syncthreads_count(done) == kBlendThreads) break;
        const uint32_t mine = first + threadIdx.x;
        if (mine < range.y) {
            uint32_t s = pairValues[mine];
            if (s >= slots) {
                atomicOr(status, kStatusIndexRange);
                s = 0;
            }
            if (kContribution || kMatte) sSlot[threadIdx.x] = s;
            sScreen[threadIdx.x] = recs[(size_t)s * 3 + 0];
            sConic[threadIdx.x] = recs[(size_t)s * 3 + 1];
            sColour[threadIdx.x] = recs[(size_t)s * 3 + 2];
        }
        __syncthreads();
        const uint32_t count = min(kBlendThreads, range.y - first);
        for (uint32_t j = 0; j < count && !done; ++j) {
            const float4 sc = sScreen[j];
            if (kUnder && underHit && sc.z >= underZ) {
                done = true;
                break;
            }
            const float4 k = sConic[j];
            const float dx = pxc - sc.x;
            const float dy = pyc - sc.y;
            const float power = ((k.x * dx) * dx + ((2.0f * k.y) * dx) * dy) + (k.z * dy) * dy;
            if (power > sc.w) continue;
            const float alpha = fminf(0.99f, falloffAlpha(fabsf(k.w), exp_f((-0.5f) * power)));
            if (alpha < kFaint) continue;
            const float weight = T * alpha;
            if (kContribution) {
                const uint32_t slot = sSlot[j];
                if (contrib.mode == 1u) {
                    atomicAdd(&contrib.words[slot], (uint32_t)(weight * 4096.0f + 0.5f));
                } else if (contrib.mode == 2u) {
                    // splat_blend.slang:366-380: the pixel with the splat taken away shows what is
                    // behind it, recovered from the whole frame; the squared change, capped at one,
                    // in 2^-24 into a 64-bit sum of two words (low, then its carries)
                    const uint32_t at = py * F.width + px;
                    const float4 whole = reinterpret_cast<const float4*>(contrib.finalColour)[at];
                    const float4 c = sColour[j];
                    const float after = fmaxf(T * (1.0f - alpha), 1.0e-4f);
                    const float cx = weight * (c.x - (whole.x - (r + weight * c.x)) / after);
                    const float cy = weight * (c.y - (whole.y - (g + weight * c.y)) / after);
                    const float cz = weight * (c.z - (whole.z - (bl + weight * c.z)) / after);
                    const float d2 = (cx * cx + cy * cy) + cz * cz;
                    const uint32_t add = (uint32_t)(fminf(d2, 1.0f) * 16777216.0f + 0.5f);
                    const uint32_t before = atomicAdd(&contrib.words[slot * 2], add);
                    if (before + add < before) atomicAdd(&contrib.words[slot * 2 + 1], 1u);
                } else if (contrib.mode == 3u) {
                    // splat_blend.slang:399-407: the weight, and the weight times the mask, in 1/1024
                    const uint32_t seen = (uint32_t)(weight * 1024.0f + 0.5f);
                    if (seen != 0u) {
                        atomicAdd(&contrib.words[slot * 2 + 1], seen);
                        const float m = fminf(fmaxf(contrib.liftMask[py * F.width + px], 0.0f), 1.0f);
                        const uint32_t within = (uint32_t)((weight * m) * 1024.0f + 0.5f);
                        if (within != 0u) atomicAdd(&contrib.words[slot * 2], within);
                    }
                } else {
                    const uint32_t at = py * F.width + px;
                    const float4 dl = reinterpret_cast<const float4*>(contrib.finalColour)[at];
                    const float dls[3] = {dl.x, dl.y, dl.z};
                    for (uint32_t ch = 0; ch < 3; ++ch) {
                        const float gc = (weight * dls[ch]) * kColourGradScale;
                        const int step = (int)floorf(gc + hash01((at * 3u + ch) ^ (slot * 2654435761u)));
                        if (step != 0) atomicAdd(&contrib.words[slot * 4 + ch], (uint32_t)step);
                    }
                    atomicAdd(&contrib.words[slot * 4 + 3], (uint32_t)(weight * kColourGradScale + 0.5f));
                }
            }
            if (kMatte && matte.out) list.add(matte.ids[sSlot[j]], weight);
            if (kMatte && matte.trace) {
                // splat_blend.slang:445-451
                trace.total = trace.total + weight;
                if (weight > trace.floor) trace.enter(sSlot[j], weight);
            }
            if (kMatte && matte.lifted) {
                // splat_blend.slang:423-435: the share a lift told the splat, or, for one no
                // lifting camera saw, its weight kept aside
                const uint32_t told = sSlot[j] * 2u;
                const uint32_t seen = matte.liftSums[told + 1u];
                if (seen != 0u) {
                    float share = (float)matte.liftSums[told] / (float)seen;
                    if (matte.hard) share = share > matte.threshold ? 1.0f : 0.0f;
                    matteKnown = matteKnown + weight;
                    matteInside = matteInside + weight * share;
                } else {
                    matteUntold = matteUntold + weight;
                }
            }
            const float4 c = sColour[j];
            r = r + weight * c.x;
            g = g + weight * c.y;
            bl = bl + weight * c.z;
            depthSum = depthSum + weight * sc.z;
            T = T * (1.0f - alpha);
            last = first - range.x + j + 1;
            if (depthAt < 0.0f && 1.0f - T >= F.depthThreshold) depthAt = sc.z;
            if (T < 1e-4f) done = true;
        }
    }
    if (!inside) return;
    const uint32_t at = py * F.width + px;
    const float coverage = 1.0f - T;
    float4 behind = make_float4(F.bg[0], F.bg[1], F.bg[2], F.bg[3]);
    if (kUnder && underHit) {
        behind = reinterpret_cast<const float4*>(under.colour)[at];
        depthSum = depthSum + T * underZ;
        if (depthAt < 0.0f) depthAt = underZ;
    }
    const float total = kUnder && underHit ? 1.0f : coverage;
    if (kMatte && matte.trace)   // splat_blend.slang:545-551: what closed the walk from behind is `under`
        trace.write(matte.trace, at, F.width * F.height, kUnder && underHit ? T : 0.0f, recs);
    if (kMatte && matte.lifted) {
        // splat_blend.slang:536-539: the untold weight at the share of the known
        const float share = matteKnown > 0.0f ? matteInside / matteKnown : 0.0f;
        matte.lifted[at] = fminf(fmaxf(matteInside + matteUntold * share, 0.0f), 1.0f);
    }
    if (kMatte && matte.out) {
        // what closed the walk takes the rest of the pixel (splat_blend.slang:525-534)
        list.add(kUnder && underHit && matte.underIds ? matte.underIds[at] : 0u, kUnder && underHit ? T : 0.0f);
        list.write(reinterpret_cast<float4*>(matte.out), at, F.width * F.height);
    }
    colour[at] = make_float4(r + T * behind.x, g + T * behind.y, bl + T * behind.z, coverage + T * behind.w);
    const float z = F.depthMode == 0 ? (total > 1e-6f ? depthSum / total : 0.0f) : fmaxf(depthAt, 0.0f);
    depth[at] = z;
    if (finalT) finalT[at] = T;
    if (lastContrib) lastContrib[at] = last;
    if (position) {
        // usd/aov_position.slang:40-51
        if (!(z > 0.0f)) {
            position[at] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        } else {
            const float scale = F.orthographic != 0 ? 1.0f : z;
            const float v0 = ((pxc - F.centreX) / F.focalX) * scale;
            const float v1 = ((pyc - F.centreY) / F.focalY) * scale;
            const float* m = F.viewToWorld;
            position[at] = make_float4(((m[0] * v0 + m[1] * v1) + m[2] * z) + m[3] * 1.0f,
                                       ((m[4] * v0 + m[5] * v1) + m[6] * z) + m[7] * 1.0f,
                                       ((m[8] * v0 + m[9] * v1) + m[10] * z) + m[11] * 1.0f, 1.0f);
        }
    }
}

}   // namespace

cudaError_t launchBlend(const FrameConst& F, uint32_t pairs, uint32_t slots, const uint2* ranges,
                        const uint32_t* pairValues, const float4* recs, float4* colour, float* depth, float4* position,
                        float* finalT, uint32_t* lastContrib, uint32_t* status, cudaStream_t stream,
                        const Contribution& contrib, const Under& under, const Matte& matte) {
    const uint32_t tiles = F.tilesX * F.tilesY;
    if (tiles == 0) return cudaSuccess;
#define ATH_BLEND(C_, U_, M_)                                                                          \
    blendKernel<C_, U_, M_><<<tiles, kBlendThreads, 0, stream>>>(F, pairs, slots, ranges, pairValues, recs, colour, \
                                                                depth, position, finalT, lastContrib, status,     \
                                                                contrib, under, matte)
    const bool c = contrib.mode != 0u, u = under.depth != nullptr,
               m = matte.out != nullptr || matte.lifted != nullptr || matte.trace != nullptr;
    if (m) {
        if (c && u) ATH_BLEND(true, true, true);
        else if (c) ATH_BLEND(true, false, true);
        else if (u) ATH_BLEND(false, true, true);
        else ATH_BLEND(false, false, true);
    } else {
        if (c && u) ATH_BLEND(true, true, false);
        else if (c) ATH_BLEND(true, false, false);
        else if (u) ATH_BLEND(false, true, false);
        else ATH_BLEND(false, false, false);
    }
#undef ATH_BLEND
    return cudaGetLastError();
}

}   // namespace ath
