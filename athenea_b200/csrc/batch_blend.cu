// The batched path's blends: a training step's forward blend, loss and blend
// adjoint in one persistent kernel over every view's tiles. This file builds
// with FMA contraction (the other kernels of the plain and batched paths do
// not): nothing here has to match the reference's FP32 to the bit, only the
// forward and the adjoint each other, and both are compiled alike. Which records
// a pixel blends is decided per pixel, the same way in both, whatever the tile
// size.
#include <cstdint>

#include <cuda_runtime.h>

#include "batch_kernels.cuh"

namespace ath {
namespace {

// A warp's box of pixels: 8x8, two pixels a lane.
constexpr uint32_t kBox = 8;
// The pixels a block takes of a tile: a span of kBlendSpan x kBlendSpan (or the
// whole tile when it is smaller), so that a block's barriers wait on fewer boxes
// and a span whose pixels are done stops staging the tile's records.
constexpr uint32_t kBlendSpan = 16;

// The footprint's half extents from the factored conic: the covariance's
// diagonal a' = cutoff (1/ca + fr^2/fs) and c' = cutoff / fs.
__device__ __forceinline__ void footprintExtent(float ca, float fr, float fs, float cutoff, float& ex, float& ey) {
    ex = ca > 0.0f && fs > 0.0f ? sqrtf(cutoff * (1.0f / ca + (fr * fr) / fs)) * 1.0001f + 1e-3f : 3.4e38f;
    ey = fs > 0.0f ? sqrtf(cutoff / fs) * 1.0001f + 1e-3f : 3.4e38f;
}

// Bit b set when box b of the tile (boxes row-major, T/8 a row) may hold a pixel
// centre inside the footprint: among the boxes whose pixel-centre columns and
// rows overlap the footprint's bounding box [cx - ex, cx + ex] x [cy - ey, cy + ey],
// those whose least power (minPowerOverBoxFactored) is within the cutoff.
// Conservative: extents and cutoff carry a margin over the per-pixel test's
// rounding.
template <uint32_t T>
__device__ __forceinline__ uint32_t boxMask(float tileX0, float tileY0, float4 screen, float ca, float fr, float fs) {
    constexpr int kAcross = (int)(T / kBox);
    float ex, ey;
    footprintExtent(ca, fr, fs, screen.w, ex, ey);
    // box column b holds pixel centres tileX0 + 8 b + 0.5 .. tileX0 + 8 b + 7.5
    const float x0 = (screen.x - ex) - (tileX0 + 0.5f), x1 = (screen.x + ex) - (tileX0 + 0.5f);
    const float y0 = (screen.y - ey) - (tileY0 + 0.5f), y1 = (screen.y + ey) - (tileY0 + 0.5f);
    const float lim = (float)kAcross;
    const int bx0 = (int)ceilf(clampf((x0 - 7.0f) * 0.125f, -1.0f, lim));
    const int bx1 = (int)floorf(clampf(x1 * 0.125f, -1.0f, lim));
    const int by0 = (int)ceilf(clampf((y0 - 7.0f) * 0.125f, -1.0f, lim));
    const int by1 = (int)floorf(clampf(y1 * 0.125f, -1.0f, lim));
    const int cx0 = max(bx0, 0), cx1 = min(bx1, kAcross - 1), cy0 = max(by0, 0), cy1 = min(by1, kAcross - 1);
    if (cx0 > cx1 || cy0 > cy1) return 0u;
    const float cb = ca * fr, cc = fs + ca * fr * fr;
    const float limit = screen.w * 1.0001f + 1e-4f;
    uint32_t mask = 0;
    for (int r = cy0; r <= cy1; ++r) {
        const float loy = (tileY0 + (float)(r * (int)kBox) + 0.5f) - screen.y;
        for (int c = cx0; c <= cx1; ++c) {
            const float lox = (tileX0 + (float)(c * (int)kBox) + 0.5f) - screen.x;
            const float least = minPowerOverBoxFactored(ca, cb, cc, fr, fs, lox, loy, lox + (float)(kBox - 1),
                                                        loy + (float)(kBox - 1));
            if (least <= limit) mask |= 1u << (r * kAcross + c);
        }
    }
    return mask;
}

// A walk's exponent e = log2(opacity) - power / (2 ln 2), so that alpha =
// min(0.99, 2^e) takes no multiply a pixel: each staged record carries
// log2(opacity) in place of its opacity (every record's opacity is at least 1/255).
__device__ __forceinline__ float log2Of(float x) {
    float lg;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(lg) : "f"(x));
    return lg;
}
// The least such exponent at which a pixel blends a record: the larger of the
// cutoff's (power at the cutoff) and log2(1/255), where alpha reaches 1/255. One
// comparison a pixel then stands for both tests. Both walks take it from the same
// record values, so the forward and the adjoint decide alike.
__device__ __forceinline__ float blendFloor(float cutoffExp, float lgOpacity) {
    constexpr float kLog2Faint = -7.99435344f;   // log2(1/255)
    return fmaxf(cutoffExp + lgOpacity, kLog2Faint);
}

// Nine values summed over a warp: the first eight by a transposed reduction
// (each level sends half of the values still held and keeps the other half,
// so three levels leave value (lane >> 2) spread over lanes differing in their
// two low bits), the ninth by a butterfly over the same three levels; the last
// two levels take the pair (value lane >> 2, the ninth) transposed as well.
// Lanes with lane % 4 == 0 end with value lane >> 2, lanes with lane % 4 == 2
// with the ninth. Every sum adds the same terms in the same pairs as a
// butterfly over each value alone, so the results are those of one.
__device__ __forceinline__ float warpSum9(float v[9], uint32_t lane) {
#pragma unroll
    for (int half = 4, bit = 16; half >= 1; half >>= 1, bit >>= 1) {
        const bool upper = (lane & (uint32_t)bit) != 0;
#pragma unroll
        for (int k = 0; k < half; ++k) {
            const float send = upper ? v[k] : v[k + half];
            const float keep = upper ? v[k + half] : v[k];
            v[k] = keep + __shfl_xor_sync(0xFFFFFFFFu, send, bit);
        }
    }
    float n = v[8];
#pragma unroll
    for (int o = 16; o > 2; o >>= 1) n += __shfl_xor_sync(0xFFFFFFFFu, n, o);
    const bool upper = (lane & 2u) != 0;
    float s = (upper ? n : v[0]) + __shfl_xor_sync(0xFFFFFFFFu, upper ? v[0] : n, 2);
    s += __shfl_xor_sync(0xFFFFFFFFu, s, 1);
    return s;
}

// ---- the blends of a training step: forward, loss and adjoint, a tile at a time ----
// One block of T*T/2 threads takes tiles off a queue (heaviest first: `order`,
// by the bit length of their pair counts, so the queue ends on light tiles)
// and, for each, runs the
// forward blend, the loss of its pixels, and the blend's adjoint, so that each
// pixel's final transmittance, last contributor and loss gradient stay in
// registers between the two walks.
//
// Forward: warp w owns an 8x8 box of the tile and each lane two pixels of it,
// (x, y) and (x, y + 4). Staging a batch of records, the block marks for each
// record the boxes its footprint can reach (a conservative test: the box's least
// power against the cutoff, with a margin); a warp then walks only the records
// marked for its box, found 32 at a time by a ballot, in list order. A pixel
// blends exactly the records it would blend walking the whole list: the
// per-pixel test decides, the box test only skips records no pixel of the box can
// pass. So the image does not depend on the tile size.
//
// Adjoint: each warp on its own once its pixels' loss gradients are known (no
// block barrier): the forward marked, for each 32-record chunk of the tile's list
// a warp walked, the records some pixel of its box blended (`live`, one word a
// chunk and box); the warp gathers those records, last first, 32 at a time into
// slots of its own and walks them from its pixels' last contributor down. What a
// lane sums over its two pixels, and the warp over its 64, are moments of
// dP = -2 dL/dpower over the pixel offsets in the factored frame (t = dx + fr dy,
// dy): sum dP t, sum dP dy, sum dP t^2, sum dP t dy, sum dP dy^2. Each visit's warp
// sums are added into the record's gradient words in global memory as they are
// (moments, opacity times dL/dopacity, dL/dcolour); the projection's adjoint turns
// the moments into the centre and conic gradients (batchMomentsToRecordGrad, which
// applies the -1/2) and divides the opacity's word by the opacity, once a record. The loss
// has no alpha term, so dL/d(alpha out) is 0 and the colour behind a record enters
// only through S.dC, one value a pixel.
//
// kTrain false: the forward blend alone (a batched render: colour and, when
// given, depth as the plain blend makes it; no target, loss or gradients).
// kCount: also count the walks' work (evaluations and warp visits) into the
// batch's words; a step timed stage by stage counts, the captured steps do not.
template <uint32_t T, uint32_t S, uint32_t NB, bool kTrain, bool kCount>
__global__ void __launch_bounds__(S * S / 2, S == 32 ? 2 : S == 16 ? (kTrain ? 8 : 7) : 16)   // 16x16 spans: no spill
    blendStepKernel(const BatchConst B, const BatchView* __restrict__ views, const uint2* __restrict__ ranges,
                    const uint64_t* __restrict__ pairs, const uint32_t* __restrict__ values,
                    const float4* __restrict__ recs, float4* __restrict__ colour, const float* __restrict__ target,
                    float* __restrict__ loss, float* __restrict__ grads, float* __restrict__ depth,
                    uint32_t* __restrict__ words, const uint32_t* __restrict__ order, uint32_t* __restrict__ live,
                    uint8_t* __restrict__ seen) {
    constexpr uint32_t kThreads = S * S / 2;
    constexpr uint32_t kAcross = S / kBox;            // boxes across a block's span
    constexpr uint32_t kSpans = (T / S) * (T / S);    // spans (blocks' work units) a tile
    constexpr uint32_t kBoxes = (T / kBox) * (T / kBox);   // boxes a tile (the live words' row)
    constexpr uint32_t kWords = 9;   // moments t, dy, tt, t dy, dy dy; alpha; colour r g b
    // a staged record, 48 bytes at one address: centre (cx, cy, depth); conic (ca, fs
    // pre-scaled, fr; log2 of the opacity); colour (r g b; the least exponent that blends)
    __shared__ float4 sStaged[NB][3];
    __shared__ uint32_t sMask[NB];
    __shared__ uint32_t sRec[NB];
    __shared__ uint32_t sTileBase[kMaxBatchViews];
    __shared__ uint32_t sTile;
    // the adjoint's gather slots, a warp's own: 32 records, each its centre with its
    // place in the tile's list and its record index (one 16-byte load a visit), its
    // conic and its colour
    constexpr uint32_t kWarpsHere = kTrain ? kThreads / 32 : 1;
    __shared__ float4 sWarpCentre[kWarpsHere][32];
    __shared__ float4 sWarpConic[kWarpsHere][32];
    __shared__ float4 sWarpColour[kWarpsHere][32];
    for (uint32_t k = threadIdx.x; k < B.views; k += kThreads) sTileBase[k] = views[k].tileBase;
    const uint64_t slotMask = (1ull << B.slotBits) - 1ull;
    const float kScale = -0.5f * 1.4426950408889634f;   // power -> base-2 exponent
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t lx = (warp % kAcross) * kBox + (lane & 7u), ly = (warp / kAcross) * kBox + (lane >> 3);
    uint32_t evaluated = 0;   // (pixel, record) evaluations of the forward this thread made
    uint32_t blended = 0;     // of them, those that blended
    uint32_t adjVisited = 0, adjLive = 0;   // the adjoint's evaluations, and those that blended
    uint32_t fwdVisits = 0, adjVisits = 0, adjSummed = 0;   // a warp's record visits (counted by lane 0)
    uint32_t staged = 0;      // records this thread staged
    float lossSum = 0.0f;     // this thread's pixels' share of the loss
    while (true) {
        __syncthreads();
        if (threadIdx.x == 0) {
            const uint32_t ticket = atomicAdd(&words[kBatchBlendTicket], 1u);
            sTile = ticket < B.totalTiles * kSpans ? order[ticket / kSpans] * kSpans + ticket % kSpans : 0xFFFFFFFFu;
        }
        __syncthreads();
        if (sTile == 0xFFFFFFFFu) break;
        const uint32_t tile = sTile / kSpans, span = sTile % kSpans;   // the block's span of the tile
        const uint32_t v = viewOf(sTileBase, B.views, tile);
        const BatchView& V = views[v];
        const uint32_t local = tile - V.tileBase;
        const uint32_t tx = local % V.tilesX, ty = local / V.tilesX;
        const uint32_t spanX = tx * T + (span % (T / S)) * S, spanY = ty * T + (span / (T / S)) * S;
        const float tileX0 = (float)spanX, tileY0 = (float)spanY;   // the span's first pixel
        const uint32_t px = spanX + lx, py[2] = {spanY + ly, spanY + ly + 4};
        const uint2 range = ranges[tile];
        const float pxc = (float)px + 0.5f, pyc[2] = {(float)py[0] + 0.5f, (float)py[1] + 0.5f};
        const size_t recBase = (size_t)v * B.count;
        // record s of this view into slot k: the factored conic's two weights pre-scaled
        // to base-2 exponent units, log2 of its opacity, the least exponent that blends,
        // and the boxes it can reach
        auto stage = [&](uint32_t k, uint32_t s) {
            if constexpr (kCount) ++staged;
            sRec[k] = s;
            const size_t at = (recBase + s) * 3;
            const float4 sc = recs[at + 0];
            const float4 c = recs[at + 1];
            const float4 rgb = recs[at + 2];
            sStaged[k][0] = make_float4(sc.x, sc.y, sc.z, 0.0f);
            const float lgo = log2Of(c.w);
            sStaged[k][1] = make_float4(c.x * kScale, c.y, c.z * kScale, lgo);
            sStaged[k][2] = make_float4(rgb.x, rgb.y, rgb.z, blendFloor(kScale * sc.w, lgo));
            sMask[k] = boxMask<S>(tileX0, tileY0, sc, c.x, c.y, c.z);
        };

        // ---- forward
        float r[2] = {0.0f, 0.0f}, g[2] = {0.0f, 0.0f}, bl[2] = {0.0f, 0.0f}, Tr[2] = {1.0f, 1.0f};
        float depthSum[2] = {0.0f, 0.0f}, depthAt[2] = {-1.0f, -1.0f};   // a render's depth
        uint32_t last[2] = {0, 0};
        bool done[2];
#pragma unroll
        for (int p = 0; p < 2; ++p) done[p] = !(px < V.width && py[p] < V.height);
        for (uint32_t first = range.x; first < range.y; first += NB) {
            if (__syncthreads_count(done[0] && done[1]) == kThreads) break;
            const uint32_t count = min(NB, range.y - first);
            for (uint32_t k = threadIdx.x; k < count; k += kThreads) stage(k, gaussianOf(pairs, values, slotMask, first + k));
            __syncthreads();
            if (__all_sync(0xFFFFFFFFu, done[0] && done[1])) continue;
            for (uint32_t base = 0; base < count; base += 32) {
                const uint32_t m = base + lane < count ? sMask[base + lane] : 0u;
                uint32_t todo = __ballot_sync(0xFFFFFFFFu, (m >> warp) & 1u);
                uint32_t laneBits = 0;   // the records of this chunk a pixel of this lane blended
                while (todo) {
                    const uint32_t j = base + (uint32_t)__ffs(todo) - 1u;
                    todo &= todo - 1u;
                    if constexpr (kCount) ++fwdVisits;
                    const float4 ce = sStaged[j][0];
                    const float4 k = sStaged[j][1];
                    const float dx = pxc - ce.x;
                    const float4 cc = sStaged[j][2];
                    bool hit = false;
                    // both pixels evaluated without branching: a pixel that does not blend the
                    // record (done, outside the cutoff, or under 1/255) takes alpha 0, which
                    // leaves its sums and transmittance as they were
#pragma unroll
                    for (int p = 0; p < 2; ++p) {
                        const float dy = pyc[p] - ce.y;
                        const float t = __fmaf_rn(k.y, dy, dx);
                        const float e = __fmaf_rn(k.x * t, t, __fmaf_rn(k.z * dy, dy, k.w));
                        const float a0 = fminf(0.99f, fastExp2(e));
                        const bool blend = !done[p] && e >= cc.w;
                        if constexpr (kCount) { evaluated += done[p] ? 0u : 1u; blended += blend ? 1u : 0u; }
                        const float alpha = blend ? a0 : 0.0f;
                        const float w = Tr[p] * alpha;
                        r[p] = __fmaf_rn(w, cc.x, r[p]);
                        g[p] = __fmaf_rn(w, cc.y, g[p]);
                        bl[p] = __fmaf_rn(w, cc.z, bl[p]);
                        if constexpr (!kTrain) depthSum[p] = __fmaf_rn(w, ce.z, depthSum[p]);
                        Tr[p] = __fmaf_rn(-Tr[p], alpha, Tr[p]);   // T (1 - alpha), one rounding
                        last[p] = blend ? first - range.x + j + 1 : last[p];
                        if constexpr (!kTrain)
                            if (blend && depthAt[p] < 0.0f && 1.0f - Tr[p] >= B.depthThreshold) depthAt[p] = ce.z;
                        done[p] = done[p] || Tr[p] < 1e-4f;
                        hit = hit || blend;
                    }
                    if constexpr (kTrain) laneBits |= hit ? 1u << (j - base) : 0u;
                }
                // the records of this chunk some pixel of the box blended
                const uint32_t liveWord = kTrain ? __reduce_or_sync(0xFFFFFFFFu, laneBits) : 0u;
                if constexpr (kTrain) {
                    if (lane == 0)
                        live[((size_t)(range.x >> 5) + tile + ((first - range.x + base) >> 5)) * kBoxes +
                             span * (kAcross * kAcross) + warp] = liveWord;
                    // the records some pixel blended take a gradient in the adjoint: mark them
                    // (lane l for record base + l; a plain store, every writer stores 1), by which
                    // the projection's adjoint groups Gaussians
                    if ((liveWord >> lane) & 1u) seen[recBase + sRec[base + lane]] = 1u;
                }
                if (__all_sync(0xFFFFFFFFu, done[0] && done[1])) break;
            }
        }

        if constexpr (!kTrain) {
#pragma unroll
            for (int p = 0; p < 2; ++p) {
                if (!(px < V.width && py[p] < V.height)) continue;
                const float coverage = 1.0f - Tr[p];
                const uint32_t at = V.pixelBase + py[p] * V.width + px;
                colour[at] = make_float4(r[p] + Tr[p] * B.bg[0], g[p] + Tr[p] * B.bg[1], bl[p] + Tr[p] * B.bg[2],
                                         coverage + Tr[p] * B.bg[3]);
                if (depth)
                    depth[at] = B.depthMode == 0 ? (coverage > 1e-6f ? depthSum[p] / coverage : 0.0f)
                                                 : fmaxf(depthAt[p], 0.0f);
            }
            continue;
        }

        // ---- the pixels' colour, the loss (the view's mean L2 over its pixels and r g b) and its gradient
        float sd[2], dC[2][3];
#pragma unroll
        for (int p = 0; p < 2; ++p) {
            dC[p][0] = dC[p][1] = dC[p][2] = 0.0f;
            if (px < V.width && py[p] < V.height) {
                const uint32_t at = V.pixelBase + py[p] * V.width + px;
                const float coverage = 1.0f - Tr[p];
                const float4 c = make_float4(r[p] + Tr[p] * B.bg[0], g[p] + Tr[p] * B.bg[1],
                                             bl[p] + Tr[p] * B.bg[2], coverage + Tr[p] * B.bg[3]);
                colour[at] = c;
                const float er = c.x - target[(size_t)at * 3 + 0], eg = c.y - target[(size_t)at * 3 + 1],
                            eb = c.z - target[(size_t)at * 3 + 2];
                lossSum += (er * er + eg * eg + eb * eb) * V.lossScale;
                const float k2 = 2.0f * V.lossScale;
                dC[p][0] = k2 * er;
                dC[p][1] = k2 * eg;
                dC[p][2] = k2 * eb;
            }
            sd[p] = (B.bg[0] * dC[p][0] + B.bg[1] * dC[p][1]) + B.bg[2] * dC[p][2];   // S.dC, S the colour behind
        }

        // ---- adjoint: each warp on its own, over the records its box blended, last first
        // (the forward's live bits), gathered 32 at a time into the warp's own slots; no
        // block barrier, no staging and no box tests
        const uint32_t warpLast = __reduce_max_sync(0xFFFFFFFFu, max(last[0], last[1]));
        const uint32_t nChunks = (warpLast + 31u) >> 5;
        const uint32_t* liveOf = live + ((size_t)(range.x >> 5) + tile) * kBoxes + span * (kAcross * kAcross) + warp;
        for (int32_t hi = (int32_t)nChunks - 1; hi >= 0; hi -= 32) {
            // lane l: the live bits of chunk hi - l (records 32 c .. 32 c + 31 of the tile)
            const int32_t ch = hi - (int32_t)lane;
            const uint32_t word = ch >= 0 ? liveOf[(size_t)ch * kBoxes] : 0u;
            const uint32_t n = __popc(word);
            uint32_t incl = n;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t u = __shfl_up_sync(0xFFFFFFFFu, incl, o);
                if (lane >= (uint32_t)o) incl += u;
            }
            const uint32_t total = __shfl_sync(0xFFFFFFFFu, incl, 31);
            const uint32_t excl = incl - n;
            for (uint32_t r0 = 0; r0 < total; r0 += 32) {
                // the records of ranks r0 .. r0 + 31 (ranked last first) into the warp's slots:
                // lane q takes rank r0 + q. Its chunk is the last lane c whose exclusive count
                // is at most the rank (a search over the lanes' counts); in that chunk's word,
                // the record is the set bit of the remaining rank, counted down from bit 31 (a
                // search over the word's halves, quarters, ...). No lane walks bits one by one.
                const uint32_t want = r0 + lane;
                uint32_t c = 0;
#pragma unroll
                for (uint32_t step = 16; step; step >>= 1)
                    if (__shfl_sync(0xFFFFFFFFu, excl, c + step) <= want) c += step;
                const uint32_t wc = __shfl_sync(0xFFFFFFFFu, word, c);
                uint32_t rem = want - __shfl_sync(0xFFFFFFFFu, excl, c), bit = 31;
#pragma unroll
                for (uint32_t step = 16; step; step >>= 1) {
                    const uint32_t below = __popc((wc >> (bit - step + 1u)) & ((1u << step) - 1u));
                    if (below <= rem) {
                        rem -= below;
                        bit -= step;
                    }
                }
                const uint32_t cnt = min(32u, total - r0);   // lane < cnt exactly when want < total
                if (lane < cnt) {
                    const uint32_t rel = (uint32_t)(hi - (int32_t)c) * 32u + bit;
                    const uint32_t gs = gaussianOf(pairs, values, slotMask, range.x + rel);
                    const size_t at = (recBase + gs) * 3;
                    const float4 sc = recs[at + 0];
                    const float4 k = recs[at + 1];
                    const float4 rgb = recs[at + 2];
                    sWarpCentre[warp][lane] =
                        make_float4(sc.x, sc.y, __uint_as_float(rel), __uint_as_float((uint32_t)(recBase + gs)));
                    const float lgo = log2Of(k.w);
                    sWarpConic[warp][lane] = make_float4(k.x * kScale, k.y, k.z * kScale, lgo);
                    sWarpColour[warp][lane] = make_float4(rgb.x, rgb.y, rgb.z, blendFloor(kScale * sc.w, lgo));
                }
                __syncwarp();
                for (uint32_t q = 0; q < cnt; ++q) {
                    if constexpr (kCount) ++adjVisits;
                    const float4 ce = sWarpCentre[warp][q];
                    const uint32_t rel = __float_as_uint(ce.z);
                    const float4 k = sWarpConic[warp][q];
                    const float4 c = sWarpColour[warp][q];
                    const float dx = pxc - ce.x;
                    // the sums start at -0, which adding leaves any value as it is (+0 would
                    // turn a -0 term into +0): the first pixel's terms are taken as they come
                    float gv[kWords];
#pragma unroll
                    for (int e = 0; e < (int)kWords; ++e) gv[e] = -0.0f;
                    // as the forward, without branching: a pixel past its last contributor or
                    // that does not blend the record takes alpha 0 (T unchanged, no terms)
#pragma unroll
                    for (int p = 0; p < 2; ++p) {
                        const float dy = pyc[p] - ce.y;
                        const float t = __fmaf_rn(k.y, dy, dx);
                        const float e = __fmaf_rn(k.x * t, t, __fmaf_rn(k.z * dy, dy, k.w));
                        const float raw = fastExp2(e);
                        const float a0 = fminf(0.99f, raw);
                        const bool on = rel < last[p] && e >= c.w;
                        if constexpr (kCount) { adjVisited += rel < last[p] ? 1u : 0u; adjLive += on ? 1u : 0u; }
                        const float alpha = on ? a0 : 0.0f;
                        const float inv = fastRcp(1.0f - alpha);
                        const float Tb = Tr[p] * inv;
                        const float w = Tb * alpha;
                        gv[6] = __fmaf_rn(w, dC[p][0], gv[6]);
                        gv[7] = __fmaf_rn(w, dC[p][1], gv[7]);
                        gv[8] = __fmaf_rn(w, dC[p][2], gv[8]);
                        const float cd = (c.x * dC[p][0] + c.y * dC[p][1]) + c.z * dC[p][2];
                        // alpha dL/dalpha where alpha is not clamped (dL/dalpha = T before it
                        // times (c - S).dC): the opacity times dL/dopacity, and -2 dL/dpower
                        const float u = cd - sd[p];
                        const float dP = on && raw < 0.99f && k.w <= 0.0f ? w * u : 0.0f;
                        sd[p] = __fmaf_rn(alpha, u, sd[p]);
                        Tr[p] = Tb;
                        gv[5] += dP;
                        const float dPt = dP * t, dPy = dP * dy;
                        gv[0] += dPt;
                        gv[1] += dPy;
                        gv[2] = __fmaf_rn(dPt, t, gv[2]);
                        gv[3] = __fmaf_rn(dPt, dy, gv[3]);
                        gv[4] = __fmaf_rn(dPy, dy, gv[4]);
                    }
                    // no test that some lane is live: a gathered record's forward live bit says a
                    // pixel of this box blended it, and the adjoint decides that pixel the same way
                    // (a record with no live lane would only add zeros, which are not stored)
                    if constexpr (kCount) ++adjSummed;
                    // the warp's sums, however few lanes are live, added by nine lanes at once
                    // into the record's words in global memory (reductions, not read back):
                    // the five moments, dL/dalpha and dL/dcolour, which the projection's
                    // adjoint turns into centre and conic gradients (linear in the moments,
                    // so sums from every box, tile and batch add up)
                    const float val = warpSum9(gv, lane);
                    const uint32_t slot = (lane & 3u) == 0u ? lane >> 2 : lane == 2u ? 8u : kWords;
                    if (slot < kWords && val != 0.0f)
                        atomicAdd(grads + (size_t)__float_as_uint(ce.w) * kGradWords + slot, val);
                }
                __syncwarp();   // the next round's gathers overwrite the slots
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) lossSum += __shfl_xor_sync(0xFFFFFFFFu, lossSum, o);
    if (kTrain && lane == 0 && lossSum != 0.0f) atomicAdd(loss, lossSum);
    if constexpr (!kCount) return;
    // the work counts: a warp's sums, one atomic each
    const uint32_t visits = lane == 0;   // a warp's visits, once
    const uint32_t counts[8] = {evaluated, blended, adjVisited, adjLive, fwdVisits * visits, adjVisits * visits,
                                adjSummed * visits, staged};
    const uint32_t at[8] = {kBatchEvaluated, kBatchBlended, kBatchAdjVisited, kBatchAdjLive, kBatchFwdVisits,
                            kBatchAdjVisits, kBatchAdjSummed, kBatchStaged};
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        uint64_t e = counts[c];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(0xFFFFFFFFu, e, o);
        if (lane == 0 && e) atomicAdd(reinterpret_cast<unsigned long long*>(words + at[c]), (unsigned long long)e);
    }
}

template <typename K>
int residentGrid(K kernel, int threads, int sms) {
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, threads, 0);
    return (n > 0 ? n : 1) * sms;
}

template <uint32_t T, uint32_t S, uint32_t NB>
cudaError_t stepWith(const BatchConst& B, const BlendLaunch& L, cudaStream_t stream, float4* colour,
                     const float* target, float* loss, float* grads, float* depth) {
    if (target && L.count) {
        const int grid = residentGrid(blendStepKernel<T, S, NB, true, true>, S * S / 2, L.sms);
        blendStepKernel<T, S, NB, true, true><<<grid, S * S / 2, 0, stream>>>(
            B, L.views, L.ranges, L.pairs, L.values, L.recs, colour, target, loss, grads, nullptr, L.words, L.order,
            L.live, L.seen);
    } else if (target) {
        const int grid = residentGrid(blendStepKernel<T, S, NB, true, false>, S * S / 2, L.sms);
        blendStepKernel<T, S, NB, true, false><<<grid, S * S / 2, 0, stream>>>(
            B, L.views, L.ranges, L.pairs, L.values, L.recs, colour, target, loss, grads, nullptr, L.words, L.order,
            L.live, L.seen);
    } else {
        const int grid = residentGrid(blendStepKernel<T, S, NB, false, false>, S * S / 2, L.sms);
        blendStepKernel<T, S, NB, false, false><<<grid, S * S / 2, 0, stream>>>(
            B, L.views, L.ranges, L.pairs, L.values, L.recs, colour, nullptr, nullptr, nullptr, depth, L.words,
            L.order, nullptr, nullptr);
    }
    return cudaGetLastError();
}

}   // namespace

#define ATH_BLEND_CASES(CALL)                                                                              \
    CALL(8, 64) CALL(8, 128) CALL(8, 256) CALL(8, 512) CALL(16, 64) CALL(16, 128) CALL(16, 256) CALL(16, 512)     \
    CALL(32, 64) CALL(32, 128) CALL(32, 256) CALL(32, 512)

cudaError_t launchBatchBlendStep(const BatchConst& B, const BlendLaunch& L, cudaStream_t stream, float4* colour,
                                 const float* target, float* loss, float* grads, float* depth) {
#define ATH_CASE(T_, NB_) \
    if (L.tile == T_ && L.blockBatch == NB_) \
        return stepWith<T_, (T_ > kBlendSpan ? kBlendSpan : T_), NB_>(B, L, stream, colour, target, loss, grads, depth);
    ATH_BLEND_CASES(ATH_CASE)
#undef ATH_CASE
    return cudaErrorInvalidValue;
}

}   // namespace ath
