// The batched path's device code: many views of one cloud in each launch.
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

#include "gauss.cuh"
#include "raster_types.cuh"
#include "splat_math.cuh"

namespace ath {

// One view of a batch.
struct BatchView {
    uint32_t width, height, tilesX, tilesY;
    float focalX, focalY, centreX, centreY, nearZ, farZ;
    uint32_t orthographic;
    uint32_t tileBase;    // its first tile among all views' tiles
    uint32_t pixelBase;   // its first pixel in the concatenated images
    float lossScale;      // 1 / (3 width height): the mean over its pixels and r g b
    float m[12];          // object -> view rows
    float eye[3];         // the camera in the cloud's space
};

constexpr uint32_t kMaxBatchViews = 256;

// Constants of a batched step.
struct BatchConst {
    uint32_t views;
    uint32_t count;          // Gaussians
    uint32_t tile;           // 8, 16 or 32
    uint32_t slotBits;       // bits of a Gaussian index in a packed pair (0 when wide)
    uint32_t keyShift;       // where the global tile starts in a pair's key: depthBits + slotBits
    uint32_t wide;           // 1: key (tile << 24 | depth) and a separate u32 Gaussian index a pair
    uint32_t depthBits;      // a pair's depth field: 24 (the depth key), or 16 + e bits for a key whose
    uint32_t expBase;        // exponent byte is renumbered from expBase (e bits; packed pairs only)
    uint32_t sizing;         // 1: the sizing pass (counts only; it also records the depths' exponent range)
    uint32_t totalTiles, totalPixels;
    uint32_t shLimit, antialias, linear, restPerColour;
    uint32_t depthMode;      // a render's depth: 0 the alpha-weighted mean, 1 the first threshold crossing
    float depthThreshold;
    float bg[4];
    uint64_t capacity;       // pairs the pair buffers hold
    InstanceConst inst;      // the cloud (params or mixed layout); m/eye per view
};

// Words of a batch's device block.
enum BatchWord : uint32_t {
    kBatchEpoch = 0,         // a step's tag for its look-back words (bumped by the step's first kernel)
    kBatchTicket = 1,        // the projection's ticket
    kBatchStatus = 2,        // kStatus* bits, sticky across steps until read
    kBatchPairsLo = 3,
    kBatchPairsHi = 4,
    kBatchBlendTicket = 5,   // the persistent blend's tile queue
    kBatchKept = 7,          // (view, Gaussian) records kept
    kBatchSortTickets = 8,   // one a sort pass (8)
    kBatchEvaluated = 16,    // 64-bit (16, 17): (pixel, record) evaluations of the forward blend
    kBatchDegenerate = 18,   // records whose conic took the FP64 path
    kBatchExpMin = 22,       // least and greatest exponent byte of the depths of the records on
    kBatchExpMax = 23,       // screen (for planning a renumbered depth key)
    kBatchBlended = 24,      // 64-bit (24, 25): forward evaluations that blended (passed the cutoff and 1/255)
    kBatchAdjVisited = 26,   // 64-bit (26, 27): adjoint evaluations (a pixel, a record before its last contributor)
    kBatchAdjLive = 28,      // 64-bit (28, 29): adjoint evaluations that blended, whose gradient terms were summed
    kBatchFwdVisits = 32,    // 64-bit (32, 33): (warp, record) visits of the forward walk
    kBatchAdjVisits = 34,    // 64-bit (34, 35): (warp, record) visits of the adjoint walk
    kBatchAdjSummed = 36,    // 64-bit (36, 37): adjoint visits with a live lane, whose sums the warp reduced
    kBatchStaged = 38,       // 64-bit (38, 39): records a block staged (loaded and box-tested) for the forward
    kBatchWords = 48,
};

// An epoch-tagged look-back word: [epoch:30][status:2][value:32]. A word with
// another step's epoch reads as "not ready", so the words need no clearing.
__device__ __forceinline__ uint64_t tagged(uint32_t epoch, uint32_t status, uint32_t value) {
    return ((uint64_t)(epoch & 0x3FFFFFFFu) << 34) | ((uint64_t)status << 32) | value;
}

__device__ __forceinline__ float fastExp2(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

__device__ __forceinline__ float fastRcp(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// minPowerOverBox for a near-degenerate footprint: the same candidate points,
// each evaluated in the factored form ca (x + fr y)^2 + fs y^2, which does not
// cancel however thin the footprint is.
__device__ __forceinline__ float minPowerOverBoxFactored(float a, float b, float c, float fr, float fs, float lox,
                                                         float loy, float hix, float hiy) {
    if (lox <= 0.0f && hix >= 0.0f && loy <= 0.0f && hiy >= 0.0f) return 0.0f;
    float best = 3.4e38f;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        float x, y;
        if (e < 2) {
            x = e == 0 ? lox : hix;
            y = c > 1e-12f ? clampf(((-b) * x) / c, loy, hiy) : loy;
        } else {
            y = e == 2 ? loy : hiy;
            x = a > 1e-12f ? clampf(((-b) * y) / a, lox, hix) : lox;
        }
        const float t = x + fr * y;
        best = fminf(best, (a * t) * t + (fs * y) * y);
    }
    return best;
}

// The Gaussian of sorted pair i: in the packed key's low bits, or the wide form's value.
__device__ __forceinline__ uint32_t gaussianOf(const uint64_t* pairs, const uint32_t* values, uint64_t slotMask,
                                              uint32_t i) {
    return values ? values[i] : (uint32_t)(pairs[i] & slotMask);
}

// The view of a global tile or pixel: the last view whose base is at most `x`.
__device__ __forceinline__ uint32_t viewOf(const uint32_t* bases, uint32_t views, uint32_t x) {
    uint32_t lo = 0, hi = views;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (bases[mid] <= x) lo = mid; else hi = mid;
    }
    return lo;
}

// The batched blend adjoint's words for a record (the warp sums it adds up):
// [0..4] the moments of -2 dL/dpower over the pixel offsets in the record's factored
// frame t = dx + fr dy, dy (sum t, dy, t^2, t dy, dy^2 times it), [5] the opacity
// times dL/dopacity, [6..8] dL/dcolour. To dL/d(centre, conic), with the -1/2 applied
// here (exact: a power of two): the conic is ca (dx + fr dy)^2 + fs dy^2, so
// dL/da = sum dP dx^2 with dx = t - fr dy, and so on; in place, in the plain path's
// kGrad* layout. Word [5] is left for the caller, which knows the opacity.
__device__ __forceinline__ void batchMomentsToRecordGrad(float ca, float fr, float fs, float g[10]) {
    const float mt = -0.5f * g[0], my = -0.5f * g[1], mtt = -0.5f * g[2], mty = -0.5f * g[3], myy = -0.5f * g[4];
    g[kGradCx] = -2.0f * ca * mt;
    g[kGradCy] = -2.0f * (fr * ca * mt + fs * my);
    g[kGradA] = mtt - 2.0f * fr * mty + fr * fr * myy;   // sum dP dx^2
    g[kGradB2] = 2.0f * (mty - fr * myy);                 // sum dP 2 dx dy
    g[kGradC] = myy;                                      // sum dP dy^2
}

// What the persistent blend of batch_blend.cu needs from a batch.
struct BlendLaunch {
    const BatchView* views;
    const uint2* ranges;
    const uint64_t* pairs;   // sorted
    const uint32_t* values;  // wide pairs: the Gaussian of each sorted pair; null when packed
    const float4* recs;
    uint32_t* words;
    const uint32_t* order;   // the tiles, heaviest first
    uint32_t* live;          // a training step's live bits: per tile, one word a 32-record chunk and box
    uint8_t* seen;           // a training step's: per record (view, Gaussian), 1 once some pixel blended it
    int sms;
    uint32_t tile, blockBatch;
    bool count;              // count the walks' work into `words` (a step timed stage by stage)
};

// The live bits' words a batch needs: chunk c of tile t's list (records 32 c ..
// 32 c + 31 after its range's start) and box b at word ((start >> 5) + t + c) boxes + b,
// so tiles never overlap (each takes at most one word-row past start / 32).
inline size_t liveWords(uint64_t capacity, uint32_t totalTiles, uint32_t tile) {
    const size_t boxes = (size_t)(tile / 8) * (tile / 8);
    return (size_t)(capacity / 32 + totalTiles + 2) * boxes;
}

// A training step's blends over every view's tiles, in one kernel: the forward
// blend into `colour`; the loss, each view's mean L2 against `target` (float3 a
// pixel) over its pixels and r g b, summed over views into *loss (which the
// caller zeroes); and the adjoint, dL/d(record) for every (view, Gaussian)
// record, added into `grads` (which start at zero). A null `target`: the
// forward blend alone, colour and (when `depth` is given) depth.
cudaError_t launchBatchBlendStep(const BatchConst& B, const BlendLaunch& L, cudaStream_t stream, float4* colour,
                                 const float* target, float* loss, float* grads, float* depth = nullptr);

}   // namespace ath
