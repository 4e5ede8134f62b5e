// The batched path's device code: many views of one cloud in each launch.
#pragma once

#include <cstdint>

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
    uint32_t slotBits;       // bits of a Gaussian index in a packed pair
    uint32_t keyShift;       // 24 + slotBits: where the global tile starts in a packed pair
    uint32_t totalTiles, totalPixels;
    uint32_t shLimit, antialias, linear, restPerColour;
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
    kBatchBackTicket = 6,    // the persistent backward's tile queue
    kBatchKept = 7,          // (view, Gaussian) records kept
    kBatchSortTickets = 8,   // one a sort pass (8)
    kBatchEvaluated = 16,    // 64-bit (16, 17): (pixel, record) evaluations of the forward blend
    kBatchDegenerate = 18,   // records whose conic took the FP64 path
    kBatchWords = 32,
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

// The view of a global tile or pixel: the last view whose base is at most `x`.
__device__ __forceinline__ uint32_t viewOf(const uint32_t* bases, uint32_t views, uint32_t x) {
    uint32_t lo = 0, hi = views;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (bases[mid] <= x) lo = mid; else hi = mid;
    }
    return lo;
}

}   // namespace ath
