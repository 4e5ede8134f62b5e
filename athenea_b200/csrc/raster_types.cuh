// What the host hands the kernels, and the device-side primitives the stages
// share (the decoupled look-back of the scans and the sort).
#pragma once

#include <cstdint>

namespace ath {

// common/edit.slang:23-36
struct EditConst {
    uint32_t active, shape, mode, invert;
    float centre[3], size[3], tint[3];
    float saturation, brightness, opacity, minOpacity, maxScale;
};

// The per-frame part of splat/frame.slang's FrameParams (setFrame,
// modules/render/src/FrameParams.h:32-82), plus what the P layer needs.
struct FrameConst {
    uint32_t width, height, tilesX, tilesY;
    float focalX, focalY, centreX, centreY, nearZ, farZ;
    uint32_t orthographic, tileBits, shLimit, depthMode;
    float depthThreshold;
    float bg[4];
    float viewToWorld[12];   // rows of the view -> world 3x4, for P
};

// The per-instance part (setObject, setCloudSpace, setEdit: FrameParams.h:84-165),
// with the cloud's device buffers in one of the layouts of gauss.cuh.
struct InstanceConst {
    // the reference's packed layout (scene/GpuClouds.h:44-52)
    const float4* positions;
    const uint4* shape;
    const uint32_t* sh;
    // FP32 training parameters, and the mixed-precision layout's SH
    const float* means;     // float4: x y z, opacity logit
    const float* scales;    // float4: log scales
    const float* quats;     // float4: w x y z
    const float* shf;       // shStride floats: DC rgb, rest rgb per basis
    const void* shLow;      // mixed: 12 bf16 a Gaussian (DC, band 1)
    const void* shHigh;     // mixed: 36 e4m3 a Gaussian (bands 2-3)
    const float* shScale;   // mixed: the bands' scale a Gaussian
    uint32_t count, base, restPerColour, shWords, shStride, linear, antialias;
    float paidAt;
    float m[12];
    float eye[3];
    EditConst edit;
};

// Words of the small device block a frame keeps its counts and status in. All
// of them are cleared at a frame's start; at its end they are copied to pinned
// host memory behind an event (the frame's status, and its counters when it
// counts), so nothing waits for them.
constexpr uint32_t kMaxClouds = 64;   // SplatCounters::kMaxClouds (TileRasterizer.h:376)
enum FrameWord : uint32_t {
    kWordTicket = 0,        // the projection's block ticket
    kWordVisible = 1,       // splats kept
    kWordStatus = 2,        // kStatus* bits of the projection's scan
    kWordPairsLo = 3,       // pairs (the sum of tiles touched), 64-bit
    kWordPairsHi = 4,
    kWordMaxTiles = 5,
    kWordCulled = 6,        // 7 words: culled by reason (count_splats)
    kWordPairsKept = 13,    // the pairs the buffers hold: min(pairs, capacity), what the sort sorts
    kWordSortTickets = 16,  // one a sort pass (up to 8)
    kWordClouds = 24,       // 2 words a cloud (visible, pairs) for the first kMaxClouds instances (count_splats)
    kWordSticky = kWordClouds + 2 * kMaxClouds,   // status the emit, sort, ranges, blends and backward raise
    kFrameWords = kWordSticky + 1,                // cleared at the start of every frame
};

enum StatusBit : uint32_t {
    kStatusLookbackTimeout = 1u,   // a look-back gave up waiting (bounded spin)
    kStatusPairOverflow = 2u,      // more pairs than the pair buffers hold
    kStatusIndexRange = 4u,        // a data-dependent index fell outside its buffer (skipped)
    kStatusDepthRange = 8u,        // a depth's exponent outside the range a step's pair keys were planned for
};

// The backward's gradient with respect to one record: ten floats a slot.
enum GradWord : uint32_t {
    kGradCx = 0, kGradCy = 1,               // screen centre
    kGradA = 2, kGradB2 = 3, kGradC = 4,    // conic a, b, c
    kGradAlpha = 5,                         // the record's opacity (after the payback)
    kGradR = 6, kGradG = 7, kGradB = 8,     // colour
    kGradZ = 9,                             // view depth (the depth layer's)
    kGradWords = 10,
};

// A look-back word: two status bits over a 62-bit count.
constexpr uint64_t kFlagAggregate = 1ull << 62;
constexpr uint64_t kFlagInclusive = 2ull << 62;
constexpr uint64_t kFlagValue = (1ull << 62) - 1;
constexpr uint32_t kSpinLimit = 1u << 20;   // spins before a wait gives up (tens of ms)

// Whether some block has already given up: the rest stop waiting at once, so
// one failure costs one time-out, not one a block.
__device__ __forceinline__ bool gaveUp(const uint32_t* status) {
    return (*reinterpret_cast<const volatile uint32_t*>(status) & 1u) != 0;
}

__device__ __forceinline__ void storeRelaxed(uint64_t* p, uint64_t v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ uint64_t loadRelaxed(const uint64_t* p) {
    uint64_t v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ uint64_t warpSum64(uint64_t v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
    return v;
}

// Decoupled look-back (Merrill and Garland, "Single-pass Parallel Prefix Scan
// with Decoupled Look-back", 2016), one warp wide: block `b` publishes its
// aggregate, then sums its predecessors' words 32 at a time until it meets an
// inclusive prefix, and publishes its own. Called by all 32 lanes of one
// warp; returns the exclusive prefix. Blocks take `b` from an atomic ticket in
// launch order, so every predecessor is resident or done and each wait ends;
// the wait is still bounded, and a block that gives up sets
// kStatusLookbackTimeout and goes on with what it has.
__device__ __forceinline__ uint64_t lookbackExclusive(uint64_t* flags, uint32_t b, uint64_t aggregate,
                                                      uint32_t* status) {
    const uint32_t lane = threadIdx.x & 31u;
    if (b == 0) {
        if (lane == 0) storeRelaxed(flags, kFlagInclusive | aggregate);
        return 0;
    }
    if (lane == 0) storeRelaxed(flags + b, kFlagAggregate | aggregate);
    uint64_t exclusive = 0;
    int64_t window = (int64_t)b - 1;
    uint32_t spins = 0;
    while (true) {
        const int64_t idx = window - (int64_t)lane;
        const uint64_t v = idx >= 0 ? loadRelaxed(flags + idx) : kFlagInclusive;
        const uint32_t st = (uint32_t)(v >> 62);
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
        exclusive += warpSum64(lane <= first ? (v & kFlagValue) : 0ull);
        if (first < 32) break;
        window -= 32;
    }
    if (lane == 0) storeRelaxed(flags + b, kFlagInclusive | (exclusive + aggregate));
    return exclusive;
}

}   // namespace ath
