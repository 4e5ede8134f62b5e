// Host-side entry points of the stage kernels (one .cu each), called by the
// rasteriser's host code (host.cu).
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/athenea_raster.h"

namespace ath {

struct FrameConst;
struct InstanceConst;

// host.cu: FrameParams' setters (modules/render/src/FrameParams.h:32-117)
FrameConst frameConstFor(const ath_projection& p, const ath_settings& s);
InstanceConst instanceConstFor(const ath_projection& p, const ath_settings& s, const ath_instance& in, uint32_t base);

// project.cu
uint32_t projectBlocks(uint32_t slots);
cudaError_t launchProject(const FrameConst& F, const InstanceConst* inst, uint32_t nInst, uint32_t slots,
                          uint32_t layout, bool countCulls, float4* recs, uint2* rects, uint32_t* keys,
                          uint32_t* offsets, uint64_t* flags, uint32_t* words, cudaStream_t stream);
// Writes the pairs the buffers hold, min(pairs, capacity), into words[kWordPairsKept],
// and raises kStatusPairOverflow in words[kWordSticky] past the capacity.
cudaError_t launchEmit(const FrameConst& F, uint32_t slots, const float4* recs, const uint2* rects,
                       const uint32_t* keys, const uint32_t* offsets, uint32_t* words, uint64_t capacity,
                       uint64_t* pairKeys, uint32_t* pairValues, cudaStream_t stream);
// Ranges over at most `pairs` sorted keys; `pairsDevice`, when given, holds the count.
cudaError_t launchRanges(uint32_t pairs, const uint32_t* pairsDevice, uint32_t tiles, const uint64_t* pairKeys,
                         uint2* ranges, uint32_t* status, cudaStream_t stream);

// sort.cu
constexpr uint32_t kSortTileKeys = 8192;   // keys a onesweep block ranks (the look-back's unit)
uint32_t sortPasses(uint32_t bits);      // 8-bit passes, or 9-bit ones where that saves a pass
uint32_t sortHistWords();                // the words of a sort's digit histograms (every pass)
uint32_t sortTiles(uint32_t n);
size_t sortFlagWords(uint32_t n, uint32_t bits);
uint32_t sortResultIndex(uint32_t n, uint32_t bits);
cudaError_t sortPrepare();
cudaError_t launchSort(uint64_t* keys[2], uint32_t* vals[2], uint32_t n, uint32_t bits, uint32_t* hist,
                       uint64_t* flags, uint32_t* tickets, uint32_t* status, cudaStream_t stream);
cudaError_t launchSortBits(uint64_t* keys[2], uint32_t* vals[2], uint32_t n, uint32_t firstBit, uint32_t bits,
                           uint32_t* hist, uint64_t* flags, uint32_t* tickets, uint32_t* status, cudaStream_t stream);
// The same with the key count on the device (at most n) and, when epochDevice is
// given, epoch-tagged look-back words that need no clearing (a captured step).
cudaError_t launchSortDevice(uint64_t* keys[2], uint32_t* vals[2], uint32_t n, const uint32_t* nDevice,
                             const uint32_t* epochDevice, uint32_t firstBit, uint32_t bits, uint32_t* hist,
                             uint64_t* flags, uint32_t* tickets, uint32_t* status, cudaStream_t stream);

// blend.cu
// The reference's contributionMode hooks of the blend (modes 1 and 4).
struct Contribution {
    uint32_t mode = 0;                   // 0 none, 1 weights, 2 squared change, 3 lifted mask, 4 colour gradients
    uint32_t* words = nullptr;
    const float* finalColour = nullptr;  // float4 a pixel: mode 2 the whole frame, mode 4 dL/dpixel
    const float* liftMask = nullptr;     // mode 3: a float a pixel
};

// An opaque layer under the splats (TileRasterizer::render's `under`): its
// colour (float4) and depth (float, 0 where it has nothing) a pixel.
struct Under {
    const float* colour = nullptr;
    const float* depth = nullptr;
};

// Cryptomatte: a uint id a slot in, 3 float4 layers a pixel out.
struct Matte {
    const uint32_t* ids = nullptr;        // Cryptomatte: the id a slot, the layers out, the under layer's ids
    float* out = nullptr;
    const uint32_t* underIds = nullptr;
    const uint32_t* liftSums = nullptr;   // the matte a lift told the splats: two words a slot (inside, seen)
    float* lifted = nullptr;              // and the matte a pixel it sums to
    uint32_t hard = 0;
    float threshold = 0.5f;
    uint32_t* trace = nullptr;            // the splats a pixel is made of (splat_trace.slang), kTraceWords planes
};

cudaError_t launchBlend(const FrameConst& F, uint32_t pairs, uint32_t slots, const uint2* ranges,
                        const uint32_t* pairValues, const float4* recs, float4* colour, float* depth, float4* position,
                        float* finalT, uint32_t* lastContrib, uint32_t* status, cudaStream_t stream,
                        const Contribution& contrib = Contribution{}, const Under& under = Under{},
                        const Matte& matte = Matte{});

// backward.cu
cudaError_t launchBlendBackward(const FrameConst& F, uint32_t pairs, uint32_t slots, const uint2* ranges,
                                const uint32_t* pairValues, const float4* recs, const float* finalT,
                                const uint32_t* lastContrib, const float4* dLdColour, const float* dLdDepth,
                                const float* depthOut, float* grads, uint32_t* status, cudaStream_t stream);
cudaError_t launchProjectBackward(const FrameConst& F, const InstanceConst& I, const uint32_t* keys,
                                  const float* grads, float4* gMeans, float4* gScales, float4* gQuats, float* gSh,
                                  cudaStream_t stream);
cudaError_t launchL2Loss(const float4* colour, const float* target, uint32_t pixels, float4* dLdColour, float* loss,
                         cudaStream_t stream);

// decode.cu
uint32_t decodeBlocks(uint32_t count);
cudaError_t launchDecode(const float* records, uint32_t count, const ath_encoding& E, float4* positions, uint4* shape,
                         uint32_t* sh, uint64_t* flags, uint32_t* words, cudaStream_t stream);

}   // namespace ath
