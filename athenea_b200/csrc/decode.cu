// The upload's decode: 3DGS-encoded float records to the packed layout the
// rasteriser reads (common/packing.slang:5-27). Follows
// scene/splat_validate.slang:16-31 (which records are kept) and
// scene/splat_decode.slang:45-173 (how each is packed), with the 3DGS field
// modes of scene/splat_encoding.slang:71-113 (logit opacity, log scale, SH DC,
// rest coefficients colour-outer). The reference validates, prefix-sums and
// decodes in three dispatches; here one kernel does all three, the compaction
// by a decoupled look-back over a ticketed block order.
//
// Built with --fmad=false: see splat_math.cuh.
#include <cuda_runtime.h>
#include <cuda_fp16.h>

#include "kernels.h"
#include "raster_types.cuh"
#include "splat_math.cuh"

namespace ath {
namespace {

constexpr uint32_t kDecodeThreads = 256;
constexpr float kSH0 = 0.28209479177387814f;

__device__ __forceinline__ float halfSafe(float v) { return fminf(fmaxf(v, -65000.0f), 65000.0f); }
__device__ __forceinline__ uint32_t toHalfBits(float v) {
    return (uint32_t)__half_as_ushort(__float2half_rn(v));
}
__device__ __forceinline__ uint32_t packHalves(float a, float b) { return toHalfBits(a) | (toHalfBits(b) << 16); }

// common/packing.slang:33-57; `round` as Slang's CUDA target emits it (roundf).
__device__ uint32_t encodeQuaternion(float q0, float q1, float q2, float q3) {
    const float kSqrtHalf = 0.70710678f;
    const float len = sqrtf(((q0 * q0 + q1 * q1) + q2 * q2) + q3 * q3);
    float q[4] = {q0 / len, q1 / len, q2 / len, q3 / len};
    uint32_t largest = 0;
    float best = fabsf(q[0]);
#pragma unroll
    for (uint32_t k = 1; k < 4; ++k) {
        if (fabsf(q[k]) > best) {
            best = fabsf(q[k]);
            largest = k;
        }
    }
    const bool flip = (largest == 0 ? q[0] : largest == 1 ? q[1] : largest == 2 ? q[2] : q[3]) < 0.0f;
    uint32_t word = largest;
    uint32_t shift = 22;
#pragma unroll
    for (uint32_t k = 0; k < 4; ++k) {
        if (k == largest) continue;
        const float v = flip ? -q[k] : q[k];
        const float unit = clampf((v / kSqrtHalf) * 0.5f + 0.5f, 0.0f, 1.0f);
        word |= (uint32_t)roundf(unit * 1023.0f) << shift;
        shift -= 10;
    }
    return word;
}

__global__ void __launch_bounds__(kDecodeThreads)
    decodeKernel(const float* __restrict__ records, uint32_t count, const ath_encoding E, float4* __restrict__ positions,
                 uint4* __restrict__ shape, uint32_t* __restrict__ sh, uint64_t* __restrict__ flags,
                 uint32_t* __restrict__ words) {
    __shared__ uint32_t sTicket;
    __shared__ uint32_t sWarp[kDecodeThreads / 32];
    __shared__ uint64_t sPrefix;
    if (threadIdx.x == 0) sTicket = atomicAdd(&words[0], 1u);
    __syncthreads();
    const uint32_t b = sTicket;
    const uint32_t i = b * kDecodeThreads + threadIdx.x;
    bool valid = false;
    float p[3] = {0, 0, 0}, a = 0.0f, ls[3] = {0, 0, 0};
    const float* r = records + (size_t)i * E.stride;
    if (i < count) {
        p[0] = r[E.x];
        p[1] = r[E.y];
        p[2] = r[E.z];
        a = 1.0f / (1.0f + exp_f(-r[E.opacity]));
        ls[0] = r[E.scale0];
        ls[1] = r[E.scale1];
        ls[2] = r[E.scale2];
        uint32_t flats = 0;
        bool ok = true;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            if (ls[k] < -30.0f) ls[k] = __int_as_float(0xFF800000);   // a surfel's flat axis
            if (ls[k] <= -1024.0f) {
                flats += 1;
            } else if (!isfinite(ls[k]) || !(fabsf(ls[k]) < 60.0f)) {
                ok = false;
            }
        }
        valid = isfinite(p[0]) && isfinite(p[1]) && isfinite(p[2]) && flats <= 1u && ok && a >= kFaint;
    }
    // compaction: exclusive scan of `valid` over the records, in record order
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t ballot = __ballot_sync(0xFFFFFFFFu, valid);
    if (lane == 0) sWarp[warp] = __popc(ballot);
    __syncthreads();
    uint32_t warpBase = 0, blockTotal = 0;
#pragma unroll
    for (uint32_t w = 0; w < kDecodeThreads / 32; ++w) {
        warpBase += w < warp ? sWarp[w] : 0u;
        blockTotal += sWarp[w];
    }
    if (warp == 0) {
        const uint64_t prefix = lookbackExclusive(flags, b, blockTotal, &words[1]);
        if (lane == 0) {
            sPrefix = prefix;
            if (b == gridDim.x - 1) words[2] = (uint32_t)(prefix + blockTotal);
        }
    }
    __syncthreads();
    if (!valid) return;
    const uint32_t j = (uint32_t)sPrefix + warpBase + __popc(ballot & ((1u << lane) - 1u));
    if (j >= count) {   // never, for a look-back that completed
        atomicOr(&words[1], kStatusIndexRange);
        return;
    }
    positions[j] = make_float4(p[0], p[1], p[2], clampf(a, 0.0f, 5.0f));
    const float q0 = r[E.rot_x], q1 = r[E.rot_y], q2 = r[E.rot_z], q3 = r[E.rot_w];
    const float qLength = sqrtf(((q0 * q0 + q1 * q1) + q2 * q2) + q3 * q3);
    const uint32_t rotation = qLength > 1e-8f ? encodeQuaternion(q0, q1, q2, q3) : encodeQuaternion(0, 0, 0, 1);
    const float base0 = 0.5f + kSH0 * r[E.dc0], base1 = 0.5f + kSH0 * r[E.dc1], base2 = 0.5f + kSH0 * r[E.dc2];
    shape[j] = make_uint4(rotation, packHalves(halfSafe(ls[0]), halfSafe(ls[1])),
                          packHalves(halfSafe(ls[2]), halfSafe(base0)), packHalves(halfSafe(base1), halfSafe(base2)));
    const uint32_t keep = E.keep_per_colour;
    const uint32_t shWords = keep == 0 ? 1 : (keep * 3 + 1) / 2;
    uint32_t* row = sh + (size_t)j * shWords;
    if (keep == 0) {
        row[0] = 0;
        return;
    }
    uint32_t half = 0, word = 0, filled = 0;
    for (uint32_t basis = 0; basis < keep; ++basis) {
        for (uint32_t colour = 0; colour < 3; ++colour) {
            const float value = r[E.rest_base + colour * E.file_per_colour + basis];
            word |= toHalfBits(halfSafe(value)) << (filled * 16);
            filled += 1;
            if (filled == 2) {
                row[half++] = word;
                word = 0;
                filled = 0;
            }
        }
    }
    if (filled == 1) row[half] = word;
}

}   // namespace

uint32_t decodeBlocks(uint32_t count) { return (count + kDecodeThreads - 1) / kDecodeThreads; }

// words: [0] ticket, [1] status, [2] kept; flags: decodeBlocks(count) words. Both zeroed by the caller.
cudaError_t launchDecode(const float* records, uint32_t count, const ath_encoding& E, float4* positions, uint4* shape,
                         uint32_t* sh, uint64_t* flags, uint32_t* words, cudaStream_t stream) {
    if (count == 0) return cudaSuccess;
    decodeKernel<<<decodeBlocks(count), kDecodeThreads, 0, stream>>>(records, count, E, positions, shape, sh, flags,
                                                                     words);
    return cudaGetLastError();
}

}   // namespace ath
