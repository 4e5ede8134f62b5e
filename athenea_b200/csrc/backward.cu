// The adjoint of the raster path, for FP32 training parameters.
//
// The reference differentiates only colour (splat_blend.slang:381-398,
// contributionMode 4: each Gaussian's colour gradient is the sum over its
// pixels of weight * dL/dpixel). This pass differentiates everything the
// forward computes from the parameters: the blend in reverse order, then the
// projection (EWA covariance, the Mip-Splatting opacity payback, SH colour,
// sRGB decode, the Jacobian with its frustum clamp).
//
// Nothing is checkpointed: the forward keeps, per pixel, only its final
// transmittance and one past the last record it blended. The reverse walk
// recomputes every record's power and alpha exactly as the forward did (this
// file is built with --fmad=false), so it skips the same records, and divides
// the transmittance back out record by record.
#include <cuda_runtime.h>

#include "adjoint.cuh"
#include "gauss.cuh"
#include "kernels.h"
#include "raster_types.cuh"
#include "splat_math.cuh"

namespace ath {
namespace {

constexpr uint32_t kBwdThreads = kTile * kTile;

__device__ __forceinline__ float warpSum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
    return v;
}

// Sums 16 values over the warp's 32 lanes in 16 shuffles (not 16 x 5): at each
// butterfly step a lane keeps one half of its values and sends the other, so
// the values a lane carries halve while the lanes summed double. Afterwards
// value k's total sits in the lanes whose bits 1..4 spell k (lane >> 1 == k:
// lanes 2k and 2k + 1 both hold it).
__device__ __forceinline__ float warpSum16(float v[16]) {
    const uint32_t lane = threadIdx.x & 31u;
#pragma unroll
    for (int half = 8, bit = 16; half >= 1; half >>= 1, bit >>= 1) {
        const bool upper = (lane & (uint32_t)bit) != 0;
#pragma unroll
        for (int k = 0; k < half; ++k) {
            const float send = upper ? v[k] : v[k + half];
            const float keep = upper ? v[k + half] : v[k];
            v[k] = keep + __shfl_xor_sync(0xFFFFFFFFu, send, bit);
        }
    }
    return v[0] + __shfl_xor_sync(0xFFFFFFFFu, v[0], 1);
}

// dL/d(record) of every slot: centre x y, conic a b c, alpha, colour r g b, view z.
__global__ void __launch_bounds__(kBwdThreads)
    blendBackwardKernel(const FrameConst F, uint32_t pairs, uint32_t slots, const uint2* __restrict__ ranges,
                        const uint32_t* __restrict__ pairValues, const float4* __restrict__ recs,
                        const float* __restrict__ finalT, const uint32_t* __restrict__ lastContrib,
                        const float4* __restrict__ dLdColour, const float* __restrict__ dLdDepth,
                        const float* __restrict__ depthOut, float* __restrict__ grads, uint32_t* __restrict__ status) {
    __shared__ float4 sScreen[kBwdThreads];
    __shared__ float4 sConic[kBwdThreads];
    __shared__ float4 sColour[kBwdThreads];
    __shared__ uint32_t sSlot[kBwdThreads];
    __shared__ float sAcc[kBwdThreads * kGradWords];
    __shared__ uint32_t sMaxLast;

    const uint32_t tile = blockIdx.x;
    const uint32_t tx = tile % F.tilesX, ty = tile / F.tilesX;
    const uint32_t px = tx * kTile + (threadIdx.x % kTile);
    const uint32_t py = ty * kTile + (threadIdx.x / kTile);
    const bool inside = px < F.width && py < F.height;
    uint2 range = ranges[tile];
    if (range.y > pairs || range.x > range.y) {
        if (threadIdx.x == 0) atomicOr(status, kStatusIndexRange);
        range = make_uint2(0, 0);
    }
    const uint32_t at = inside ? py * F.width + px : 0u;
    const float pxc = (float)px + 0.5f, pyc = (float)py + 0.5f;

    const float Tfinal = inside ? finalT[at] : 1.0f;
    const uint32_t last = inside ? min(lastContrib[at], range.y - range.x) : 0u;
    const float4 dC = inside ? dLdColour[at] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    const float dD = (inside && dLdDepth) ? dLdDepth[at] : 0.0f;
    const float cov = 1.0f - Tfinal;
    const bool depthLive = F.depthMode == 0 && cov > 1e-6f && dD != 0.0f;
    const float dDcov = depthLive ? dD / cov : 0.0f;
    const float D = depthLive ? depthOut[at] : 0.0f;
    // alpha channel: 1 - T_N + T_N bg_a, so dA/dalpha_k = T_N (1 - bg_a) / (1 - alpha_k)
    const float dAlphaOut = dC.w * Tfinal * (1.0f - F.bg[3]);

    if (threadIdx.x == 0) sMaxLast = 0;
    __syncthreads();
    if (last) atomicMax(&sMaxLast, last);
    __syncthreads();
    const uint32_t end = range.x + sMaxLast;

    float T = Tfinal;
    float Sr = F.bg[0], Sg = F.bg[1], Sb = F.bg[2], Sz = 0.0f;
    const uint32_t lane = threadIdx.x & 31u;
    for (uint32_t batchEnd = end; batchEnd > range.x;) {
        const uint32_t batchStart = batchEnd - range.x > kBwdThreads ? batchEnd - kBwdThreads : range.x;
        const uint32_t count = batchEnd - batchStart;
        if (threadIdx.x < count) {
            uint32_t s = pairValues[batchStart + threadIdx.x];
            if (s >= slots) {
                atomicOr(status, kStatusIndexRange);
                s = 0;
            }
            sSlot[threadIdx.x] = s;
            sScreen[threadIdx.x] = recs[(size_t)s * 3 + 0];
            sConic[threadIdx.x] = recs[(size_t)s * 3 + 1];
            sColour[threadIdx.x] = recs[(size_t)s * 3 + 2];
        }
        for (uint32_t k = threadIdx.x; k < kBwdThreads * kGradWords; k += kBwdThreads) sAcc[k] = 0.0f;
        __syncthreads();
        for (int j = (int)count - 1; j >= 0; --j) {
            const uint32_t rel = batchStart + (uint32_t)j - range.x;
            float g[kGradWords];
#pragma unroll
            for (int k = 0; k < (int)kGradWords; ++k) g[k] = 0.0f;
            bool live = false;
            if (rel < last) {
                const float4 sc = sScreen[j];
                const float4 k = sConic[j];
                const float dx = pxc - sc.x;
                const float dy = pyc - sc.y;
                const float power = ((k.x * dx) * dx + ((2.0f * k.y) * dx) * dy) + (k.z * dy) * dy;
                if (power <= sc.w) {
                    const float G = exp_f((-0.5f) * power);
                    const float raw = falloffAlpha(fabsf(k.w), G);
                    const float alpha = fminf(0.99f, raw);
                    if (alpha >= kFaint) {
                        live = true;
                        const float4 c = sColour[j];
                        const float oneMinus = 1.0f - alpha;
                        const float Tb = T / oneMinus;
                        const float w = Tb * alpha;
                        g[kGradR] = w * dC.x;
                        g[kGradG] = w * dC.y;
                        g[kGradB] = w * dC.z;
                        float dAlpha = Tb * ((c.x - Sr) * dC.x + (c.y - Sg) * dC.y + (c.z - Sb) * dC.z) +
                                       dAlphaOut / oneMinus;
                        if (depthLive) {
                            g[kGradZ] = dDcov * w;
                            dAlpha += dDcov * (Tb * (sc.z - Sz) - D * Tfinal / oneMinus);
                        }
                        Sr = alpha * c.x + oneMinus * Sr;
                        Sg = alpha * c.y + oneMinus * Sg;
                        Sb = alpha * c.z + oneMinus * Sb;
                        Sz = alpha * sc.z + oneMinus * Sz;
                        T = Tb;
                        if (raw < 0.99f && k.w <= 1.0f) {
                            // alpha = a' G, G = exp(-power / 2)
                            g[kGradAlpha] = dAlpha * G;
                            const float dPower = -0.5f * alpha * dAlpha;
                            g[kGradA] = dPower * (dx * dx);
                            g[kGradB2] = dPower * (2.0f * dx * dy);
                            g[kGradC] = dPower * (dy * dy);
                            g[kGradCx] = dPower * (-2.0f * (k.x * dx + k.y * dy));
                            g[kGradCy] = dPower * (-2.0f * (k.y * dx + k.z * dy));
                        }
                    }
                }
            }
            if (__any_sync(0xFFFFFFFFu, live)) {
                float v16[16];
#pragma unroll
                for (int k = 0; k < 16; ++k) v16[k] = k < (int)kGradWords ? g[k] : 0.0f;
                const float v = warpSum16(v16);
                const uint32_t k = lane >> 1;   // lanes 2k and 2k + 1 hold value k's total
                if ((lane & 1u) == 0 && k < kGradWords && v != 0.0f) atomicAdd(&sAcc[j * kGradWords + k], v);
            }
        }
        __syncthreads();
        for (uint32_t k = threadIdx.x; k < count * kGradWords; k += kBwdThreads) {
            const float v = sAcc[k];
            if (v != 0.0f) atomicAdd(&grads[(size_t)sSlot[k / kGradWords] * kGradWords + k % kGradWords], v);
        }
        __syncthreads();
        batchEnd = batchStart;
    }
}

// The projection's adjoint, one thread a Gaussian: dL/d(record) -> dL/d(parameters), added in.
__global__ void __launch_bounds__(128)
    projectBackwardKernel(const FrameConst F, const InstanceConst I, const uint32_t* __restrict__ keys,
                          const float* __restrict__ grads, float4* __restrict__ gMeans, float4* __restrict__ gScales,
                          float4* __restrict__ gQuats, float* __restrict__ gSh) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= I.count) return;
    const uint32_t slot = I.base + i;
    if (keys[slot] >= kCulledKey) return;
    const float* gr = grads + (size_t)slot * kGradWords;
    float gw[kGradWords];
#pragma unroll
    for (int k = 0; k < (int)kGradWords; ++k) gw[k] = gr[k];
    ParamGrad acc;
    acc.clear();
    projectAdjoint<kLayoutParams>(F, I, i, gw, acc);
    acc.addTo(i, I.shStride, gMeans, gScales, gQuats, gSh);
}

// L = mean over pixels and r g b of (colour - target)^2: its value (added into
// *loss) and dL/dcolour (float4 a pixel, alpha 0).
__global__ void __launch_bounds__(256)
    l2LossKernel(const float4* __restrict__ colour, const float* __restrict__ target, uint32_t pixels, float scale,
                 float4* __restrict__ dLdColour, float* __restrict__ loss) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    float l = 0.0f;
    if (p < pixels) {
        const float4 c = colour[p];
        const float er = c.x - target[p * 3 + 0], eg = c.y - target[p * 3 + 1], eb = c.z - target[p * 3 + 2];
        l = (er * er + eg * eg + eb * eb) * scale;
        dLdColour[p] = make_float4(2.0f * scale * er, 2.0f * scale * eg, 2.0f * scale * eb, 0.0f);
    }
    __shared__ float sPart[8];
    l = warpSum(l);
    if ((threadIdx.x & 31u) == 0) sPart[threadIdx.x >> 5] = l;
    __syncthreads();
    if (threadIdx.x == 0) {
        float b = 0.0f;
#pragma unroll
        for (int w = 0; w < 8; ++w) b += sPart[w];
        if (b != 0.0f) atomicAdd(loss, b);
    }
}

}   // namespace

cudaError_t launchBlendBackward(const FrameConst& F, uint32_t pairs, uint32_t slots, const uint2* ranges,
                                const uint32_t* pairValues, const float4* recs, const float* finalT,
                                const uint32_t* lastContrib, const float4* dLdColour, const float* dLdDepth,
                                const float* depthOut, float* grads, uint32_t* status, cudaStream_t stream) {
    const uint32_t tiles = F.tilesX * F.tilesY;
    if (tiles == 0) return cudaSuccess;
    blendBackwardKernel<<<tiles, kBwdThreads, 0, stream>>>(F, pairs, slots, ranges, pairValues, recs, finalT,
                                                          lastContrib, dLdColour, dLdDepth, depthOut, grads, status);
    return cudaGetLastError();
}

cudaError_t launchProjectBackward(const FrameConst& F, const InstanceConst& I, const uint32_t* keys,
                                  const float* grads, float4* gMeans, float4* gScales, float4* gQuats, float* gSh,
                                  cudaStream_t stream) {
    if (I.count == 0) return cudaSuccess;
    projectBackwardKernel<<<(I.count + 127) / 128, 128, 0, stream>>>(F, I, keys, grads, gMeans, gScales, gQuats, gSh);
    return cudaGetLastError();
}

cudaError_t launchL2Loss(const float4* colour, const float* target, uint32_t pixels, float4* dLdColour, float* loss,
                         cudaStream_t stream) {
    if (pixels == 0) return cudaSuccess;
    l2LossKernel<<<(pixels + 255) / 256, 256, 0, stream>>>(colour, target, pixels, 1.0f / (3.0f * (float)pixels),
                                                          dLdColour, loss);
    return cudaGetLastError();
}

}   // namespace ath
