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

// common/sh.slang:25-51's basis functions (after the constant term) and their
// gradients with respect to the direction's three components.
__device__ __forceinline__ void shBasis(uint32_t degree, float x, float y, float z, float Y[15], float dY[15][3]) {
    const float C1 = 0.4886025119029199f;
    const float C2[5] = {1.0925484305920792f, -1.0925484305920792f, 0.31539156525252005f, -1.0925484305920792f,
                         0.5462742152960396f};
    const float C3[7] = {-0.5900435899266435f, 2.890611442640554f, -0.4570457994644658f, 0.3731763325901154f,
                         -0.4570457994644658f, 1.445305721320277f, -0.5900435899266435f};
#pragma unroll
    for (int k = 0; k < 15; ++k) {
        Y[k] = 0.0f;
        dY[k][0] = dY[k][1] = dY[k][2] = 0.0f;
    }
    if (degree < 1) return;
    Y[0] = -C1 * y; dY[0][1] = -C1;
    Y[1] = C1 * z;  dY[1][2] = C1;
    Y[2] = -C1 * x; dY[2][0] = -C1;
    if (degree < 2) return;
    const float xx = x * x, yy = y * y, zz = z * z, xy = x * y, yz = y * z, xz = x * z;
    Y[3] = C2[0] * xy;                   dY[3][0] = C2[0] * y; dY[3][1] = C2[0] * x;
    Y[4] = C2[1] * yz;                   dY[4][1] = C2[1] * z; dY[4][2] = C2[1] * y;
    Y[5] = C2[2] * (2.0f * zz - xx - yy); dY[5][0] = -2.0f * C2[2] * x; dY[5][1] = -2.0f * C2[2] * y; dY[5][2] = 4.0f * C2[2] * z;
    Y[6] = C2[3] * xz;                   dY[6][0] = C2[3] * z; dY[6][2] = C2[3] * x;
    Y[7] = C2[4] * (xx - yy);            dY[7][0] = 2.0f * C2[4] * x; dY[7][1] = -2.0f * C2[4] * y;
    if (degree < 3) return;
    Y[8] = C3[0] * y * (3.0f * xx - yy);
    dY[8][0] = C3[0] * 6.0f * xy; dY[8][1] = C3[0] * (3.0f * xx - 3.0f * yy);
    Y[9] = C3[1] * xy * z;
    dY[9][0] = C3[1] * yz; dY[9][1] = C3[1] * xz; dY[9][2] = C3[1] * xy;
    Y[10] = C3[2] * y * (4.0f * zz - xx - yy);
    dY[10][0] = C3[2] * (-2.0f * xy); dY[10][1] = C3[2] * (4.0f * zz - xx - 3.0f * yy); dY[10][2] = C3[2] * 8.0f * yz;
    Y[11] = C3[3] * z * (2.0f * zz - 3.0f * xx - 3.0f * yy);
    dY[11][0] = C3[3] * (-6.0f * xz); dY[11][1] = C3[3] * (-6.0f * yz); dY[11][2] = C3[3] * (6.0f * zz - 3.0f * xx - 3.0f * yy);
    Y[12] = C3[4] * x * (4.0f * zz - xx - yy);
    dY[12][0] = C3[4] * (4.0f * zz - 3.0f * xx - yy); dY[12][1] = C3[4] * (-2.0f * xy); dY[12][2] = C3[4] * 8.0f * xz;
    Y[13] = C3[5] * z * (xx - yy);
    dY[13][0] = C3[5] * 2.0f * xz; dY[13][1] = C3[5] * (-2.0f * yz); dY[13][2] = C3[5] * (xx - yy);
    Y[14] = C3[6] * x * (xx - 3.0f * yy);
    dY[14][0] = C3[6] * (3.0f * xx - 3.0f * yy); dY[14][1] = C3[6] * (-6.0f * xy);
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

    const Gauss g = loadGauss<kLayoutParams>(I, i);
    const Geometry G = projectGeometry(F, I, g, g.opacity);
    const float* m = I.m;

    // ---- colour: c = decode(base + rest(dir)) ------------------------------
    float dp[3] = {0.0f, 0.0f, 0.0f};
    const uint32_t degree = min(degreeOf(I.restPerColour), F.shLimit);
    const float ex = g.px - I.eye[0], ey = g.py - I.eye[1], ez = g.pz - I.eye[2];
    const float len = sqrtf((ex * ex + ey * ey) + ez * ez);
    const float dir[3] = {ex / len, ey / len, ez / len};
    float Y[15], dY[15][3];
    shBasis(degree, dir[0], dir[1], dir[2], Y, dY);
    const float* shRow = I.shf + (size_t)i * I.shStride;
    float* gRow = gSh + (size_t)i * I.shStride;
    const uint32_t bases = degree == 3 ? 15 : degree == 2 ? 8 : degree == 1 ? 3 : 0;
    float dDir[3] = {0.0f, 0.0f, 0.0f};
    const float gc[3] = {gw[kGradR], gw[kGradG], gw[kGradB]};
#pragma unroll
    for (int ch = 0; ch < 3; ++ch) {
        float v = g.base[ch];
#pragma unroll
        for (uint32_t k = 0; k < 15; ++k)
            if (k < bases) v += Y[k] * shRow[3 + k * 3 + ch];
        float dcdv;
        if (I.linear != 0) {
            dcdv = v > 0.0f ? 1.0f : 0.0f;
        } else {
            dcdv = v <= 0.0f ? 0.0f : v <= 0.04045f ? 1.0f / 12.92f : (2.4f / 1.055f) * pow_f((v + 0.055f) / 1.055f, 1.4f);
        }
        const float dv = gc[ch] * dcdv;
        gRow[ch] += kSH0 * dv;
#pragma unroll
        for (uint32_t k = 0; k < 15; ++k) {
            if (k >= bases) continue;
            gRow[3 + k * 3 + ch] += Y[k] * dv;
            const float coef = shRow[3 + k * 3 + ch] * dv;
            dDir[0] += dY[k][0] * coef;
            dDir[1] += dY[k][1] * coef;
            dDir[2] += dY[k][2] * coef;
        }
    }
    {
        // dir = e / |e|
        const float dd = dDir[0] * dir[0] + dDir[1] * dir[1] + dDir[2] * dir[2];
#pragma unroll
        for (int k = 0; k < 3; ++k) dp[k] += (dDir[k] - dir[k] * dd) / len;
    }

    // ---- opacity and the payback: alpha = paidOpacity(sigmoid(logit), paid) ----
    const float o = g.opacity;
    float dAlphaDo, dAlphaDpaid;
    if (o > 1.0f) {
        dAlphaDo = 1.0f;
        dAlphaDpaid = 0.0f;
    } else if (G.paid * o >= kFaint) {
        dAlphaDo = G.paid;
        dAlphaDpaid = o - kFaint;
    } else {
        dAlphaDo = G.paid;
        dAlphaDpaid = o;
    }
    const float dLogit = gw[kGradAlpha] * dAlphaDo * o * (1.0f - o);
    const float dPaid = gw[kGradAlpha] * dAlphaDpaid;
    float dDetBefore = 0.0f, dDet = 0.0f;
    if (G.detBefore > 0.0f && G.paid > 0.0f) {
        float dFiltered = 0.0f;
        const float filtered = sqrtf(G.detBefore / G.det);
        if (I.antialias != 0) {
            dFiltered = dPaid;
        } else if (I.paidAt > 0.0f && filtered / I.paidAt < 1.0f) {
            dFiltered = dPaid / I.paidAt;
        }
        dDetBefore = dFiltered * 0.5f * filtered / G.detBefore;
        dDet = -dFiltered * 0.5f * filtered / G.det;
    }

    // ---- the conic: (A, B, C) = (c', -b, a') / det, a' = a + 0.3, c' = c + 0.3 --
    const float a2 = G.a + 0.3f, c2 = G.c + 0.3f, b = G.b;
    const float det = G.det, det2 = det * det;
    const float gA = gw[kGradA], gB = gw[kGradB2], gC = gw[kGradC];
    float da2 = gA * (-c2 * c2 / det2) + gB * (b * c2 / det2) + gC * (1.0f / det - a2 * c2 / det2);
    float db = gA * (2.0f * b * c2 / det2) + gB * (-1.0f / det - 2.0f * b * b / det2) + gC * (2.0f * a2 * b / det2);
    float dc2 = gA * (1.0f / det - c2 * a2 / det2) + gB * (b * a2 / det2) + gC * (-a2 * a2 / det2);
    da2 += dDet * c2;
    dc2 += dDet * a2;
    db += dDet * (-2.0f * b);
    const float da = da2 + dDetBefore * G.c;
    const float dc = dc2 + dDetBefore * G.a;
    db += dDetBefore * (-2.0f * b);

    // ---- the covariance: a = ax.ax, b = ax.ay, c = ay.ay; ax = t3 M, ay = u3 M --
    float ax[3], ay[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        ax[j] = (G.t3[0] * G.M[0][j] + G.t3[1] * G.M[1][j]) + G.t3[2] * G.M[2][j];
        ay[j] = (G.u3[0] * G.M[0][j] + G.u3[1] * G.M[1][j]) + G.u3[2] * G.M[2][j];
    }
    float dax[3], day[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        dax[j] = 2.0f * da * ax[j] + db * ay[j];
        day[j] = db * ax[j] + 2.0f * dc * ay[j];
    }
    float dt3[3], du3[3], dScale[3] = {0.0f, 0.0f, 0.0f}, dR[3][3];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        dt3[r] = G.M[r][0] * dax[0] + G.M[r][1] * dax[1] + G.M[r][2] * dax[2];
        du3[r] = G.M[r][0] * day[0] + G.M[r][1] * day[1] + G.M[r][2] * day[2];
#pragma unroll
        for (int col = 0; col < 3; ++col) {
            const float dM = G.t3[r] * dax[col] + G.u3[r] * day[col];
            dScale[col] += dM * G.R[r][col];
            dR[r][col] = dM * g.scale[col];
        }
    }
    // ---- the rotation: R(q), q = raw / |raw| --------------------------------
    const float x = g.q[0], y = g.q[1], z = g.q[2], w = g.q[3];
    float dq[4];   // x y z w
    dq[0] = 2.0f * (y * dR[0][1] + z * dR[0][2] + y * dR[1][0] - 2.0f * x * dR[1][1] - w * dR[1][2] + z * dR[2][0] +
                    w * dR[2][1] - 2.0f * x * dR[2][2]);
    dq[1] = 2.0f * (-2.0f * y * dR[0][0] + x * dR[0][1] + w * dR[0][2] + x * dR[1][0] + z * dR[1][2] - w * dR[2][0] +
                    z * dR[2][1] - 2.0f * y * dR[2][2]);
    dq[2] = 2.0f * (-2.0f * z * dR[0][0] - w * dR[0][1] + x * dR[0][2] + w * dR[1][0] - 2.0f * z * dR[1][1] +
                    y * dR[1][2] + x * dR[2][0] + y * dR[2][1]);
    dq[3] = 2.0f * (-z * dR[0][1] + y * dR[0][2] + z * dR[1][0] - x * dR[1][2] - y * dR[2][0] + x * dR[2][1]);
    const float4 qraw = __ldg(reinterpret_cast<const float4*>(I.quats) + i);
    const float qlen = sqrtf(((qraw.x * qraw.x + qraw.y * qraw.y) + qraw.z * qraw.z) + qraw.w * qraw.w);
    const float qd = dq[0] * x + dq[1] * y + dq[2] * z + dq[3] * w;
    const float4 dQuat = make_float4((dq[3] - w * qd) / qlen, (dq[0] - x * qd) / qlen, (dq[1] - y * qd) / qlen,
                                     (dq[2] - z * qd) / qlen);   // w x y z

    // ---- the Jacobian and the centre: t = W p + tw -------------------------
    const float djx0 = dt3[0] * m[0] + dt3[1] * m[1] + dt3[2] * m[2];
    const float djx2 = dt3[0] * m[8] + dt3[1] * m[9] + dt3[2] * m[10];
    const float djy1 = du3[0] * m[4] + du3[1] * m[5] + du3[2] * m[6];
    const float djy2 = du3[0] * m[8] + du3[1] * m[9] + du3[2] * m[10];
    float dt[3] = {0.0f, 0.0f, gw[kGradZ]};
    if (F.orthographic != 0) {
        dt[0] += gw[kGradCx] * F.focalX;
        dt[1] += gw[kGradCy] * F.focalY;
    } else {
        const float invZ = 1.0f / G.tz, invZ2 = invZ * invZ, invZ3 = invZ2 * invZ;
        dt[0] += gw[kGradCx] * F.focalX * invZ;
        dt[1] += gw[kGradCy] * F.focalY * invZ;
        dt[2] += -gw[kGradCx] * F.focalX * G.tx * invZ2 - gw[kGradCy] * F.focalY * G.ty * invZ2;
        dt[2] += -djx0 * F.focalX * invZ2 - djy1 * F.focalY * invZ2;
        if (G.clampX) {
            dt[2] += djx2 * F.focalX * G.txc * invZ3;
        } else {
            dt[0] += -djx2 * F.focalX * invZ2;
            dt[2] += djx2 * 2.0f * F.focalX * G.tx * invZ3;
        }
        if (G.clampY) {
            dt[2] += djy2 * F.focalY * G.tyc * invZ3;
        } else {
            dt[1] += -djy2 * F.focalY * invZ2;
            dt[2] += djy2 * 2.0f * F.focalY * G.ty * invZ3;
        }
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) dp[k] += m[k] * dt[0] + m[4 + k] * dt[1] + m[8 + k] * dt[2];

    float4 gm = gMeans[i];
    gm.x += dp[0]; gm.y += dp[1]; gm.z += dp[2]; gm.w += dLogit;
    gMeans[i] = gm;
    float4 gs = gScales[i];
    gs.x += dScale[0] * g.scale[0]; gs.y += dScale[1] * g.scale[1]; gs.z += dScale[2] * g.scale[2];
    gScales[i] = gs;
    float4 gq = gQuats[i];
    gq.x += dQuat.x; gq.y += dQuat.y; gq.z += dQuat.z; gq.w += dQuat.w;
    gQuats[i] = gq;
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
