// One Gaussian as the projection reads it, from each storage layout the
// rasteriser accepts, and the projection's geometry (splat/splat_project.slang:
// 497-776) as one device function the forward and the backward both call, so
// the backward recomputes exactly what the forward computed.
#pragma once

#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_fp8.h>

#include "raster_types.cuh"
#include "splat_math.cuh"

namespace ath {

// Storage layouts of a cloud.
enum Layout : uint32_t {
    kLayoutPacked = 0,   // common/packing.slang: float4 position+opacity, uint4 shape, f16 SH words
    kLayoutParams = 1,   // FP32 training parameters (ath_params)
    kLayoutMixed = 2,    // FP32 geometry, BF16 SH DC and band 1, FP8 e4m3 bands 2-3 with an FP32 scale
};

constexpr float kSH0 = 0.28209479177387814f;   // common/packing.slang:445

struct Gauss {
    float px, py, pz, opacity;
    float scale[3];
    float q[4];     // x y z w
    float base[3];  // the constant term's colour, 0.5 + SH0 dc
};

// ---- packed (the reference's GpuSplats) ---------------------------------------
__device__ __forceinline__ Gauss loadPacked(const InstanceConst& I, uint32_t i) {
    Gauss g;
    const float4 po = __ldg(I.positions + i);
    const uint4 sh4 = __ldg(I.shape + i);
    g.px = po.x; g.py = po.y; g.pz = po.z; g.opacity = po.w;
    g.scale[0] = exp_f(lowHalf(sh4.y));
    g.scale[1] = exp_f(highHalf(sh4.y));
    g.scale[2] = exp_f(lowHalf(sh4.z));
    decodeQuaternion(sh4.x, g.q);
    g.base[0] = highHalf(sh4.z);
    g.base[1] = lowHalf(sh4.w);
    g.base[2] = highHalf(sh4.w);
    return g;
}

// ---- FP32 training parameters ------------------------------------------------
// means float4 (x y z, opacity logit), scales float4 (log scales), quats float4
// (w x y z, any length), shf: DC rgb then rest rgb per basis, shStride floats.
__device__ __forceinline__ float sigmoid_f(float v) { return 1.0f / (1.0f + exp_f(-v)); }

__device__ __forceinline__ Gauss loadParams(const InstanceConst& I, uint32_t i) {
    Gauss g;
    const float4 m = __ldg(reinterpret_cast<const float4*>(I.means) + i);
    const float4 s = __ldg(reinterpret_cast<const float4*>(I.scales) + i);
    const float4 q = __ldg(reinterpret_cast<const float4*>(I.quats) + i);
    g.px = m.x; g.py = m.y; g.pz = m.z;
    g.opacity = sigmoid_f(m.w);
    g.scale[0] = exp_f(s.x);
    g.scale[1] = exp_f(s.y);
    g.scale[2] = exp_f(s.z);
    const float len = sqrtf(((q.x * q.x + q.y * q.y) + q.z * q.z) + q.w * q.w);
    g.q[0] = q.y / len;   // x
    g.q[1] = q.z / len;   // y
    g.q[2] = q.w / len;   // z
    g.q[3] = q.x / len;   // w
    const float* c = I.shf + (size_t)i * I.shStride;
    g.base[0] = 0.5f + kSH0 * __ldg(c + 0);
    g.base[1] = 0.5f + kSH0 * __ldg(c + 1);
    g.base[2] = 0.5f + kSH0 * __ldg(c + 2);
    return g;
}

// ---- the rest coefficients, coefficient `index` = basis * 3 + channel -----------
template <uint32_t L>
__device__ __forceinline__ float restAt(const InstanceConst& I, uint32_t i, uint32_t index) {
    if constexpr (L == kLayoutPacked) {
        const uint32_t word = __ldg(I.sh + (size_t)i * I.shWords + index / 2);
        return (index & 1u) == 0u ? lowHalf(word) : highHalf(word);
    } else if constexpr (L == kLayoutParams) {
        return __ldg(I.shf + (size_t)i * I.shStride + 3 + index);
    } else {
        // mixed: DC and band 1 (indices < 9) in BF16 after the DC's 3; bands 2-3 in FP8 e4m3 times a scale
        if (index < 9) {
            const __nv_bfloat16* b = reinterpret_cast<const __nv_bfloat16*>(I.shLow) + (size_t)i * 12;
            return __bfloat162float(b[3 + index]);
        }
        const __nv_fp8_e4m3* e = reinterpret_cast<const __nv_fp8_e4m3*>(I.shHigh) + (size_t)i * 36;
        return float(e[index - 9]) * __ldg(I.shScale + i);
    }
}

// ---- the mixed layout's SH of one Gaussian, held packed in 16 registers -------
// Loaded with 13 word loads instead of one load a coefficient; rest(index) is
// restAt<kLayoutMixed>'s value to the bit (a BF16's bits are a float's top
// half; an e4m3 widens exactly and takes the same FP32 product with the scale).
struct MixedSh {
    uint32_t low[6];    // 12 BF16: DC r g b, then band 1's 9
    uint32_t high[9];   // 36 e4m3: bands 2 and 3
    float scale;

    __device__ __forceinline__ float bf16At(uint32_t k) const {
        const uint32_t word = low[k >> 1];
        return __uint_as_float((k & 1u) ? (word & 0xFFFF0000u) : (word << 16));
    }
    // coefficient `index` = basis * 3 + channel of the rest (after the DC)
    __device__ __forceinline__ float rest(uint32_t index) const {
        if (index < 9) return bf16At(3 + index);
        const uint32_t k = index - 9;
        __nv_fp8_e4m3 e;
        e.__x = (__nv_fp8_storage_t)((high[k >> 2] >> (8 * (k & 3u))) & 0xFFu);
        return float(e) * scale;
    }
};

__device__ __forceinline__ MixedSh loadMixedSh(const InstanceConst& I, uint32_t i) {
    MixedSh s;
    const uint2* low = reinterpret_cast<const uint2*>(reinterpret_cast<const uint8_t*>(I.shLow) + (size_t)i * 24);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const uint2 w = __ldg(low + k);
        s.low[2 * k] = w.x;
        s.low[2 * k + 1] = w.y;
    }
    const uint32_t* high = reinterpret_cast<const uint32_t*>(reinterpret_cast<const uint8_t*>(I.shHigh) + (size_t)i * 36);
#pragma unroll
    for (int k = 0; k < 9; ++k) s.high[k] = __ldg(high + k);
    s.scale = __ldg(I.shScale + i);
    return s;
}

template <uint32_t L>
__device__ __forceinline__ Gauss loadGauss(const InstanceConst& I, uint32_t i) {
    if constexpr (L == kLayoutPacked) {
        return loadPacked(I, i);
    } else if constexpr (L == kLayoutParams) {
        return loadParams(I, i);
    } else {
        Gauss g;
        const float4 m = __ldg(reinterpret_cast<const float4*>(I.means) + i);
        const float4 s = __ldg(reinterpret_cast<const float4*>(I.scales) + i);
        const float4 q = __ldg(reinterpret_cast<const float4*>(I.quats) + i);
        g.px = m.x; g.py = m.y; g.pz = m.z;
        g.opacity = sigmoid_f(m.w);
        g.scale[0] = exp_f(s.x);
        g.scale[1] = exp_f(s.y);
        g.scale[2] = exp_f(s.z);
        const float len = sqrtf(((q.x * q.x + q.y * q.y) + q.z * q.z) + q.w * q.w);
        g.q[0] = q.y / len;
        g.q[1] = q.z / len;
        g.q[2] = q.w / len;
        g.q[3] = q.x / len;
        const __nv_bfloat16* b = reinterpret_cast<const __nv_bfloat16*>(I.shLow) + (size_t)i * 12;
        g.base[0] = 0.5f + kSH0 * __bfloat162float(b[0]);
        g.base[1] = 0.5f + kSH0 * __bfloat162float(b[1]);
        g.base[2] = 0.5f + kSH0 * __bfloat162float(b[2]);
        return g;
    }
}

// ---- the projection's geometry ------------------------------------------------
struct Geometry {
    uint32_t cull;        // 0 kept, else the cull reason (frame.slang:43-48) of what ran so far
    float tx, ty, tz;     // view position
    float cx, cy;         // screen centre
    float a, b, c;        // the 2D covariance before the dilation
    float det, detBefore; // after and before the +0.3 dilation
    float paid, alpha;
    float ca, cb, cc;     // the conic
    float fr, fs;         // the factored conic's ratio and tail (mixed path only)
    float cutoff;
    bool clampX, clampY;  // the Jacobian's point was clamped to the frustum's 1.3x
    bool wide;            // determinants and conic from wideCovariance (mixed path only)
    float txc, tyc;
    float jx0, jx2, jy1, jy2;
    float t3[3], u3[3];   // J W rows
    float M[3][3];        // R diag(s)
    float R[3][3];
};

// ---- near-degenerate footprints in FP64 ----------------------------------------
// A footprint whose dilated 2D covariance has det < 1e-6 trace^2 (a long thin
// needle seen across hundreds of pixels) loses its determinant to cancellation
// in FP32: a' c' ~ b^2, and the undilated determinant a c - b^2 that sets the
// paid opacity can come out at zero or below. The mixed-precision path
// recomputes that covariance from the same FP32 Jacobian rows and R diag(s) in
// FP64 (the products of FP32 factors are exact there), and takes the
// determinants, the paid opacity and the inverse from it.
struct WideCovariance {
    double a2, b, c2;        // the dilated covariance
    double det, detBefore;   // its determinant, and the undilated one
};

__device__ __forceinline__ WideCovariance wideCovariance(const float t3[3], const float u3[3], const float M[3][3]) {
    double ax[3], ay[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        ax[j] = ((double)t3[0] * M[0][j] + (double)t3[1] * M[1][j]) + (double)t3[2] * M[2][j];
        ay[j] = ((double)u3[0] * M[0][j] + (double)u3[1] * M[1][j]) + (double)u3[2] * M[2][j];
    }
    WideCovariance W;
    const double a = (ax[0] * ax[0] + ax[1] * ax[1]) + ax[2] * ax[2];
    W.b = (ax[0] * ay[0] + ax[1] * ay[1]) + ax[2] * ay[2];
    const double c = (ay[0] * ay[0] + ay[1] * ay[1]) + ay[2] * ay[2];
    W.a2 = a + 0.3;
    W.c2 = c + 0.3;
    W.detBefore = a * c - W.b * W.b;
    W.det = W.a2 * W.c2 - W.b * W.b;
    return W;
}

// The rotation of the splat's normalised quaternion g.q (x y z w), row-major.
__device__ __forceinline__ void rotationOf(const Gauss& g, float R[3][3]) {
    const float x = g.q[0], y = g.q[1], z = g.q[2], w = g.q[3];
    R[0][0] = 1.0f - 2.0f * (y * y + z * z); R[0][1] = 2.0f * (x * y - w * z); R[0][2] = 2.0f * (x * z + w * y);
    R[1][0] = 2.0f * (x * y + w * z); R[1][1] = 1.0f - 2.0f * (x * x + z * z); R[1][2] = 2.0f * (y * z - w * x);
    R[2][0] = 2.0f * (x * z - w * y); R[2][1] = 2.0f * (y * z + w * x); R[2][2] = 1.0f - 2.0f * (x * x + y * y);
}

// splat_project.slang:519-757 for one splat (no lens, no shutter, no catcher or
// sheet; a surfel is drawn as the thin Gaussian it projects to).
// kWide: the mixed-precision path, which takes near-degenerate footprints
// through wideCovariance (G.wide set); the plain path's arithmetic is unchanged.
template <bool kWide = false>
__device__ __forceinline__ Geometry projectGeometry(const FrameConst& F, const InstanceConst& I, const Gauss& g,
                                                    float opacity) {
    Geometry G;
    G.cull = 0;
    G.wide = false;
    const float* m = I.m;
    G.tx = ((m[0] * g.px + m[1] * g.py) + m[2] * g.pz) + m[3];
    G.ty = ((m[4] * g.px + m[5] * g.py) + m[6] * g.pz) + m[7];
    G.tz = ((m[8] * g.px + m[9] * g.py) + m[10] * g.pz) + m[11];
    if (!(G.tz > F.nearZ) || G.tz > F.farZ) {
        G.cull = kCullDepth;
        return G;
    }
    rotationOf(g, G.R);
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int col = 0; col < 3; ++col) G.M[r][col] = G.R[r][col] * g.scale[col];

    G.clampX = G.clampY = false;
    if (F.orthographic != 0) {
        G.jx0 = F.focalX; G.jx2 = 0.0f;
        G.jy1 = F.focalY; G.jy2 = 0.0f;
        G.cx = F.focalX * G.tx + F.centreX;
        G.cy = F.focalY * G.ty + F.centreY;
        G.txc = G.tx;
        G.tyc = G.ty;
    } else {
        const float invZ = 1.0f / G.tz;
        G.cx = (F.focalX * G.tx) * invZ + F.centreX;
        G.cy = (F.focalY * G.ty) * invZ + F.centreY;
        const float limLoX = ((-0.15f) * (float)F.width - F.centreX) / F.focalX;
        const float limHiX = (1.15f * (float)F.width - F.centreX) / F.focalX;
        const float limLoY = ((-0.15f) * (float)F.height - F.centreY) / F.focalY;
        const float limHiY = (1.15f * (float)F.height - F.centreY) / F.focalY;
        const float ux = G.tx * invZ, uy = G.ty * invZ;
        G.clampX = ux < limLoX || ux > limHiX;
        G.clampY = uy < limLoY || uy > limHiY;
        G.txc = clampf(ux, limLoX, limHiX) * G.tz;
        G.tyc = clampf(uy, limLoY, limHiY) * G.tz;
        G.jx0 = F.focalX * invZ;
        G.jx2 = (((-F.focalX) * G.txc) * invZ) * invZ;
        G.jy1 = F.focalY * invZ;
        G.jy2 = (((-F.focalY) * G.tyc) * invZ) * invZ;
    }
    float ax[3], ay[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        G.t3[j] = (G.jx0 * m[j] + 0.0f * m[4 + j]) + G.jx2 * m[8 + j];
        G.u3[j] = (0.0f * m[j] + G.jy1 * m[4 + j]) + G.jy2 * m[8 + j];
    }
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        ax[j] = (G.t3[0] * G.M[0][j] + G.t3[1] * G.M[1][j]) + G.t3[2] * G.M[2][j];
        ay[j] = (G.u3[0] * G.M[0][j] + G.u3[1] * G.M[1][j]) + G.u3[2] * G.M[2][j];
    }
    G.a = (ax[0] * ax[0] + ax[1] * ax[1]) + ax[2] * ax[2];
    G.b = (ax[0] * ay[0] + ax[1] * ay[1]) + ax[2] * ay[2];
    G.c = (ay[0] * ay[0] + ay[1] * ay[1]) + ay[2] * ay[2];
    G.detBefore = G.a * G.c - G.b * G.b;
    const float a2 = G.a + 0.3f, c2 = G.c + 0.3f;
    G.det = a2 * c2 - G.b * G.b;
    WideCovariance W{};
    if (kWide && G.det < 1e-6f * ((a2 + c2) * (a2 + c2))) {
        W = wideCovariance(G.t3, G.u3, G.M);
        G.wide = true;
        G.det = W.det > 1e-12 ? (float)W.det : 0.0f;
        G.detBefore = (float)W.detBefore;
    }
    if (!(G.det > 1e-12f)) {
        G.cull = kCullDegenerate;
        return G;
    }
    const float filtered = G.wide ? (float)sqrt(fmax(W.detBefore, 0.0) / W.det)
                                  : sqrtf(fmaxf(G.detBefore, 0.0f) / G.det);
    G.paid = I.antialias != 0 ? filtered : I.paidAt > 0.0f ? fminf(filtered / I.paidAt, 1.0f) : 1.0f;
    G.alpha = opacity > 1.0f ? opacity : paidOpacity(opacity, G.paid);
    if (!(G.alpha >= kFaint)) {
        G.cull = kCullFaint;
        return G;
    }
    if (G.wide) {
        G.ca = (float)(W.c2 / W.det);
        G.cb = (float)(-W.b / W.det);
        G.cc = (float)(W.a2 / W.det);
    } else {
        const float boundDet = a2 * c2 - G.b * G.b;
        G.ca = c2 / boundDet;
        G.cb = (-G.b) / boundDet;
        G.cc = a2 / boundDet;
    }
    if (kWide) {
        // the factored conic: with D the determinant, the conic (c', -b, a') / D
        // is ca (x + fr y)^2 + fs y^2 with ca = c'/D, fr = -b/c', fs = 1/c'
        // (fs = cc - cb^2/ca). D is its only input that cancels.
        G.fr = G.wide ? (float)(-W.b / W.c2) : (-G.b) / c2;
        G.fs = G.wide ? (float)(1.0 / W.c2) : 1.0f / c2;
    }
    G.cutoff = G.alpha > 1.0f ? falloffCutoff(G.alpha) : cutoffPower(G.alpha);
    return G;
}

// frame.slang:383-402: the footprint's tile rect; false when it is off screen.
__device__ __forceinline__ bool tileRectOf(const FrameConst& F, const Geometry& G, uint32_t& rx0, uint32_t& ry0,
                                          uint32_t& rx1, uint32_t& ry1) {
    const float det2 = G.ca * G.cc - G.cb * G.cb;
    const float inv = det2 > 1e-20f ? 1.0f / det2 : 0.0f;
    const float ex = sqrtf(fmaxf((G.cutoff * G.cc) * inv, 0.0f));
    const float ey = sqrtf(fmaxf((G.cutoff * G.ca) * inv, 0.0f));
    const float x1 = G.cx - ex, y1 = G.cy - ey, x2 = G.cx + ex, y2 = G.cy + ey;
    if (x2 < 0.0f || y2 < 0.0f || x1 >= (float)F.width || y1 >= (float)F.height) return false;
    rx0 = (uint32_t)fmaxf(x1, 0.0f) / kTile;
    ry0 = (uint32_t)fmaxf(y1, 0.0f) / kTile;
    rx1 = (uint32_t)fminf(x2, (float)F.width - 1.0f) / kTile;
    ry1 = (uint32_t)fminf(y2, (float)F.height - 1.0f) / kTile;
    return rx0 <= rx1 && ry0 <= ry1;
}

}   // namespace ath
