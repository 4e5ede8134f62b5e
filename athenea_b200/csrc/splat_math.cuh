// Device arithmetic of the plain splat path, shared by the projection, the
// binning and the blend. Every function states the reference shader it
// restates. The translation units that include it are built with
// --fmad=false: a*b+c stays two roundings, as written, so the CPU restatement
// (built with -ffp-contract=off) and this code agree bit for bit.
#pragma once

#include <cstdint>
#include <cuda_fp16.h>

namespace ath {

constexpr uint32_t kTile = 16;                 // splat/frame.slang:34
constexpr uint32_t kCulledKey = 0xFF000000u;   // frame.slang:42
constexpr uint32_t kCullEdit = 1, kCullDepth = 2, kCullDegenerate = 3, kCullFaint = 4, kCullOffscreen = 5,
                   kCullNoTile = 6;            // frame.slang:43-48
constexpr float kFaint = 1.0f / 255.0f;

// ---- exp / log / pow --------------------------------------------------------
// Cody & Waite (1980) reduction: x = n ln2 + r, ln 2 = hi + lo with hi holding
// 11 significant bits so n*hi is exact; e^r from its Taylor polynomial of
// degree 7 (|r| <= ln2/2: truncation < 6e-9 relative), by Horner.
// log: x = m 2^e, m in [sqrt(1/2), sqrt(2)); log m = 2 atanh(s), s = (m-1)/(m+1),
// from the odd series to s^11 (|s| <= 0.1716).
__device__ __forceinline__ float pow2i(int k) { return __uint_as_float(uint32_t(k + 127) << 23); }

__device__ __forceinline__ float exp_f(float x) {
    const float kLog2e = 1.44269502162933349609375f;
    const float kLn2Hi = 0.693115234375f;
    const float kLn2Lo = 3.1946183298714458942413330078125e-05f;
    if (x != x) return x;
    if (x > 88.72284f) return __int_as_float(0x7F800000);
    if (x < -104.0f) return 0.0f;
    const float n = rintf(x * kLog2e);
    float r = x - n * kLn2Hi;
    r = r - n * kLn2Lo;
    float p = 1.98412701138295233249664306641e-04f;   // 1/7!
    p = p * r + 1.38888892251998186111450195312e-03f;  // 1/6!
    p = p * r + 8.33333376795053482055664062500e-03f;  // 1/5!
    p = p * r + 4.16666679084300994873046875000e-02f;  // 1/4!
    p = p * r + 1.66666671633720397949218750000e-01f;  // 1/3!
    p = p * r + 0.5f;
    p = p * r + 1.0f;
    p = p * r + 1.0f;
    const int ni = (int)n;
    const int n1 = ni / 2;
    return (p * pow2i(n1)) * pow2i(ni - n1);
}

__device__ __forceinline__ float log_f(float x) {
    if (x != x || x < 0.0f) return __int_as_float(0x7FC00000);
    if (x == 0.0f) return __int_as_float(0xFF800000);
    if (x == __int_as_float(0x7F800000)) return x;
    int e = 0;
    uint32_t bits = __float_as_uint(x);
    if (bits < 0x00800000u) {
        x = x * 8388608.0f;
        bits = __float_as_uint(x);
        e = -23;
    }
    e += (int)((bits >> 23) & 0xFFu) - 127;
    float m = __uint_as_float((bits & 0x007FFFFFu) | 0x3F800000u);
    if (m > 1.41421353816986083984375f) {
        m = m * 0.5f;
        e += 1;
    }
    const float s = (m - 1.0f) / (m + 1.0f);
    const float z = s * s;
    float p = 9.09090936183929443359375e-02f;          // 1/11
    p = p * z + 1.11111111938953399658203125e-01f;      // 1/9
    p = p * z + 1.42857149243354797363281250e-01f;      // 1/7
    p = p * z + 2.00000002980232238769531250e-01f;      // 1/5
    p = p * z + 3.33333343267440795898437500e-01f;      // 1/3
    p = p * z + 1.0f;
    const float lm = (2.0f * s) * p;
    const float fe = (float)e;
    return fe * 0.693115234375f + (lm + fe * 3.1946183298714458942413330078125e-05f);
}

__device__ __forceinline__ float pow_f(float x, float y) {
    if (x == 0.0f) return y > 0.0f ? 0.0f : __int_as_float(0x7F800000);
    return exp_f(y * log_f(x));
}

// ---- packing (common/packing.slang) ---------------------------------------
__device__ __forceinline__ float lowHalf(uint32_t w) { return __half2float(__ushort_as_half((unsigned short)(w & 0xFFFFu))); }
__device__ __forceinline__ float highHalf(uint32_t w) { return __half2float(__ushort_as_half((unsigned short)(w >> 16))); }

// packing.slang:59-76
__device__ __forceinline__ void decodeQuaternion(uint32_t word, float q[4]) {
    const float kSqrtHalf = 0.70710678f;
    const uint32_t largest = word & 3u;
    const float s0 = (((float)((word >> 22) & 1023u) / 1023.0f) * 2.0f - 1.0f) * kSqrtHalf;
    const float s1 = (((float)((word >> 12) & 1023u) / 1023.0f) * 2.0f - 1.0f) * kSqrtHalf;
    const float s2 = (((float)((word >> 2) & 1023u) / 1023.0f) * 2.0f - 1.0f) * kSqrtHalf;
    const float rest = sqrtf(fmaxf(0.0f, 1.0f - ((s0 * s0 + s1 * s1) + s2 * s2)));
    // the dropped component goes to `largest`, the three kept fill the rest in order
    q[0] = largest == 0 ? rest : s0;
    q[1] = largest == 1 ? rest : (largest == 0 ? s0 : s1);
    q[2] = largest == 2 ? rest : (largest <= 1 ? s1 : s2);
    q[3] = largest == 3 ? rest : s2;
}

// ---- frame.slang helpers ---------------------------------------------------
// frame.slang:316-319
__device__ __forceinline__ float paidOpacity(float alpha, float paid) {
    const float spread = paid * alpha;
    return spread >= kFaint ? spread + (1.0f - paid) * kFaint : spread;
}

// frame.slang:325-327
__device__ __forceinline__ float cutoffPower(float alpha) {
    return fminf(2.0f * log_f(fmaxf(255.0f * alpha, 1.0001f)), 9.0f);
}

// frame.slang:337-348: an opacity over 1 is Spark's harder kernel.
__device__ __forceinline__ float falloffCount(float d) { return exp_f((d * d - 1.0f) * 0.36787944f); }
__device__ __forceinline__ float falloffAlpha(float d, float g) {
    return d > 1.0f ? 1.0f - pow_f(fmaxf(1.0f - g, 0.0f), falloffCount(d)) : d * g;
}
__device__ __forceinline__ float falloffCutoff(float d) {
    const float r = 3.0f + 0.7f * (fminf(d, 5.0f) - 1.0f);
    return fminf(2.0f * log_f(255.0f * falloffCount(d)), r * r);
}

__device__ __forceinline__ float clampf(float v, float lo, float hi) { return fminf(fmaxf(v, lo), hi); }

// frame.slang:354-371: the least of a x^2 + 2 b x y + c y^2 over a box.
__device__ __forceinline__ float minPowerOverBox(float a, float b, float c, float lox, float loy, float hix,
                                                  float hiy) {
    if (lox <= 0.0f && hix >= 0.0f && loy <= 0.0f && hiy >= 0.0f) return 0.0f;
    float best = 3.4e38f;
#pragma unroll
    for (int e = 0; e < 2; ++e) {
        const float x = e == 0 ? lox : hix;
        const float y = c > 1e-12f ? clampf(((-b) * x) / c, loy, hiy) : loy;
        best = fminf(best, ((a * x) * x + ((2.0f * b) * x) * y) + (c * y) * y);
    }
#pragma unroll
    for (int e = 0; e < 2; ++e) {
        const float y = e == 0 ? loy : hiy;
        const float x = a > 1e-12f ? clampf(((-b) * y) / a, lox, hix) : lox;
        best = fminf(best, ((a * x) * x + ((2.0f * b) * x) * y) + (c * y) * y);
    }
    return best;
}

// frame.slang:374-379: does tile (tx, ty) hold a pixel centre inside the footprint?
__device__ __forceinline__ bool tileTouched(uint32_t width, uint32_t height, float cx, float cy, float ca, float cb,
                                            float cc, float cutoff, uint32_t tx, uint32_t ty) {
    const float fx = (float)(tx * kTile) + 0.5f;
    const float fy = (float)(ty * kTile) + 0.5f;
    const float lx = (float)(min((tx + 1) * kTile, width) - 1) + 0.5f;
    const float ly = (float)(min((ty + 1) * kTile, height) - 1) + 0.5f;
    return minPowerOverBox(ca, cb, cc, fx - cx, fy - cy, lx - cx, ly - cy) <= cutoff;
}

// common/color.slang:7-10
__device__ __forceinline__ float srgbToLinear(float c) {
    c = fmaxf(c, 0.0f);
    return c <= 0.04045f ? c / 12.92f : pow_f((c + 0.055f) / 1.055f, 2.4f);
}

// common/color.slang:43-47: a hash of v to [0, 1] (PCG-style), the dither of
// the colour gradient's rounding (splat_blend.slang:393-394).
__host__ __device__ __forceinline__ float hash01(uint32_t v) {
    const uint32_t state = v * 747796405u + 2891336453u;
    const uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
    return (float)((word >> 22u) ^ word) / 4294967295.0f;
}

// common/sh.slang:94-96
__device__ __forceinline__ uint32_t degreeOf(uint32_t restPerColour) {
    return restPerColour >= 15 ? 3 : restPerColour >= 8 ? 2 : restPerColour >= 3 ? 1 : 0;
}

}   // namespace ath
