// ORACLE -- TEST INFRASTRUCTURE ONLY (see oracle.h). A C++ restatement of the
// reference's plain splat raster path, float32 without contraction. Each
// function names the reference file:line it follows.
#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <type_traits>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr uint32_t kTile = 16;                    // splat/frame.slang:34

// The frame's tile size: the reference's 16 (frame.slang:34), or another the
// batched path bins at (8 or 32), set by orc_frame_set_tile.
inline uint32_t tileOf(const orc_frame& f) { return f.tile ? f.tile : kTile; }
constexpr uint32_t kCulledKey = 0xFF000000u;      // frame.slang:42-49
constexpr uint32_t kCullEdit = 1, kCullDepth = 2, kCullDegenerate = 3, kCullFaint = 4, kCullOffscreen = 5,
                   kCullNoTile = 6;
constexpr float kSqrtHalf = 0.70710678f;          // common/packing.slang:30
constexpr float kSH0 = 0.28209479177387814f;      // common/packing.slang:445

inline uint32_t bitsOf(float v) {
    uint32_t u;
    std::memcpy(&u, &v, 4);
    return u;
}
inline float floatOf(uint32_t u) {
    float v;
    std::memcpy(&v, &u, 4);
    return v;
}

// ---------------------------------------------------------------------------
// exp / log / pow. Published methods, restated: Cody and Waite (1980) argument
// reduction x = n ln2 + r with ln2 split into a short high part (11 significant
// bits, so n * hi is exact) and a low part; e^r by its Taylor series to r^7
// (|r| <= ln2/2, truncation below 6e-9 relative). log m for m in [sqrt(1/2),
// sqrt(2)) by 2 atanh((m-1)/(m+1)), its odd series to s^11.
// ---------------------------------------------------------------------------
const float kLog2e = (float)1.4426950408889634;
const float kLn2Hi = 0.693115234375f;
const float kLn2Lo = (float)(0.69314718055994530942 - 0.693115234375);
const float kInvF2 = 0.5f, kInvF3 = (float)(1.0 / 6.0), kInvF4 = (float)(1.0 / 24.0),
            kInvF5 = (float)(1.0 / 120.0), kInvF6 = (float)(1.0 / 720.0), kInvF7 = (float)(1.0 / 5040.0);
const float kInv3 = (float)(1.0 / 3.0), kInv5 = (float)(1.0 / 5.0), kInv7 = (float)(1.0 / 7.0),
            kInv9 = (float)(1.0 / 9.0), kInv11 = (float)(1.0 / 11.0);
const float kSqrt2 = (float)1.4142135623730951;

inline float pow2i(int k) {   // 2^k for -126 <= k <= 127
    return floatOf(uint32_t(k + 127) << 23);
}

float expf_(float x) {
    if (x != x) return x;
    if (x > 88.72284f) return INFINITY;
    if (x < -104.0f) return 0.0f;
    const float n = std::rint(x * kLog2e);
    float r = x - n * kLn2Hi;
    r = r - n * kLn2Lo;
    float p = kInvF7;
    p = p * r + kInvF6;
    p = p * r + kInvF5;
    p = p * r + kInvF4;
    p = p * r + kInvF3;
    p = p * r + kInvF2;
    p = p * r + 1.0f;
    p = p * r + 1.0f;
    const int ni = (int)n;
    const int n1 = ni / 2;
    const int n2 = ni - n1;
    return (p * pow2i(n1)) * pow2i(n2);
}

float logf_(float x) {
    if (x != x || x < 0.0f) return NAN;
    if (x == 0.0f) return -INFINITY;
    if (std::isinf(x)) return x;
    int e = 0;
    uint32_t bits = bitsOf(x);
    if (bits < 0x00800000u) {   // subnormal: exact scaling by 2^23
        x = x * 8388608.0f;
        bits = bitsOf(x);
        e = -23;
    }
    e += (int)((bits >> 23) & 0xFFu) - 127;
    float m = floatOf((bits & 0x007FFFFFu) | 0x3F800000u);
    if (m > kSqrt2) {
        m = m * 0.5f;
        e += 1;
    }
    const float s = (m - 1.0f) / (m + 1.0f);
    const float z = s * s;
    float p = kInv11;
    p = p * z + kInv9;
    p = p * z + kInv7;
    p = p * z + kInv5;
    p = p * z + kInv3;
    p = p * z + 1.0f;
    const float lm = (2.0f * s) * p;
    const float fe = (float)e;
    return fe * kLn2Hi + (lm + fe * kLn2Lo);
}

float powf_(float x, float y) {
    if (x == 0.0f) return y > 0.0f ? 0.0f : INFINITY;
    return expf_(y * logf_(x));
}

// ---------------------------------------------------------------------------
// f16 (common/packing.slang:319-328: f32tof16 rounds to nearest even).
// ---------------------------------------------------------------------------
uint16_t toHalf(float v) {
    const uint32_t x = bitsOf(v);
    const uint32_t sign = (x >> 16) & 0x8000u;
    const uint32_t a = x & 0x7FFFFFFFu;
    if (a >= 0x7F800000u) return (uint16_t)(sign | (a > 0x7F800000u ? 0x7E00u : 0x7C00u));
    if (a >= 0x477FF000u) return (uint16_t)(sign | 0x7C00u);   // rounds past 65504
    if (a < 0x38800000u) {                                     // below 2^-14: subnormal or zero
        if (a <= 0x33000000u) return (uint16_t)sign;           // at most 2^-25: ties to even zero
        const uint32_t m = (a & 0x7FFFFFu) | 0x800000u;
        const int e = (int)(a >> 23);
        const int s = 126 - e;
        uint32_t h = m >> s;
        const uint32_t rem = m & ((1u << s) - 1u);
        const uint32_t half = 1u << (s - 1);
        if (rem > half || (rem == half && (h & 1u))) h += 1;
        return (uint16_t)(sign | h);
    }
    const uint32_t e = (a >> 23) - 112u;
    const uint32_t mant = a & 0x7FFFFFu;
    uint32_t h = (e << 10) | (mant >> 13);
    const uint32_t rem = mant & 0x1FFFu;
    if (rem > 0x1000u || (rem == 0x1000u && (h & 1u))) h += 1;
    return (uint16_t)(sign | h);
}

float fromHalf(uint16_t h) {
    const uint32_t sign = (uint32_t)(h & 0x8000u) << 16;
    const uint32_t e = (h >> 10) & 0x1Fu;
    const uint32_t m = h & 0x3FFu;
    if (e == 0) {
        if (m == 0) return floatOf(sign);
        // subnormal: m * 2^-24, exact in float
        const float v = (float)m * 5.9604644775390625e-08f;
        return sign ? -v : v;
    }
    if (e == 31) return floatOf(sign | 0x7F800000u | (m << 13));
    return floatOf(sign | ((e + 112u) << 23) | (m << 13));
}

inline float lowHalf(uint32_t w) { return fromHalf((uint16_t)(w & 0xFFFFu)); }
inline float highHalf(uint32_t w) { return fromHalf((uint16_t)(w >> 16)); }
inline uint32_t packHalves(float a, float b) { return (uint32_t)toHalf(a) | ((uint32_t)toHalf(b) << 16); }
// Slang's min/max/clamp are IEEE minNum/maxNum (a NaN operand yields the other).
inline float halfSafe(float v) { return std::fmin(std::fmax(v, -65000.0f), 65000.0f); }   // packing.slang:328

inline float clampf(float v, float lo, float hi) { return std::fmin(std::fmax(v, lo), hi); }

// common/packing.slang:59-76
void decodeQuaternion(uint32_t word, float q[4]) {
    const uint32_t largest = word & 3u;
    float s0 = (float)((word >> 22) & 1023u), s1 = (float)((word >> 12) & 1023u), s2 = (float)((word >> 2) & 1023u);
    s0 = ((s0 / 1023.0f) * 2.0f - 1.0f) * kSqrtHalf;
    s1 = ((s1 / 1023.0f) * 2.0f - 1.0f) * kSqrtHalf;
    s2 = ((s2 / 1023.0f) * 2.0f - 1.0f) * kSqrtHalf;
    const float rest = std::sqrt(std::max(0.0f, 1.0f - ((s0 * s0 + s1 * s1) + s2 * s2)));
    const float small[3] = {s0, s1, s2};
    uint32_t next = 0;
    for (uint32_t k = 0; k < 4; ++k) {
        if (k == largest) {
            q[k] = rest;
        } else {
            q[k] = small[next++];
        }
    }
}

// common/packing.slang:33-57. `round` as Slang's CUDA target emits it
// (roundf: halves away from zero).
uint32_t encodeQuaternion(const float in[4]) {
    const float len = std::sqrt(((in[0] * in[0] + in[1] * in[1]) + in[2] * in[2]) + in[3] * in[3]);
    float q[4] = {in[0] / len, in[1] / len, in[2] / len, in[3] / len};
    uint32_t largest = 0;
    float best = std::fabs(q[0]);
    for (uint32_t k = 1; k < 4; ++k) {
        if (std::fabs(q[k]) > best) {
            best = std::fabs(q[k]);
            largest = k;
        }
    }
    if (q[largest] < 0.0f) {
        for (float& v : q) v = -v;
    }
    uint32_t word = largest;
    uint32_t shift = 22;
    for (uint32_t k = 0; k < 4; ++k) {
        if (k == largest) continue;
        const float unit = clampf((q[k] / kSqrtHalf) * 0.5f + 0.5f, 0.0f, 1.0f);
        word |= (uint32_t)std::round(unit * 1023.0f) << shift;
        shift -= 10;
    }
    return word;
}

// common/color.slang:7-10,39-41
inline float srgbToLinear(float c) {
    c = std::max(c, 0.0f);
    return c <= 0.04045f ? c / 12.92f : powf_((c + 0.055f) / 1.055f, 2.4f);
}

struct Fate {
    bool removed, graded;
    float opacity;
};

// common/edit.slang:46-78
Fate editFate(const orc_edit& e, const float p[3], float opacity, const float s[3]) {
    Fate fate{false, false, opacity};
    if (e.active == 0) return fate;
    if (e.minOpacity > 0.0f && opacity < e.minOpacity) {
        fate.removed = true;
        return fate;
    }
    if (e.maxScale > 0.0f &&
        std::max(std::max(std::fabs(s[0]), std::fabs(s[1])), std::fabs(s[2])) > e.maxScale) {
        fate.removed = true;
        return fate;
    }
    const float rx = p[0] - e.centre[0], ry = p[1] - e.centre[1], rz = p[2] - e.centre[2];
    bool inside = e.shape == 1 ? ((rx * rx + ry * ry) + rz * rz) <= e.size[0] * e.size[0]
                               : (std::fabs(rx) <= e.size[0] && std::fabs(ry) <= e.size[1] &&
                                  std::fabs(rz) <= e.size[2]);
    if (e.invert != 0) inside = !inside;
    if ((e.mode == 0 && !inside) || (e.mode == 1 && inside)) {
        fate.removed = true;
        return fate;
    }
    if (inside) {
        fate.graded = true;
        fate.opacity = opacity * e.opacity;
        fate.removed = !(fate.opacity >= 1.0f / 255.0f);
    }
    return fate;
}

// common/edit.slang:86-90
void editGrade(const orc_edit& e, float c[3]) {
    float g[3];
    for (int k = 0; k < 3; ++k) g[k] = (c[k] * e.tint[k]) * e.brightness;
    const float luma = (g[0] * 0.2126f + g[1] * 0.7152f) + g[2] * 0.0722f;
    for (int k = 0; k < 3; ++k) {
        // lerp(a, b, t) = a + (b - a) * t
        c[k] = std::max(luma + (g[k] - luma) * e.saturation, 0.0f);
    }
}

// splat/frame.slang:316-319
inline float paidOpacity(float alpha, float paid) {
    const float spread = paid * alpha;
    return spread >= 1.0f / 255.0f ? spread + (1.0f - paid) * (1.0f / 255.0f) : spread;
}

// frame.slang:325-327
inline float cutoffPower(float alpha) { return std::min(2.0f * logf_(std::max(255.0f * alpha, 1.0001f)), 9.0f); }

// frame.slang:335-348 (an opacity over 1: Spark's harder kernel)
inline float falloffCount(float d) { return expf_((d * d - 1.0f) * 0.36787944f); }
inline float falloffAlpha(float d, float g) {
    return d > 1.0f ? 1.0f - powf_(std::max(1.0f - g, 0.0f), falloffCount(d)) : d * g;
}
inline float falloffCutoff(float d) {
    const float r = 3.0f + 0.7f * (std::min(d, 5.0f) - 1.0f);
    return std::min(2.0f * logf_(255.0f * falloffCount(d)), r * r);
}

// frame.slang:354-371
float minPowerOverBox(float a, float b, float c, float lox, float loy, float hix, float hiy) {
    if (lox <= 0.0f && hix >= 0.0f && loy <= 0.0f && hiy >= 0.0f) return 0.0f;
    float best = 3.4e38f;
    for (int e = 0; e < 2; ++e) {
        const float x = e == 0 ? lox : hix;
        const float y = c > 1e-12f ? clampf(((-b) * x) / c, loy, hiy) : loy;
        best = std::min(best, ((a * x) * x + ((2.0f * b) * x) * y) + (c * y) * y);
    }
    for (int e = 0; e < 2; ++e) {
        const float y = e == 0 ? loy : hiy;
        const float x = a > 1e-12f ? clampf(((-b) * y) / a, lox, hix) : lox;
        best = std::min(best, ((a * x) * x + ((2.0f * b) * x) * y) + (c * y) * y);
    }
    return best;
}

// frame.slang:374-379
inline bool tileTouched(const orc_frame& f, float cx, float cy, float ca, float cb, float cc, float cutoff,
                        uint32_t tx, uint32_t ty) {
    const float fx = (float)(tx * tileOf(f)) + 0.5f;
    const float fy = (float)(ty * tileOf(f)) + 0.5f;
    const float lx = (float)(std::min((tx + 1) * tileOf(f), f.width) - 1) + 0.5f;
    const float ly = (float)(std::min((ty + 1) * tileOf(f), f.height) - 1) + 0.5f;
    return minPowerOverBox(ca, cb, cc, fx - cx, fy - cy, lx - cx, ly - cy) <= cutoff;
}

inline uint32_t degreeOf(uint32_t restPerColour) {   // common/sh.slang:94-96
    return restPerColour >= 15 ? 3 : restPerColour >= 8 ? 2 : restPerColour >= 3 ? 1 : 0;
}

// common/sh.slang:15-51, one colour channel `ch` at a time.
inline float halfAt(const uint32_t* sh, uint32_t row, uint32_t index) {
    const uint32_t word = sh[row + index / 2];
    return (index & 1u) == 0u ? lowHalf(word) : highHalf(word);
}

template <typename Coef>
void evaluateRest(Coef coef, uint32_t degree, float x, float y, float z, float out[3]) {
    const float kC1 = 0.4886025119029199f;
    const float kC2[5] = {1.0925484305920792f, -1.0925484305920792f, 0.31539156525252005f, -1.0925484305920792f,
                          0.5462742152960396f};
    const float kC3[7] = {-0.5900435899266435f, 2.890611442640554f, -0.4570457994644658f, 0.3731763325901154f,
                          -0.4570457994644658f, 1.445305721320277f, -0.5900435899266435f};
    for (int ch = 0; ch < 3; ++ch) out[ch] = 0.0f;
    if (degree == 0) return;
    for (int ch = 0; ch < 3; ++ch) {
        auto B = [&](uint32_t k) { return coef(k * 3 + (uint32_t)ch); };
        float r = (((-kC1) * y) * B(0) + (kC1 * z) * B(1)) - (kC1 * x) * B(2);
        if (degree >= 2) {
            const float xx = x * x, yy = y * y, zz = z * z;
            const float xy = x * y, yz = y * z, xz = x * z;
            const float t = (((((kC2[0] * xy) * B(3) + (kC2[1] * yz) * B(4)) +
                              (kC2[2] * ((2.0f * zz - xx) - yy)) * B(5)) +
                             (kC2[3] * xz) * B(6)) +
                            (kC2[4] * (xx - yy)) * B(7));
            r = r + t;
            if (degree >= 3) {
                const float u = ((((((((kC3[0] * y) * (3.0f * xx - yy)) * B(8) + ((kC3[1] * xy) * z) * B(9)) +
                                     ((kC3[2] * y) * ((4.0f * zz - xx) - yy)) * B(10)) +
                                    ((kC3[3] * z) * ((2.0f * zz - 3.0f * xx) - 3.0f * yy)) * B(11)) +
                                   ((kC3[4] * x) * ((4.0f * zz - xx) - yy)) * B(12)) +
                                  ((kC3[5] * z) * (xx - yy)) * B(13)) +
                                 ((kC3[6] * x) * (xx - 3.0f * yy)) * B(14));
                r = r + u;
            }
        }
        out[ch] = r;
    }
}

void cullSlot(uint32_t slot, uint32_t reason, float* records, uint32_t* rects, uint32_t* touched,
              uint32_t* depthKeys, uint32_t* visible) {
    // splat_project.slang:138-148
    touched[slot] = 0;
    visible[slot] = 0;
    depthKeys[slot] = kCulledKey | reason;
    rects[slot * 4 + 0] = 1;
    rects[slot * 4 + 1] = 1;
    rects[slot * 4 + 2] = 0;
    rects[slot * 4 + 3] = 0;
    for (int k = 0; k < 12; ++k) records[slot * 12 + k] = 0.0f;
}

// One Gaussian as the projection reads it (position, opacity, linear scales,
// unit quaternion x y z w, the constant term's colour).
struct G32 {
    float px, py, pz, opacity;
    float scale[3];
    float q[4];
    float base[3];
};

G32 loadPacked(const float* positions, const uint32_t* shape, uint32_t i) {
    G32 g;
    g.px = positions[i * 4 + 0];
    g.py = positions[i * 4 + 1];
    g.pz = positions[i * 4 + 2];
    g.opacity = positions[i * 4 + 3];
    const uint32_t row = i * 4;
    g.scale[0] = expf_(lowHalf(shape[row + 1]));
    g.scale[1] = expf_(highHalf(shape[row + 1]));
    g.scale[2] = expf_(lowHalf(shape[row + 2]));
    decodeQuaternion(shape[row], g.q);
    g.base[0] = highHalf(shape[row + 2]);
    g.base[1] = lowHalf(shape[row + 3]);
    g.base[2] = highHalf(shape[row + 3]);
    return g;
}

// The FP32 training layout: means float4 (xyz, opacity logit), scales float4
// (log scales), quats float4 (w x y z, any length), sh: DC rgb then rest rgb
// per basis. Decoded as the upload would: sigmoid, exp, normalise, 0.5 + SH0 dc.
G32 loadParams(const float* means, const float* scales, const float* quats, const float* sh, uint32_t stride,
               uint32_t i) {
    G32 g;
    g.px = means[i * 4 + 0];
    g.py = means[i * 4 + 1];
    g.pz = means[i * 4 + 2];
    g.opacity = 1.0f / (1.0f + expf_(-means[i * 4 + 3]));
    for (int k = 0; k < 3; ++k) g.scale[k] = expf_(scales[i * 4 + k]);
    const float* q = quats + (size_t)i * 4;
    const float len = std::sqrt(((q[0] * q[0] + q[1] * q[1]) + q[2] * q[2]) + q[3] * q[3]);
    g.q[0] = q[1] / len;
    g.q[1] = q[2] / len;
    g.q[2] = q[3] / len;
    g.q[3] = q[0] / len;
    const float* c = sh + (size_t)i * stride;
    for (int k = 0; k < 3; ++k) g.base[k] = 0.5f + kSH0 * c[k];
    return g;
}

template <typename RestFn>
void projectCore(const orc_frame& f, const G32& g, RestFn rest3, uint32_t slot, float* records, uint32_t* rects,
                 uint32_t* touchedOut, uint32_t* depthKeys, uint32_t* visible) {
    // splat_project.slang:497-523
    const float px = g.px, py = g.py, pz = g.pz;
    float opacity = g.opacity;
    const float* scale = g.scale;
    const float pos[3] = {px, py, pz};
    const Fate fate = editFate(f.edit, pos, opacity, scale);
    if (fate.removed) {
        cullSlot(slot, kCullEdit, records, rects, touchedOut, depthKeys, visible);
        return;
    }
    opacity = fate.opacity;
    const float* m = f.m;
    const float tx = ((m[0] * px + m[1] * py) + m[2] * pz) + m[3];
    const float ty = ((m[4] * px + m[5] * py) + m[6] * pz) + m[7];
    const float tz = ((m[8] * px + m[9] * py) + m[10] * pz) + m[11];
    if (!(tz > f.nearZ) || tz > f.farZ) {
        cullSlot(slot, kCullDepth, records, rects, touchedOut, depthKeys, visible);
        return;
    }
    // :526-532
    const float x = g.q[0], y = g.q[1], z = g.q[2], w = g.q[3];
    const float r[3][3] = {{1.0f - 2.0f * (y * y + z * z), 2.0f * (x * y - w * z), 2.0f * (x * z + w * y)},
                           {2.0f * (x * y + w * z), 1.0f - 2.0f * (x * x + z * z), 2.0f * (y * z - w * x)},
                           {2.0f * (x * z - w * y), 2.0f * (y * z + w * x), 1.0f - 2.0f * (x * x + y * y)}};
    float M[3][3];
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) M[a][b] = r[a][b] * scale[b];
    // :535-557
    float jx[3], jy[3], cx, cy;
    if (f.orthographic != 0) {
        jx[0] = f.focalX; jx[1] = 0.0f; jx[2] = 0.0f;
        jy[0] = 0.0f; jy[1] = f.focalY; jy[2] = 0.0f;
        cx = f.focalX * tx + f.centreX;
        cy = f.focalY * ty + f.centreY;
    } else {
        const float invZ = 1.0f / tz;
        cx = (f.focalX * tx) * invZ + f.centreX;
        cy = (f.focalY * ty) * invZ + f.centreY;
        const float limLoX = ((-0.15f) * (float)f.width - f.centreX) / f.focalX;
        const float limHiX = (1.15f * (float)f.width - f.centreX) / f.focalX;
        const float limLoY = ((-0.15f) * (float)f.height - f.centreY) / f.focalY;
        const float limHiY = (1.15f * (float)f.height - f.centreY) / f.focalY;
        const float txc = clampf(tx * invZ, limLoX, limHiX) * tz;
        const float tyc = clampf(ty * invZ, limLoY, limHiY) * tz;
        jx[0] = f.focalX * invZ; jx[1] = 0.0f; jx[2] = (((-f.focalX) * txc) * invZ) * invZ;
        jy[0] = 0.0f; jy[1] = f.focalY * invZ; jy[2] = (((-f.focalY) * tyc) * invZ) * invZ;
    }
    // :558-565: row vectors times W, then times M
    const float W[3][3] = {{m[0], m[1], m[2]}, {m[4], m[5], m[6]}, {m[8], m[9], m[10]}};
    float tx3[3], ty3[3], ax[3], ay[3];
    for (int j = 0; j < 3; ++j) {
        tx3[j] = (jx[0] * W[0][j] + jx[1] * W[1][j]) + jx[2] * W[2][j];
        ty3[j] = (jy[0] * W[0][j] + jy[1] * W[1][j]) + jy[2] * W[2][j];
    }
    for (int j = 0; j < 3; ++j) {
        ax[j] = (tx3[0] * M[0][j] + tx3[1] * M[1][j]) + tx3[2] * M[2][j];
        ay[j] = (ty3[0] * M[0][j] + ty3[1] * M[1][j]) + ty3[2] * M[2][j];
    }
    float a = (ax[0] * ax[0] + ax[1] * ax[1]) + ax[2] * ax[2];
    float b = (ax[0] * ay[0] + ax[1] * ay[1]) + ax[2] * ay[2];
    float c = (ay[0] * ay[0] + ay[1] * ay[1]) + ay[2] * ay[2];
    const float detBefore = a * c - b * b;
    const float spreadPaid = 1.0f;   // no lens, no shutter on the plain path
    // :651-657
    a = a + 0.3f;
    c = c + 0.3f;
    const float det = a * c - b * b;
    if (!(det > 1e-12f)) {
        cullSlot(slot, kCullDegenerate, records, rects, touchedOut, depthKeys, visible);
        return;
    }
    const float filtered = std::sqrt(std::max(detBefore, 0.0f) / det);
    const float paid = f.antialias != 0 ? filtered : f.paidAt > 0.0f ? std::min(filtered / f.paidAt, 1.0f) : spreadPaid;
    // :744-751 (no catcher, no sheet; a surfel is drawn as the thin gaussian it projects to)
    const float alpha = opacity > 1.0f ? opacity : paidOpacity(opacity, paid);
    if (!(alpha >= 1.0f / 255.0f)) {
        cullSlot(slot, kCullFaint, records, rects, touchedOut, depthKeys, visible);
        return;
    }
    // :752-763
    const float boundDet = a * c - b * b;
    const float ca = c / boundDet, cb = (-b) / boundDet, cc = a / boundDet;
    const float cutoff = alpha > 1.0f ? falloffCutoff(alpha) : cutoffPower(alpha);
    // frame.slang:383-387
    const float det2 = ca * cc - cb * cb;
    const float inv = det2 > 1e-20f ? 1.0f / det2 : 0.0f;
    const float ex = std::sqrt(std::max((cutoff * cc) * inv, 0.0f));
    const float ey = std::sqrt(std::max((cutoff * ca) * inv, 0.0f));
    // frame.slang:390-402
    const float x1 = cx - ex, y1 = cy - ey, x2 = cx + ex, y2 = cy + ey;
    uint32_t rx0, ry0, rx1, ry1;
    if (x2 < 0.0f || y2 < 0.0f || x1 >= (float)f.width || y1 >= (float)f.height) {
        rx0 = 1; ry0 = 1; rx1 = 0; ry1 = 0;
    } else {
        rx0 = (uint32_t)std::max(x1, 0.0f) / tileOf(f);
        ry0 = (uint32_t)std::max(y1, 0.0f) / tileOf(f);
        rx1 = (uint32_t)std::min(x2, (float)f.width - 1.0f) / tileOf(f);
        ry1 = (uint32_t)std::min(y2, (float)f.height - 1.0f) / tileOf(f);
    }
    if (rx0 > rx1 || ry0 > ry1) {
        cullSlot(slot, kCullOffscreen, records, rects, touchedOut, depthKeys, visible);
        return;
    }
    // :765-776
    uint32_t touched = 0;
    for (uint32_t ty2 = ry0; ty2 <= ry1; ++ty2)
        for (uint32_t tx2 = rx0; tx2 <= rx1; ++tx2)
            if (tileTouched(f, cx, cy, ca, cb, cc, cutoff, tx2, ty2)) touched += 1;
    if (touched == 0) {
        cullSlot(slot, kCullNoTile, records, rects, touchedOut, depthKeys, visible);
        return;
    }
    // :781-785
    const uint32_t degree = std::min(degreeOf(f.restPerColour), f.shLimit);
    const float dx = px - f.eye[0], dy = py - f.eye[1], dz = pz - f.eye[2];
    const float len = std::sqrt((dx * dx + dy * dy) + dz * dz);
    float restv[3];
    rest3(degree, dx / len, dy / len, dz / len, restv);
    float colour[3];
    for (int k = 0; k < 3; ++k) {
        const float v = g.base[k] + restv[k];
        colour[k] = f.linearCloud != 0 ? std::max(v, 0.0f) : srgbToLinear(v);
    }
    if (fate.graded) editGrade(f.edit, colour);
    // :1080-1129
    float* rec = records + slot * 12;
    rec[0] = cx; rec[1] = cy; rec[2] = tz; rec[3] = cutoff;
    rec[4] = ca; rec[5] = cb; rec[6] = cc; rec[7] = alpha;
    rec[8] = colour[0]; rec[9] = colour[1]; rec[10] = colour[2]; rec[11] = 0.0f;
    rects[slot * 4 + 0] = rx0;
    rects[slot * 4 + 1] = ry0;
    rects[slot * 4 + 2] = rx1;
    rects[slot * 4 + 3] = ry1;
    touchedOut[slot] = touched;
    visible[slot] = 1;
    depthKeys[slot] = bitsOf(tz) >> 7;
}

void projectOne(const orc_frame& f, uint32_t i, uint32_t slot, const float* positions, const uint32_t* shape,
                const uint32_t* sh, float* records, uint32_t* rects, uint32_t* touchedOut, uint32_t* depthKeys,
                uint32_t* visible) {
    const G32 g = loadPacked(positions, shape, i);
    projectCore(f, g,
                [&](uint32_t degree, float x, float y, float z, float out[3]) {
                    evaluateRest([&](uint32_t index) { return halfAt(sh, i * f.shWords, index); }, degree, x, y, z,
                                 out);
                },
                slot, records, rects, touchedOut, depthKeys, visible);
}

// One pixel's walk: splat_blend.slang:236-578 with composite, matte, trace off.
struct Walk {
    float rgb[3] = {0, 0, 0};
    float t = 1.0f;
    float depthSum = 0.0f;
    float depthAt = -1.0f;
    uint32_t last = 0;        // one past the last record blended (relative to the range start)
    uint32_t evaluated = 0;
};

// underZ > 0: an opaque layer under the splats at that depth ends the walk at
// the first record at or behind it (splat_blend.slang:249-251,329-333). `visit`
// sees each blended splat before the walk adds it: (slot, weight), or (slot,
// weight, the walk so far, alpha, the record) where it takes those.
template <typename Visit>
Walk walkPixel(const orc_frame& f, uint32_t start, uint32_t end, const uint32_t* pairSplats, const float* records,
               float pxc, float pyc, Visit visit, float underZ = 0.0f) {
    Walk wk;
    for (uint32_t j = start; j < end; ++j) {
        const uint32_t s = pairSplats[j];
        const float* rec = records + s * 12;
        if (underZ > 0.0f && rec[2] >= underZ) break;
        wk.evaluated += 1;
        const float dx = pxc - rec[0];
        const float dy = pyc - rec[1];
        const float power = ((rec[4] * dx) * dx + ((2.0f * rec[5]) * dx) * dy) + (rec[6] * dy) * dy;
        if (power > rec[3]) continue;
        const float alpha = std::min(0.99f, falloffAlpha(std::fabs(rec[7]), expf_((-0.5f) * power)));
        if (alpha < 1.0f / 255.0f) continue;
        const float weight = wk.t * alpha;
        if constexpr (std::is_invocable_v<Visit, uint32_t, float, const Walk&, float, const float*>)
            visit(s, weight, static_cast<const Walk&>(wk), alpha, rec);
        else
            visit(s, weight);
        for (int k = 0; k < 3; ++k) wk.rgb[k] = wk.rgb[k] + weight * rec[8 + k];
        wk.depthSum = wk.depthSum + weight * rec[2];
        wk.t = wk.t * (1.0f - alpha);
        wk.last = j - start + 1;
        if (wk.depthAt < 0.0f && 1.0f - wk.t >= f.depthThreshold) wk.depthAt = rec[2];
        if (wk.t < 1e-4f) break;
    }
    return wk;
}

inline int threadsOr(int threads) {
#ifdef _OPENMP
    return threads > 0 ? threads : omp_get_max_threads();
#else
    (void)threads;
    return 1;
#endif
}

// common/color.slang:43-47
inline float hash01(uint32_t v) {
    const uint32_t state = v * 747796405u + 2891336453u;
    const uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
    return (float)((word >> 22u) ^ word) / 4294967295.0f;
}

}   // namespace

extern "C" {

float orc_exp(float x) { return expf_(x); }
float orc_log(float x) { return logf_(x); }
float orc_pow(float x, float y) { return powf_(x, y); }
uint16_t orc_f32_to_f16(float v) { return toHalf(v); }
float orc_f16_to_f32(uint16_t h) { return fromHalf(h); }
uint32_t orc_encode_quaternion(const float q[4]) { return encodeQuaternion(q); }
void orc_decode_quaternion(uint32_t word, float q[4]) { decodeQuaternion(word, q); }

uint32_t orc_decode(const float* records, uint32_t count, const orc_encoding* e, float* positions, uint32_t* shape,
                    uint32_t* sh, uint32_t* origin) {
    const uint32_t keep = e->keepPerColour;
    const uint32_t shWords = keep == 0 ? 1 : (keep * 3 + 1) / 2;
    uint32_t j = 0;
    for (uint32_t i = 0; i < count; ++i) {
        const float* r = records + (size_t)i * e->stride;
        // scene/splat_encoding.slang:71-85 (3DGS modes: logit opacity, log scale, SH DC)
        const float p[3] = {r[e->x], r[e->y], r[e->z]};
        const float a = 1.0f / (1.0f + expf_(-r[e->opacity]));
        float ls[3] = {r[e->scale0], r[e->scale1], r[e->scale2]};
        for (float& v : ls) v = v < -30.0f ? -INFINITY : v;
        // scene/splat_validate.slang:16-31 and splat_encoding.slang:101-108
        bool flatOk = true;
        uint32_t flats = 0;
        for (float v : ls) {
            if (v <= -1024.0f) {
                flats += 1;
            } else if (!std::isfinite(v) || !(std::fabs(v) < 60.0f)) {
                flatOk = false;
            }
        }
        const bool finite = std::isfinite(p[0]) && std::isfinite(p[1]) && std::isfinite(p[2]) && flats <= 1u && flatOk;
        if (!(finite && a >= 1.0f / 255.0f)) continue;
        // scene/splat_decode.slang:53-76
        if (origin) origin[j] = i;
        positions[j * 4 + 0] = p[0];
        positions[j * 4 + 1] = p[1];
        positions[j * 4 + 2] = p[2];
        positions[j * 4 + 3] = clampf(a, 0.0f, 5.0f);
        const float q[4] = {r[e->rotX], r[e->rotY], r[e->rotZ], r[e->rotW]};
        const float qLength = std::sqrt(((q[0] * q[0] + q[1] * q[1]) + q[2] * q[2]) + q[3] * q[3]);
        const float identity[4] = {0.0f, 0.0f, 0.0f, 1.0f};
        const uint32_t rotation = encodeQuaternion(qLength > 1e-8f ? q : identity);
        const float base[3] = {0.5f + kSH0 * r[e->dc0], 0.5f + kSH0 * r[e->dc1], 0.5f + kSH0 * r[e->dc2]};
        shape[j * 4 + 0] = rotation;
        shape[j * 4 + 1] = packHalves(halfSafe(ls[0]), halfSafe(ls[1]));
        shape[j * 4 + 2] = packHalves(halfSafe(ls[2]), halfSafe(base[0]));
        shape[j * 4 + 3] = packHalves(halfSafe(base[1]), halfSafe(base[2]));
        // :140-172: rest coefficients, rgb per basis
        uint32_t* row = sh + (size_t)j * shWords;
        if (keep == 0) {
            row[0] = 0;
        } else {
            uint32_t half = 0, word = 0, filled = 0;
            for (uint32_t basis = 0; basis < keep; ++basis) {
                for (uint32_t colour = 0; colour < 3; ++colour) {
                    const float value = r[e->restBase + colour * e->filePerColour + basis];
                    const uint32_t h = toHalf(halfSafe(value));
                    word |= h << (filled * 16);
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
        j += 1;
    }
    return j;
}

// ---- camera (modules/render/src/Camera.cpp; aofx::xform restated) --------
static void matMul(const double* a, const double* b, double* out) {
    double r[16];
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) {
            double s = 0.0;
            for (int k = 0; k < 4; ++k) s += a[i * 4 + k] * b[k * 4 + j];
            r[i * 4 + j] = s;
        }
    std::memcpy(out, r, sizeof(r));
}

// The inverse of an affine matrix (rotation/scale + translation), by the
// inverse of its 3x3 (cofactors) and -A^-1 t.
static void inverseAffine(const double* m, double* out) {
    const double a = m[0], b = m[1], c = m[2], d = m[4], e = m[5], f = m[6], g = m[8], h = m[9], i = m[10];
    const double A = e * i - f * h, B = -(d * i - f * g), C = d * h - e * g;
    const double det = a * A + b * B + c * C;
    const double inv[9] = {A / det, -(b * i - c * h) / det, (b * f - c * e) / det,
                           B / det, (a * i - c * g) / det, -(a * f - c * d) / det,
                           C / det, -(a * h - b * g) / det, (a * e - b * d) / det};
    const double t[3] = {m[3], m[7], m[11]};
    for (int r = 0; r < 3; ++r) {
        out[r * 4 + 0] = inv[r * 3 + 0];
        out[r * 4 + 1] = inv[r * 3 + 1];
        out[r * 4 + 2] = inv[r * 3 + 2];
        out[r * 4 + 3] = -(inv[r * 3 + 0] * t[0] + inv[r * 3 + 1] * t[1] + inv[r * 3 + 2] * t[2]);
    }
    out[12] = 0; out[13] = 0; out[14] = 0; out[15] = 1;
}

void orc_camera_looking_at(const double eye[3], const double target[3], const double up[3], orc_camera* out) {
    // A camera looking down its own -Z: z = normalize(eye - target), x = normalize(up x z), y = z x x.
    double z[3] = {eye[0] - target[0], eye[1] - target[1], eye[2] - target[2]};
    const double distance = std::sqrt(z[0] * z[0] + z[1] * z[1] + z[2] * z[2]);
    for (double& v : z) v /= distance;
    double x[3] = {up[1] * z[2] - up[2] * z[1], up[2] * z[0] - up[0] * z[2], up[0] * z[1] - up[1] * z[0]};
    const double xl = std::sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
    for (double& v : x) v /= xl;
    const double y[3] = {z[1] * x[2] - z[2] * x[1], z[2] * x[0] - z[0] * x[2], z[0] * x[1] - z[1] * x[0]};
    std::memset(out, 0, sizeof(*out));
    double* m = out->cameraToWorld;
    for (int r = 0; r < 3; ++r) {
        m[r * 4 + 0] = x[r];
        m[r * 4 + 1] = y[r];
        m[r * 4 + 2] = z[r];
        m[r * 4 + 3] = eye[r];
    }
    m[15] = 1.0;
    out->orthographic = 0;
    out->focal = 50.0;
    out->haperture = 24.576;
    out->nearZ = std::max(distance * 1e-3, 1e-5);
    out->farZ = 10000.0;
    out->windowScale[0] = out->windowScale[1] = 1.0;
}

void orc_projection_for(const orc_camera* camera, uint32_t width, uint32_t height, orc_projection* out) {
    std::memset(out, 0, sizeof(*out));
    double inv[16];
    inverseAffine(camera->cameraToWorld, inv);
    const double flip[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, -1, 0, 0, 0, 0, 1};
    matMul(flip, inv, out->worldToView);
    if (std::fabs(camera->windowRoll) > 1e-12) {
        const double t = camera->windowRoll * 3.14159265358979323846 / 180.0;
        const double c = std::cos(t), s = std::sin(t);
        const double rz[16] = {c, -s, 0, 0, s, c, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};
        matMul(rz, out->worldToView, out->worldToView);
    }
    const double w = (double)width, h = (double)height;
    const double focal = w * std::max(camera->focal, 1e-9) / std::max(camera->haperture, 1e-9);
    out->focalX = focal * camera->windowScale[0];
    out->focalY = focal * camera->windowScale[1];
    out->centreX = w * 0.5 + camera->windowTranslate[0] * w * 0.5;
    out->centreY = h * 0.5 + camera->windowTranslate[1] * w * 0.5;
    out->nearZ = camera->nearZ;
    out->farZ = camera->farZ;
    out->orthographic = camera->orthographic;
    out->eyeWorld[0] = camera->cameraToWorld[3];
    out->eyeWorld[1] = camera->cameraToWorld[7];
    out->eyeWorld[2] = camera->cameraToWorld[11];
}

void orc_frame_for(const orc_projection* p, const double objectToWorld[16], uint32_t width, uint32_t height,
                   uint32_t antialias, int32_t antialiased, float madeSpread, uint32_t surfels, uint32_t maxShDegree,
                   uint32_t restPerColour, uint32_t shWords, uint32_t linearCloud, const float bg[4],
                   uint32_t depthMode, float depthThreshold, const orc_edit* edit, orc_frame* f) {
    std::memset(f, 0, sizeof(*f));
    f->width = width;
    f->height = height;
    f->tile = kTile;
    f->tilesX = (width + kTile - 1) / kTile;
    f->tilesY = (height + kTile - 1) / kTile;
    f->focalX = (float)p->focalX;
    f->focalY = (float)p->focalY;
    f->centreX = (float)p->centreX;
    f->centreY = (float)p->centreY;
    f->nearZ = (float)p->nearZ;
    f->farZ = (float)p->farZ;
    f->orthographic = p->orthographic;
    // FrameParams.h:103-117 (antialiasOf, paidAt)
    const bool whole = antialiased >= 0 ? antialiased != 0 : antialias != 0;
    f->antialias = whole ? 1u : 0u;
    const float made = madeSpread * madeSpread;
    f->paidAt = !whole && made > 0.0f ? made / (made + 0.3f) : 0.0f;
    f->surfels = surfels;
    double o2v[16];
    matMul(p->worldToView, objectToWorld, o2v);
    for (int k = 0; k < 12; ++k) f->m[k] = (float)o2v[k];
    double w2o[16];
    inverseAffine(objectToWorld, w2o);
    for (int r = 0; r < 3; ++r)
        f->eye[r] = (float)(w2o[r * 4 + 0] * p->eyeWorld[0] + w2o[r * 4 + 1] * p->eyeWorld[1] +
                            w2o[r * 4 + 2] * p->eyeWorld[2] + w2o[r * 4 + 3]);
    f->restPerColour = restPerColour;
    f->shWords = shWords;
    f->shLimit = maxShDegree;
    f->linearCloud = linearCloud;
    f->depthMode = depthMode;
    f->depthThreshold = depthThreshold;
    for (int k = 0; k < 4; ++k) f->bg[k] = bg[k];
    if (edit) f->edit = *edit;
}

void orc_project(const orc_frame* f, uint32_t count, uint32_t base, const float* positions, const uint32_t* shape,
                 const uint32_t* sh, float* records, uint32_t* rects, uint32_t* touched, uint32_t* depthKeys,
                 uint32_t* visible, int threads) {
#pragma omp parallel for schedule(static, 4096) num_threads(threadsOr(threads))
    for (int64_t i = 0; i < (int64_t)count; ++i) {
        projectOne(*f, (uint32_t)i, base + (uint32_t)i, positions, shape, sh, records, rects, touched, depthKeys,
                   visible);
    }
}

void orc_project_params(const orc_frame* f, uint32_t count, uint32_t base, const float* means, const float* scales,
                        const float* quats, const float* sh, uint32_t shStride, float* records, uint32_t* rects,
                        uint32_t* touched, uint32_t* depthKeys, uint32_t* visible, int threads) {
#pragma omp parallel for schedule(static, 4096) num_threads(threadsOr(threads))
    for (int64_t ii = 0; ii < (int64_t)count; ++ii) {
        const uint32_t i = (uint32_t)ii;
        const G32 g = loadParams(means, scales, quats, sh, shStride, i);
        const float* row = sh + (size_t)i * shStride + 3;
        projectCore(*f, g,
                    [&](uint32_t degree, float x, float y, float z, float out[3]) {
                        evaluateRest([&](uint32_t index) { return row[index]; }, degree, x, y, z, out);
                    },
                    base + i, records, rects, touched, depthKeys, visible);
    }
}

void orc_colour_gradient_exact(const orc_frame* f, const uint32_t* ranges, const uint32_t* pairSplats,
                               const float* records, const float* dLdPixel, double* gradient) {
    const uint32_t tiles = f->tilesX * f->tilesY;
    for (uint32_t t = 0; t < tiles; ++t) {
        const uint32_t tx = t % f->tilesX, ty = t / f->tilesX;
        for (uint32_t ly = 0; ly < tileOf(*f); ++ly) {
            for (uint32_t lx = 0; lx < tileOf(*f); ++lx) {
                const uint32_t px = tx * tileOf(*f) + lx, py = ty * tileOf(*f) + ly;
                if (px >= f->width || py >= f->height) continue;
                const uint32_t at = py * f->width + px;
                walkPixel(*f, ranges[t * 2], ranges[t * 2 + 1], pairSplats, records, (float)px + 0.5f,
                          (float)py + 0.5f, [&](uint32_t s, float weight) {
                              for (uint32_t c = 0; c < 3; ++c)
                                  gradient[s * 3 + c] += (double)weight * (double)dLdPixel[at * 4 + c];
                          });
            }
        }
    }
}

void orc_frame_set_tile(orc_frame* f, uint32_t tile) {
    f->tile = tile;
    f->tilesX = (f->width + tile - 1) / tile;
    f->tilesY = (f->height + tile - 1) / tile;
}

namespace {

// The two-sort binning of orc_bin; with tileStride > 1, only the pairs of tiles
// t with t % tileStride == tileOffset are written (in the same relative order:
// the emit's test is per pair, and dropping whole tiles leaves each kept tile's
// run as the stable tile sort makes it).
uint64_t binSampled(const orc_frame* f, uint32_t slots, const float* records, const uint32_t* rects,
                    const uint32_t* touched, const uint32_t* depthKeys, const uint32_t* visible, uint32_t* pairTiles,
                    uint32_t* pairSplats, uint32_t* ranges, uint32_t* visibleCount, uint32_t tileStride,
                    uint32_t tileOffset) {
    const bool sampled = tileStride > 1;
    // splat_compact.slang:16-26 -- visible slots in slot order
    std::vector<uint32_t> order;
    order.reserve(slots);
    for (uint32_t s = 0; s < slots; ++s)
        if (visible[s] != 0) order.push_back(s);
    if (visibleCount) *visibleCount = (uint32_t)order.size();
    // RadixSort::sort(depthSort_, V, 24): stable on the 24-bit depth key
    std::stable_sort(order.begin(), order.end(),
                     [&](uint32_t a, uint32_t b) { return depthKeys[a] < depthKeys[b]; });
    // splat_gather_counts + PrefixSum + splat_emit.slang:17-50
    uint64_t pairs = 0;
    std::vector<uint64_t> offsets(order.size());
    for (size_t k = 0; k < order.size(); ++k) {
        offsets[k] = pairs;
        pairs += touched[order[k]];
    }
    uint64_t kept = 0;   // sampled: pairs written so far, in emit order
    for (size_t k = 0; k < order.size(); ++k) {
        const uint32_t s = order[k];
        const uint32_t expected = touched[s];
        if (expected == 0) continue;
        const float* rec = records + (size_t)s * 12;
        const uint32_t* rect = rects + (size_t)s * 4;
        uint32_t written = 0;
        for (uint32_t ty = rect[1]; ty <= rect[3] && written < expected; ++ty) {
            for (uint32_t tx = rect[0]; tx <= rect[2] && written < expected; ++tx) {
                if (!tileTouched(*f, rec[0], rec[1], rec[4], rec[5], rec[6], rec[3], tx, ty)) continue;
                const uint32_t t = ty * f->tilesX + tx;
                written += 1;
                if (sampled && t % tileStride != tileOffset) continue;
                const uint64_t at = sampled ? kept++ : offsets[k] + written - 1;
                if (!pairTiles) continue;   // counting only
                pairTiles[at] = t;
                pairSplats[at] = s;
            }
        }
    }
    if (sampled) pairs = kept;
    if (!pairTiles) return pairs;
    // RadixSort::sort(tileSort_, P, bitsFor(tiles)): stable on the tile
    std::vector<uint64_t> idx(pairs);
    std::iota(idx.begin(), idx.end(), 0);
    std::stable_sort(idx.begin(), idx.end(), [&](uint64_t a, uint64_t b) { return pairTiles[a] < pairTiles[b]; });
    std::vector<uint32_t> t2(pairs), s2(pairs);
    for (uint64_t i = 0; i < pairs; ++i) {
        t2[i] = pairTiles[idx[i]];
        s2[i] = pairSplats[idx[i]];
    }
    std::copy(t2.begin(), t2.end(), pairTiles);
    std::copy(s2.begin(), s2.end(), pairSplats);
    // splat_tiles_clear.slang + splat_ranges.slang:11-25
    const uint32_t tiles = f->tilesX * f->tilesY;
    std::fill(ranges, ranges + 2 * (size_t)tiles, 0u);
    for (uint64_t i = 0; i < pairs; ++i) {
        const uint32_t t = pairTiles[i];
        if (i == 0 || pairTiles[i - 1] != t) ranges[t * 2] = (uint32_t)i;
        if (i + 1 == pairs || pairTiles[i + 1] != t) ranges[t * 2 + 1] = (uint32_t)(i + 1);
    }
    return pairs;
}

}   // namespace

uint64_t orc_bin(const orc_frame* f, uint32_t slots, const float* records, const uint32_t* rects,
                 const uint32_t* touched, const uint32_t* depthKeys, const uint32_t* visible, uint32_t* pairTiles,
                 uint32_t* pairSplats, uint32_t* ranges, uint32_t* visibleCount) {
    return binSampled(f, slots, records, rects, touched, depthKeys, visible, pairTiles, pairSplats, ranges,
                      visibleCount, 1, 0);
}

uint64_t orc_bin_sampled(const orc_frame* f, uint32_t slots, const float* records, const uint32_t* rects,
                         const uint32_t* touched, const uint32_t* depthKeys, const uint32_t* visible,
                         uint32_t* pairTiles, uint32_t* pairSplats, uint32_t* ranges, uint32_t tileStride,
                         uint32_t tileOffset) {
    return binSampled(f, slots, records, rects, touched, depthKeys, visible, pairTiles, pairSplats, ranges, nullptr,
                      std::max(tileStride, 1u), tileOffset);
}

uint64_t orc_blend(const orc_frame* f, const uint32_t* ranges, const uint32_t* pairSplats, const float* records,
                   float* colour, float* depth, float* finalT, uint32_t* lastContrib, int threads) {
    const uint32_t tiles = f->tilesX * f->tilesY;
    uint64_t evaluated = 0;
#pragma omp parallel for schedule(dynamic, 4) reduction(+ : evaluated) num_threads(threadsOr(threads))
    for (int64_t ti = 0; ti < (int64_t)tiles; ++ti) {
        const uint32_t t = (uint32_t)ti;
        const uint32_t tx = t % f->tilesX, ty = t / f->tilesX;
        const uint32_t start = ranges[t * 2], end = ranges[t * 2 + 1];
        for (uint32_t ly = 0; ly < tileOf(*f); ++ly) {
            for (uint32_t lx = 0; lx < tileOf(*f); ++lx) {
                const uint32_t px = tx * tileOf(*f) + lx, py = ty * tileOf(*f) + ly;
                if (px >= f->width || py >= f->height) continue;
                const Walk wk = walkPixel(*f, start, end, pairSplats, records, (float)px + 0.5f, (float)py + 0.5f,
                                          [](uint32_t, float) {});
                evaluated += wk.evaluated;
                const uint32_t at = py * f->width + px;
                const float coverage = 1.0f - wk.t;
                colour[at * 4 + 0] = wk.rgb[0] + wk.t * f->bg[0];
                colour[at * 4 + 1] = wk.rgb[1] + wk.t * f->bg[1];
                colour[at * 4 + 2] = wk.rgb[2] + wk.t * f->bg[2];
                colour[at * 4 + 3] = coverage + wk.t * f->bg[3];
                depth[at] = f->depthMode == 0 ? (coverage > 1e-6f ? wk.depthSum / coverage : 0.0f)
                                              : std::max(wk.depthAt, 0.0f);
                if (finalT) finalT[at] = wk.t;
                if (lastContrib) lastContrib[at] = wk.last;
            }
        }
    }
    return evaluated;
}

void orc_blend_over(const orc_frame* f, const uint32_t* ranges, const uint32_t* pairSplats, const float* records,
                    const float* underColour, const float* underDepth, float* colour, float* depth, int threads) {
    // splat_blend.slang:236-578 with composite = true and only the under layer
    // (no points, catchers or media): the walk stops at the layer, which then
    // takes the rest of the pixel (:516-523,555-575).
    const uint32_t tiles = f->tilesX * f->tilesY;
#pragma omp parallel for schedule(dynamic, 4) num_threads(threadsOr(threads))
    for (int64_t ti = 0; ti < (int64_t)tiles; ++ti) {
        const uint32_t t = (uint32_t)ti;
        const uint32_t tx = t % f->tilesX, ty = t / f->tilesX;
        const uint32_t start = ranges[t * 2], end = ranges[t * 2 + 1];
        for (uint32_t ly = 0; ly < tileOf(*f); ++ly) {
            for (uint32_t lx = 0; lx < tileOf(*f); ++lx) {
                const uint32_t px = tx * tileOf(*f) + lx, py = ty * tileOf(*f) + ly;
                if (px >= f->width || py >= f->height) continue;
                const uint32_t at = py * f->width + px;
                const float underZ = underDepth[at];
                const bool hit = underZ > 0.0f;
                Walk wk = walkPixel(*f, start, end, pairSplats, records, (float)px + 0.5f, (float)py + 0.5f,
                                    [](uint32_t, float) {}, hit ? underZ : 0.0f);
                const float coverage = 1.0f - wk.t;
                float behind[4] = {f->bg[0], f->bg[1], f->bg[2], f->bg[3]};
                if (hit) {
                    for (int k = 0; k < 4; ++k) behind[k] = underColour[at * 4 + k];
                    wk.depthSum = wk.depthSum + wk.t * underZ;
                    if (wk.depthAt < 0.0f) wk.depthAt = underZ;
                }
                const float total = hit ? 1.0f : coverage;
                colour[at * 4 + 0] = wk.rgb[0] + wk.t * behind[0];
                colour[at * 4 + 1] = wk.rgb[1] + wk.t * behind[1];
                colour[at * 4 + 2] = wk.rgb[2] + wk.t * behind[2];
                colour[at * 4 + 3] = coverage + wk.t * behind[3];
                depth[at] = f->depthMode == 0 ? (total > 1e-6f ? wk.depthSum / total : 0.0f)
                                              : std::max(wk.depthAt, 0.0f);
            }
        }
    }
}

void orc_blend_matte(const orc_frame* f, const uint32_t* ranges, const uint32_t* pairSplats, const float* records,
                     const uint32_t* cryptoIds, const float* underDepth, const uint32_t* underCrypto, float* crypto,
                     int threads) {
    // splat_blend.slang:88-143 (CryptoList), :420-421 (each splat's weight under its
    // id), :525-534 (the under layer's id takes the light left): 6 ids a pixel,
    // written ranked as 3 float4 layers. underDepth may be null (no layer).
    constexpr uint32_t kSlots = 6;
    const uint32_t tiles = f->tilesX * f->tilesY;
    const uint32_t pixels = f->width * f->height;
#pragma omp parallel for schedule(dynamic, 4) num_threads(threadsOr(threads))
    for (int64_t ti = 0; ti < (int64_t)tiles; ++ti) {
        const uint32_t t = (uint32_t)ti;
        const uint32_t tx = t % f->tilesX, ty = t / f->tilesX;
        for (uint32_t ly = 0; ly < tileOf(*f); ++ly) {
            for (uint32_t lx = 0; lx < tileOf(*f); ++lx) {
                const uint32_t px = tx * tileOf(*f) + lx, py = ty * tileOf(*f) + ly;
                if (px >= f->width || py >= f->height) continue;
                const uint32_t at = py * f->width + px;
                uint32_t ids[kSlots] = {0, 0, 0, 0, 0, 0};
                float weights[kSlots] = {0, 0, 0, 0, 0, 0};
                const auto add = [&](uint32_t id, float w) {
                    if (w <= 0.0f || id == 0) return;
                    uint32_t lightest = 0;
                    for (uint32_t k = 0; k < kSlots; ++k) {
                        if (ids[k] == id && weights[k] > 0.0f) {
                            weights[k] += w;
                            return;
                        }
                        if (weights[k] < weights[lightest]) lightest = k;
                    }
                    if (w > weights[lightest]) {
                        ids[lightest] = id;
                        weights[lightest] = w;
                    }
                };
                const float underZ = underDepth ? underDepth[at] : 0.0f;
                const bool hit = underZ > 0.0f;
                const Walk wk = walkPixel(*f, ranges[t * 2], ranges[t * 2 + 1], pairSplats, records, (float)px + 0.5f,
                                          (float)py + 0.5f, [&](uint32_t s, float w) { add(cryptoIds[s], w); },
                                          hit ? underZ : 0.0f);
                add(hit && underCrypto ? underCrypto[at] : 0u, hit ? wk.t : 0.0f);
                uint32_t order[kSlots];
                for (uint32_t k = 0; k < kSlots; ++k) order[k] = k;
                for (uint32_t i = 1; i < kSlots; ++i) {
                    const uint32_t pick = order[i];
                    uint32_t j = i;
                    while (j > 0 && weights[order[j - 1]] < weights[pick]) {
                        order[j] = order[j - 1];
                        --j;
                    }
                    order[j] = pick;
                }
                for (uint32_t layer = 0; layer < kSlots / 2; ++layer) {
                    const uint32_t a = order[layer * 2], b = order[layer * 2 + 1];
                    float* out = crypto + ((size_t)layer * pixels + at) * 4;
                    float idA = 0.0f, idB = 0.0f;
                    if (weights[a] > 0.0f) std::memcpy(&idA, &ids[a], 4);
                    if (weights[b] > 0.0f) std::memcpy(&idB, &ids[b], 4);
                    out[0] = idA;
                    out[1] = std::max(weights[a], 0.0f);
                    out[2] = idB;
                    out[3] = std::max(weights[b], 0.0f);
                }
            }
        }
    }
}

void orc_colour_gradient(const orc_frame* f, const uint32_t* ranges, const uint32_t* pairSplats,
                         const float* records, const float* dLdPixel, int32_t* contribution) {
    const uint32_t tiles = f->tilesX * f->tilesY;
    const float kScale = 256.0f;   // frame.slang:36
    for (uint32_t t = 0; t < tiles; ++t) {
        const uint32_t tx = t % f->tilesX, ty = t / f->tilesX;
        for (uint32_t ly = 0; ly < tileOf(*f); ++ly) {
            for (uint32_t lx = 0; lx < tileOf(*f); ++lx) {
                const uint32_t px = tx * tileOf(*f) + lx, py = ty * tileOf(*f) + ly;
                if (px >= f->width || py >= f->height) continue;
                const uint32_t at = py * f->width + px;
                walkPixel(*f, ranges[t * 2], ranges[t * 2 + 1], pairSplats, records, (float)px + 0.5f,
                          (float)py + 0.5f, [&](uint32_t s, float weight) {
                              // splat_blend.slang:381-398
                              for (uint32_t c = 0; c < 3; ++c) {
                                  const float g = (weight * dLdPixel[at * 4 + c]) * kScale;
                                  const int step =
                                      (int)std::floor(g + hash01((at * 3u + c) ^ (s * 2654435761u)));
                                  contribution[s * 4 + c] += step;
                              }
                              contribution[s * 4 + 3] += (int32_t)(uint32_t)(weight * kScale + 0.5f);
                          });
            }
        }
    }
}

void orc_contribution_weight(const orc_frame* f, const uint32_t* ranges, const uint32_t* pairSplats,
                             const float* records, uint32_t* contribution) {
    const uint32_t tiles = f->tilesX * f->tilesY;
    for (uint32_t t = 0; t < tiles; ++t) {
        const uint32_t tx = t % f->tilesX, ty = t / f->tilesX;
        for (uint32_t ly = 0; ly < tileOf(*f); ++ly) {
            for (uint32_t lx = 0; lx < tileOf(*f); ++lx) {
                const uint32_t px = tx * tileOf(*f) + lx, py = ty * tileOf(*f) + ly;
                if (px >= f->width || py >= f->height) continue;
                walkPixel(*f, ranges[t * 2], ranges[t * 2 + 1], pairSplats, records, (float)px + 0.5f,
                          (float)py + 0.5f, [&](uint32_t s, float weight) {
                              // splat_blend.slang:364-365
                              contribution[s] += (uint32_t)(weight * 4096.0f + 0.5f);
                          });
            }
        }
    }
}

void orc_contribution_change(const orc_frame* f, const uint32_t* ranges, const uint32_t* pairSplats,
                             const float* records, const float* wholeFrame, uint32_t* contribution) {
    // splat_blend.slang:366-380, summed in 64 bits a slot and written as (low, high) words
    const uint32_t tiles = f->tilesX * f->tilesY;
    uint32_t slots = 0;
    for (uint32_t t = 0; t < tiles; ++t)
        for (uint32_t j = ranges[t * 2]; j < ranges[t * 2 + 1]; ++j) slots = std::max(slots, pairSplats[j] + 1);
    std::vector<uint64_t> sums(slots, 0);
    for (uint32_t t = 0; t < tiles; ++t) {
        const uint32_t tx = t % f->tilesX, ty = t / f->tilesX;
        for (uint32_t ly = 0; ly < tileOf(*f); ++ly) {
            for (uint32_t lx = 0; lx < tileOf(*f); ++lx) {
                const uint32_t px = tx * tileOf(*f) + lx, py = ty * tileOf(*f) + ly;
                if (px >= f->width || py >= f->height) continue;
                const float* whole = wholeFrame + (size_t)(py * f->width + px) * 4;
                walkPixel(*f, ranges[t * 2], ranges[t * 2 + 1], pairSplats, records, (float)px + 0.5f,
                          (float)py + 0.5f, [&](uint32_t s, float weight, const Walk& wk, float alpha, const float* rec) {
                              const float after = std::fmax(wk.t * (1.0f - alpha), 1.0e-4f);
                              float ch[3];
                              for (int k = 0; k < 3; ++k)
                                  ch[k] = weight * (rec[8 + k] - (whole[k] - (wk.rgb[k] + weight * rec[8 + k])) / after);
                              const float d2 = (ch[0] * ch[0] + ch[1] * ch[1]) + ch[2] * ch[2];
                              sums[s] += (uint32_t)(std::fmin(d2, 1.0f) * 16777216.0f + 0.5f);
                          });
            }
        }
    }
    for (uint32_t s = 0; s < slots; ++s) {
        contribution[s * 2] += (uint32_t)sums[s];
        contribution[s * 2 + 1] += (uint32_t)(sums[s] >> 32);
    }
}

void orc_contribution_lift(const orc_frame* f, const uint32_t* ranges, const uint32_t* pairSplats,
                           const float* records, const float* liftMask, uint32_t* contribution) {
    // splat_blend.slang:399-407
    const uint32_t tiles = f->tilesX * f->tilesY;
    for (uint32_t t = 0; t < tiles; ++t) {
        const uint32_t tx = t % f->tilesX, ty = t / f->tilesX;
        for (uint32_t ly = 0; ly < tileOf(*f); ++ly) {
            for (uint32_t lx = 0; lx < tileOf(*f); ++lx) {
                const uint32_t px = tx * tileOf(*f) + lx, py = ty * tileOf(*f) + ly;
                if (px >= f->width || py >= f->height) continue;
                const float m = std::fmin(std::fmax(liftMask[py * f->width + px], 0.0f), 1.0f);
                walkPixel(*f, ranges[t * 2], ranges[t * 2 + 1], pairSplats, records, (float)px + 0.5f,
                          (float)py + 0.5f, [&](uint32_t s, float weight) {
                              const uint32_t seen = (uint32_t)(weight * 1024.0f + 0.5f);
                              if (seen == 0u) return;
                              contribution[s * 2 + 1] += seen;
                              contribution[s * 2] += (uint32_t)((weight * m) * 1024.0f + 0.5f);
                          });
            }
        }
    }
}

void orc_matte_lift(const orc_frame* f, const uint32_t* ranges, const uint32_t* pairSplats, const float* records,
                    const uint32_t* liftSums, uint32_t hard, float threshold, float* matte) {
    // splat_blend.slang:423-435,536-539
    const uint32_t tiles = f->tilesX * f->tilesY;
    for (uint32_t t = 0; t < tiles; ++t) {
        const uint32_t tx = t % f->tilesX, ty = t / f->tilesX;
        for (uint32_t ly = 0; ly < tileOf(*f); ++ly) {
            for (uint32_t lx = 0; lx < tileOf(*f); ++lx) {
                const uint32_t px = tx * tileOf(*f) + lx, py = ty * tileOf(*f) + ly;
                if (px >= f->width || py >= f->height) continue;
                float known = 0.0f, inside = 0.0f, untold = 0.0f;
                walkPixel(*f, ranges[t * 2], ranges[t * 2 + 1], pairSplats, records, (float)px + 0.5f,
                          (float)py + 0.5f, [&](uint32_t s, float weight) {
                              const uint32_t seen = liftSums[s * 2 + 1];
                              if (seen != 0u) {
                                  float share = (float)liftSums[s * 2] / (float)seen;
                                  if (hard) share = share > threshold ? 1.0f : 0.0f;
                                  known = known + weight;
                                  inside = inside + weight * share;
                              } else {
                                  untold = untold + weight;
                              }
                          });
                const float share = known > 0.0f ? inside / known : 0.0f;
                matte[py * f->width + px] = std::fmin(std::fmax(inside + untold * share, 0.0f), 1.0f);
            }
        }
    }
}

void orc_trace(const orc_frame* f, const uint32_t* ranges, const uint32_t* pairSplats, const float* records,
               uint32_t* trace) {
    // splat_blend.slang:445-451,545-551 with splat_trace.slang:33-128 (no layer under the splats)
    constexpr uint32_t K = 4, kWords = K * 2 + K / 2 + 1;
    const uint32_t pixels = f->width * f->height, tiles = f->tilesX * f->tilesY;
    for (uint32_t t = 0; t < tiles; ++t) {
        const uint32_t tx = t % f->tilesX, ty = t / f->tilesX;
        for (uint32_t ly = 0; ly < tileOf(*f); ++ly) {
            for (uint32_t lx = 0; lx < tileOf(*f); ++lx) {
                const uint32_t px = tx * tileOf(*f) + lx, py = ty * tileOf(*f) + ly;
                if (px >= f->width || py >= f->height) continue;
                uint32_t slots[K] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu};
                float weights[K] = {0, 0, 0, 0}, total = 0.0f, floor = 0.0f;
                uint32_t lightest = 0;
                walkPixel(*f, ranges[t * 2], ranges[t * 2 + 1], pairSplats, records, (float)px + 0.5f,
                          (float)py + 0.5f, [&](uint32_t s, float weight) {
                              total = total + weight;
                              if (!(weight > floor)) return;
                              slots[lightest] = s;
                              weights[lightest] = weight;
                              lightest = 0;
                              for (uint32_t k = 1; k < K; ++k)
                                  if (weights[k] < weights[lightest]) lightest = k;
                              floor = weights[lightest];
                          });
                const uint32_t at = py * f->width + px;
                if (!(total > 0.0f)) {
                    trace[at] = 0xFFFFFFFEu;
                    continue;
                }
                uint32_t order[K] = {0, 1, 2, 3};
                for (uint32_t i = 1; i < K; ++i) {
                    const uint32_t pick = order[i];
                    uint32_t j = i;
                    while (j > 0 && weights[order[j - 1]] < weights[pick]) {
                        order[j] = order[j - 1];
                        --j;
                    }
                    order[j] = pick;
                }
                float held = 0.0f;
                for (uint32_t k = 0; k < K; ++k) {
                    const uint32_t from = order[k];
                    const bool some = weights[from] > 0.0f;
                    trace[k * pixels + at] = some ? slots[from] : 0xFFFFFFFFu;
                    uint32_t bits = 0;
                    if (some) std::memcpy(&bits, &records[(size_t)slots[from] * 12 + 2], 4);
                    trace[(K + k) * pixels + at] = bits;
                    held = held + weights[from];
                }
                for (uint32_t pair = 0; pair < K / 2; ++pair)
                    trace[(K * 2 + pair) * pixels + at] = packHalves(weights[order[pair * 2]], weights[order[pair * 2 + 1]]);
                trace[(kWords - 1) * pixels + at] = packHalves(std::fmax(total - held, 0.0f), 0.0f);
            }
        }
    }
}

void orc_position(uint32_t width, uint32_t height, uint32_t orthographic, float focalX, float focalY, float centreX,
                  float centreY, const float r[12], const float* depth, float* position) {
    // usd/aov_position.slang:34-52
    for (uint32_t pixel = 0; pixel < width * height; ++pixel) {
        const float z = depth[pixel];
        float* out = position + (size_t)pixel * 4;
        if (!(z > 0.0f)) {
            out[0] = out[1] = out[2] = out[3] = 0.0f;
            continue;
        }
        const float px = (float)(pixel % width) + 0.5f;
        const float py = (float)(pixel / width) + 0.5f;
        const float scale = orthographic != 0 ? 1.0f : z;
        const float v[4] = {((px - centreX) / focalX) * scale, ((py - centreY) / focalY) * scale, z, 1.0f};
        for (int k = 0; k < 3; ++k)
            out[k] = ((r[k * 4 + 0] * v[0] + r[k * 4 + 1] * v[1]) + r[k * 4 + 2] * v[2]) + r[k * 4 + 3] * v[3];
        out[3] = 1.0f;
    }
}

}   // extern "C"
