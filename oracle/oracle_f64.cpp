// ORACLE -- TEST INFRASTRUCTURE ONLY (see oracle.h). The plain splat path
// evaluated in double: splat/splat_project.slang:497-785 (projectSplat<0>) for
// the footprint and colour, reference/reference_blend.slang:28-144 for the
// walk, with the rasteriser's own order (24-bit depth key, then slot:
// splat/frame.slang:6-20) so that what it measures is arithmetic, not order.
#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr uint32_t kTile = 16;
constexpr double kSH0 = 0.28209479177387814;

struct Gauss64 {
    double p[3];
    double opacity;
    double scale[3];
    double q[4];   // x y z w, unit
    double base[3];
    double rest[15][3];
    uint32_t degree;
};

struct Rec64 {
    bool live = false;
    bool faintNear = false;   // alpha within the margin of 1/255 (live or not)
    double cx, cy, z, cutoff, a, b, c, alpha, colour[3];
    uint32_t key;
    uint32_t slot;
    double ex, ey;
};

float halfToFloat(uint16_t h) { return orc_f16_to_f32(h); }

double srgbToLinear(double c) {
    c = std::max(c, 0.0);
    return c <= 0.04045 ? c / 12.92 : std::pow((c + 0.055) / 1.055, 2.4);
}

void evaluateRest(const Gauss64& g, uint32_t degree, double x, double y, double z, double out[3]) {
    const double kC1 = 0.4886025119029199;
    const double kC2[5] = {1.0925484305920792, -1.0925484305920792, 0.31539156525252005, -1.0925484305920792,
                           0.5462742152960396};
    const double kC3[7] = {-0.5900435899266435, 2.890611442640554, -0.4570457994644658, 0.3731763325901154,
                           -0.4570457994644658, 1.445305721320277, -0.5900435899266435};
    for (int ch = 0; ch < 3; ++ch) {
        const auto B = [&](int k) { return g.rest[k][ch]; };
        double r = 0.0;
        if (degree >= 1) r = -kC1 * y * B(0) + kC1 * z * B(1) - kC1 * x * B(2);
        if (degree >= 2) {
            const double xx = x * x, yy = y * y, zz = z * z, xy = x * y, yz = y * z, xz = x * z;
            r += kC2[0] * xy * B(3) + kC2[1] * yz * B(4) + kC2[2] * (2.0 * zz - xx - yy) * B(5) +
                 kC2[3] * xz * B(6) + kC2[4] * (xx - yy) * B(7);
            if (degree >= 3) {
                r += kC3[0] * y * (3.0 * xx - yy) * B(8) + kC3[1] * xy * z * B(9) +
                     kC3[2] * y * (4.0 * zz - xx - yy) * B(10) + kC3[3] * z * (2.0 * zz - 3.0 * xx - 3.0 * yy) * B(11) +
                     kC3[4] * x * (4.0 * zz - xx - yy) * B(12) + kC3[5] * z * (xx - yy) * B(13) +
                     kC3[6] * x * (xx - 3.0 * yy) * B(14);
            }
        }
        out[ch] = r;
    }
}

double minPowerOverBox(double a, double b, double c, double lox, double loy, double hix, double hiy) {
    if (lox <= 0.0 && hix >= 0.0 && loy <= 0.0 && hiy >= 0.0) return 0.0;
    double best = 1e300;
    for (int e = 0; e < 2; ++e) {
        const double x = e == 0 ? lox : hix;
        const double y = c > 1e-12 ? std::min(std::max(-b * x / c, loy), hiy) : loy;
        best = std::min(best, a * x * x + 2.0 * b * x * y + c * y * y);
    }
    for (int e = 0; e < 2; ++e) {
        const double y = e == 0 ? loy : hiy;
        const double x = a > 1e-12 ? std::min(std::max(-b * y / a, lox), hix) : lox;
        best = std::min(best, a * x * x + 2.0 * b * x * y + c * y * y);
    }
    return best;
}

// projectSplat<0> in double; `margin` widens the faint cull into a band that
// is recorded (faintNear) rather than decided.
Rec64 project64(const orc_frame64& f, const Gauss64& g, double margin) {
    Rec64 r;
    const double* m = f.m;
    const double tx = m[0] * g.p[0] + m[1] * g.p[1] + m[2] * g.p[2] + m[3];
    const double ty = m[4] * g.p[0] + m[5] * g.p[1] + m[6] * g.p[2] + m[7];
    const double tz = m[8] * g.p[0] + m[9] * g.p[1] + m[10] * g.p[2] + m[11];
    if (!(tz > f.nearZ) || tz > f.farZ) return r;
    const double x = g.q[0], y = g.q[1], z = g.q[2], w = g.q[3];
    const double R[3][3] = {{1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)},
                            {2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)},
                            {2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)}};
    double M[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) M[i][j] = R[i][j] * g.scale[j];
    double jx[3], jy[3], cx, cy;
    if (f.orthographic) {
        jx[0] = f.focalX; jx[1] = 0; jx[2] = 0;
        jy[0] = 0; jy[1] = f.focalY; jy[2] = 0;
        cx = f.focalX * tx + f.centreX;
        cy = f.focalY * ty + f.centreY;
    } else {
        const double invZ = 1.0 / tz;
        cx = f.focalX * tx * invZ + f.centreX;
        cy = f.focalY * ty * invZ + f.centreY;
        const double loX = (-0.15 * f.width - f.centreX) / f.focalX, hiX = (1.15 * f.width - f.centreX) / f.focalX;
        const double loY = (-0.15 * f.height - f.centreY) / f.focalY, hiY = (1.15 * f.height - f.centreY) / f.focalY;
        const double txc = std::min(std::max(tx * invZ, loX), hiX) * tz;
        const double tyc = std::min(std::max(ty * invZ, loY), hiY) * tz;
        jx[0] = f.focalX * invZ; jx[1] = 0; jx[2] = -f.focalX * txc * invZ * invZ;
        jy[0] = 0; jy[1] = f.focalY * invZ; jy[2] = -f.focalY * tyc * invZ * invZ;
    }
    const double W[3][3] = {{m[0], m[1], m[2]}, {m[4], m[5], m[6]}, {m[8], m[9], m[10]}};
    double t3[3], u3[3], ax[3], ay[3];
    for (int j = 0; j < 3; ++j) {
        t3[j] = jx[0] * W[0][j] + jx[1] * W[1][j] + jx[2] * W[2][j];
        u3[j] = jy[0] * W[0][j] + jy[1] * W[1][j] + jy[2] * W[2][j];
    }
    for (int j = 0; j < 3; ++j) {
        ax[j] = t3[0] * M[0][j] + t3[1] * M[1][j] + t3[2] * M[2][j];
        ay[j] = u3[0] * M[0][j] + u3[1] * M[1][j] + u3[2] * M[2][j];
    }
    double a = ax[0] * ax[0] + ax[1] * ax[1] + ax[2] * ax[2];
    const double b = ax[0] * ay[0] + ax[1] * ay[1] + ax[2] * ay[2];
    double c = ay[0] * ay[0] + ay[1] * ay[1] + ay[2] * ay[2];
    const double before = a * c - b * b;
    a += 0.3;
    c += 0.3;
    const double det = a * c - b * b;
    if (!(det > 1e-12)) return r;
    const double filtered = std::sqrt(std::max(before, 0.0) / det);
    const double paid = f.antialias ? filtered : f.paidAt > 0.0 ? std::min(filtered / f.paidAt, 1.0) : 1.0;
    const double spread = paid * g.opacity;
    const double alpha =
        g.opacity > 1.0 ? g.opacity : (spread >= 1.0 / 255.0 ? spread + (1.0 - paid) / 255.0 : spread);
    const double faint = 1.0 / 255.0;
    r.faintNear = std::fabs(alpha - faint) <= margin * faint;
    if (!(alpha >= faint) && !r.faintNear) return r;
    r.cx = cx;
    r.cy = cy;
    r.z = tz;
    r.a = c / det;
    r.b = -b / det;
    r.c = a / det;
    r.alpha = alpha;
    r.cutoff = std::min(2.0 * std::log(std::max(255.0 * alpha, 1.0001)), 9.0);
    const double d2 = r.a * r.c - r.b * r.b;
    r.ex = std::sqrt(std::max(r.cutoff * r.c / d2, 0.0)) * (1.0 + 1e-6) + 1e-6;
    r.ey = std::sqrt(std::max(r.cutoff * r.a / d2, 0.0)) * (1.0 + 1e-6) + 1e-6;
    const uint32_t degree = std::min(g.degree, f.shLimit);
    double d[3] = {g.p[0] - f.eye[0], g.p[1] - f.eye[1], g.p[2] - f.eye[2]};
    const double len = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    double rest[3];
    evaluateRest(g, degree, d[0] / len, d[1] / len, d[2] / len, rest);
    for (int k = 0; k < 3; ++k) {
        const double v = g.base[k] + rest[k];
        r.colour[k] = f.linearCloud ? std::max(v, 0.0) : srgbToLinear(v);
    }
    // The blend order is the method's, a discrete choice the arithmetic does not
    // refine: the 24-bit key of the FP32 depth, from the FP32 rows of the object ->
    // view transform, as the rasteriser computes it (splat_project.slang:519-523,
    // frame.slang:17-20), then the slot.
    const float zf = (((float)f.m[8] * (float)g.p[0] + (float)f.m[9] * (float)g.p[1]) + (float)f.m[10] * (float)g.p[2]) +
                     (float)f.m[11];
    uint32_t bits;
    std::memcpy(&bits, &zf, 4);
    r.key = bits >> 7;
    r.live = alpha >= faint;
    return r;
}

struct Frame64 {
    std::vector<Rec64> recs;
    std::vector<std::vector<uint32_t>> lists;   // per tile: record indices in blend order
    uint32_t tilesX = 0, tilesY = 0;
};

void bin64(const orc_frame64& f, Frame64& fr, double margin, uint32_t tileStride, uint32_t tileOffset) {
    fr.tilesX = (f.width + kTile - 1) / kTile;
    fr.tilesY = (f.height + kTile - 1) / kTile;
    const uint32_t tiles = fr.tilesX * fr.tilesY;
    fr.lists.assign(tiles, {});
    for (uint32_t s = 0; s < fr.recs.size(); ++s) {
        const Rec64& r = fr.recs[s];
        if (!r.live && !r.faintNear) continue;
        const double x1 = r.cx - r.ex, x2 = r.cx + r.ex, y1 = r.cy - r.ey, y2 = r.cy + r.ey;
        if (x2 < 0 || y2 < 0 || x1 >= f.width || y1 >= f.height) continue;
        const uint32_t tx0 = (uint32_t)std::max(x1, 0.0) / kTile, ty0 = (uint32_t)std::max(y1, 0.0) / kTile;
        const uint32_t tx1 = (uint32_t)std::min(x2, f.width - 1.0) / kTile,
                       ty1 = (uint32_t)std::min(y2, f.height - 1.0) / kTile;
        for (uint32_t ty = ty0; ty <= ty1; ++ty) {
            for (uint32_t tx = tx0; tx <= tx1; ++tx) {
                const uint32_t t = ty * fr.tilesX + tx;
                if (t % tileStride != tileOffset) continue;
                const double fx = tx * kTile + 0.5, fy = ty * kTile + 0.5;
                const double lx = std::min((tx + 1) * kTile, f.width) - 1 + 0.5;
                const double ly = std::min((ty + 1) * kTile, f.height) - 1 + 0.5;
                if (minPowerOverBox(r.a, r.b, r.c, fx - r.cx, fy - r.cy, lx - r.cx, ly - r.cy) <=
                    r.cutoff * (1.0 + margin) + 1e-12)
                    fr.lists[t].push_back(s);
            }
        }
    }
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t t = 0; t < (int64_t)tiles; ++t) {
        auto& l = fr.lists[t];
        std::stable_sort(l.begin(), l.end(), [&](uint32_t a, uint32_t b) {
            return fr.recs[a].key != fr.recs[b].key ? fr.recs[a].key < fr.recs[b].key : a < b;
        });
    }
}

void blend64(const orc_frame64& f, const Frame64& fr, double* colour, double* depth, uint8_t* nearOut, double margin,
             uint32_t tileStride, uint32_t tileOffset, int threads) {
    const uint32_t tiles = fr.tilesX * fr.tilesY;
#pragma omp parallel for schedule(dynamic, 4) num_threads(threads > 0 ? threads : omp_get_max_threads())
    for (int64_t ti = 0; ti < (int64_t)tiles; ++ti) {
        const uint32_t t = (uint32_t)ti;
        if (t % tileStride != tileOffset) continue;
        const uint32_t tx = t % fr.tilesX, ty = t / fr.tilesX;
        for (uint32_t ly = 0; ly < kTile; ++ly) {
            for (uint32_t lx = 0; lx < kTile; ++lx) {
                const uint32_t px = tx * kTile + lx, py = ty * kTile + ly;
                if (px >= f.width || py >= f.height) continue;
                const double pxc = px + 0.5, pyc = py + 0.5;
                double rgb[3] = {0, 0, 0}, T = 1.0, depthSum = 0.0;
                bool nearD = false;

                for (uint32_t s : fr.lists[t]) {
                    const Rec64& r = fr.recs[s];
                    const double dx = pxc - r.cx, dy = pyc - r.cy;
                    const double power = r.a * dx * dx + 2.0 * r.b * dx * dy + r.c * dy * dy;
                    if (std::fabs(power - r.cutoff) <= margin * std::max(r.cutoff, 1e-3)) nearD = true;
                    if (r.faintNear && power <= r.cutoff * (1.0 + margin)) nearD = true;
                    if (!r.live || power > r.cutoff) continue;
                    const double g = std::exp(-0.5 * power);
                    double alpha = r.alpha > 1.0 ? 1.0 - std::pow(std::max(1.0 - g, 0.0),
                                                                 std::exp((r.alpha * r.alpha - 1.0) * 0.36787944))
                                                 : r.alpha * g;
                    if (std::fabs(alpha - 0.99) <= margin) nearD = true;
                    alpha = std::min(0.99, alpha);
                    if (std::fabs(alpha - 1.0 / 255.0) <= margin / 255.0) nearD = true;
                    if (alpha < 1.0 / 255.0) continue;
                    const double weight = T * alpha;
                    for (int k = 0; k < 3; ++k) rgb[k] += weight * r.colour[k];
                    depthSum += weight * r.z;
                    T *= 1.0 - alpha;
                    // T is a product of as many factors as the walk has blended, each
                    // rounded in FP32 on the GPU: its relative error grows with their
                    // count, so the stop at T = 1e-4 is flagged within a relative 1e-3
                    if (margin > 0.0 && std::fabs(T - 1e-4) <= std::max(margin, 1e-3) * 1e-4) nearD = true;
                    if (T < 1e-4) break;
                }
                const size_t at = (size_t)py * f.width + px;
                const double coverage = 1.0 - T;
                colour[at * 4 + 0] = rgb[0] + T * f.bg[0];
                colour[at * 4 + 1] = rgb[1] + T * f.bg[1];
                colour[at * 4 + 2] = rgb[2] + T * f.bg[2];
                colour[at * 4 + 3] = coverage + T * f.bg[3];
                depth[at] = coverage > 1e-6 ? depthSum / coverage : 0.0;
                if (nearOut) nearOut[at] = nearD ? 1 : 0;
            }
        }
    }
}

double sigmoid(double v) { return 1.0 / (1.0 + std::exp(-v)); }

}   // namespace

extern "C" {

void orc_frame64_from(const orc_projection* p, const double objectToWorld[16], uint32_t width, uint32_t height,
                      uint32_t antialias, uint32_t maxShDegree, uint32_t restPerColour, uint32_t shWords,
                      uint32_t linearCloud, const double bg[4], orc_frame64* f) {
    std::memset(f, 0, sizeof(*f));
    f->focalX = p->focalX;
    f->focalY = p->focalY;
    f->centreX = p->centreX;
    f->centreY = p->centreY;
    f->nearZ = p->nearZ;
    f->farZ = p->farZ;
    f->width = width;
    f->height = height;
    f->orthographic = p->orthographic;
    f->antialias = antialias;
    f->paidAt = 0.0;
    double o2v[16];
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) {
            double s = 0.0;
            for (int k = 0; k < 4; ++k) s += p->worldToView[i * 4 + k] * objectToWorld[k * 4 + j];
            o2v[i * 4 + j] = s;
        }
    for (int k = 0; k < 12; ++k) f->m[k] = o2v[k];
    // eye in the cloud's space: objectToWorld is affine; solve by its inverse.
    const double* m = objectToWorld;
    const double a = m[0], b = m[1], c = m[2], d = m[4], e = m[5], g = m[6], h = m[8], i = m[9], k = m[10];
    const double A = e * k - g * i, B = -(d * k - g * h), C = d * i - e * h;
    const double det = a * A + b * B + c * C;
    const double inv[9] = {A / det, -(b * k - c * i) / det, (b * g - c * e) / det,
                           B / det, (a * k - c * h) / det, -(a * g - c * d) / det,
                           C / det, -(a * i - b * h) / det, (a * e - b * d) / det};
    const double v[3] = {p->eyeWorld[0] - m[3], p->eyeWorld[1] - m[7], p->eyeWorld[2] - m[11]};
    for (int r = 0; r < 3; ++r) f->eye[r] = inv[r * 3] * v[0] + inv[r * 3 + 1] * v[1] + inv[r * 3 + 2] * v[2];
    f->restPerColour = restPerColour;
    f->shWords = shWords;
    f->shLimit = maxShDegree;
    f->linearCloud = linearCloud;
    for (int q = 0; q < 4; ++q) f->bg[q] = bg[q];
}

void orc_render_f64(const orc_frame64* f, uint32_t count, const float* positions, const uint32_t* shape,
                    const uint32_t* sh, double* colour, double* depth, uint8_t* nearDecision, double margin,
                    uint32_t tileStride, uint32_t tileOffset, int threads) {
    Frame64 fr;
    fr.recs.resize(count);
    const uint32_t degree = f->restPerColour >= 15 ? 3 : f->restPerColour >= 8 ? 2 : f->restPerColour >= 3 ? 1 : 0;
#pragma omp parallel for schedule(static, 4096) num_threads(threads > 0 ? threads : omp_get_max_threads())
    for (int64_t ii = 0; ii < (int64_t)count; ++ii) {
        const uint32_t i = (uint32_t)ii;
        Gauss64 g{};
        for (int k = 0; k < 3; ++k) g.p[k] = positions[i * 4 + k];
        g.opacity = positions[i * 4 + 3];
        const uint32_t* s = shape + (size_t)i * 4;
        g.scale[0] = std::exp((double)halfToFloat((uint16_t)(s[1] & 0xFFFF)));
        g.scale[1] = std::exp((double)halfToFloat((uint16_t)(s[1] >> 16)));
        g.scale[2] = std::exp((double)halfToFloat((uint16_t)(s[2] & 0xFFFF)));
        // packing.slang:59-76 in double
        const uint32_t largest = s[0] & 3u;
        const double sm[3] = {((double)((s[0] >> 22) & 1023u) / 1023.0 * 2.0 - 1.0) * std::sqrt(0.5),
                              ((double)((s[0] >> 12) & 1023u) / 1023.0 * 2.0 - 1.0) * std::sqrt(0.5),
                              ((double)((s[0] >> 2) & 1023u) / 1023.0 * 2.0 - 1.0) * std::sqrt(0.5)};
        const double rest = std::sqrt(std::max(0.0, 1.0 - (sm[0] * sm[0] + sm[1] * sm[1] + sm[2] * sm[2])));
        uint32_t next = 0;
        for (uint32_t k = 0; k < 4; ++k) g.q[k] = k == largest ? rest : sm[next++];
        g.base[0] = halfToFloat((uint16_t)(s[2] >> 16));
        g.base[1] = halfToFloat((uint16_t)(s[3] & 0xFFFF));
        g.base[2] = halfToFloat((uint16_t)(s[3] >> 16));
        g.degree = degree;
        const uint32_t* row = sh + (size_t)i * f->shWords;
        for (uint32_t b = 0; b < f->restPerColour && b < 15; ++b)
            for (uint32_t ch = 0; ch < 3; ++ch) {
                const uint32_t idx = b * 3 + ch;
                const uint32_t word = row[idx / 2];
                g.rest[b][ch] = halfToFloat((uint16_t)((idx & 1u) ? word >> 16 : word & 0xFFFF));
            }
        fr.recs[i] = project64(*f, g, margin);
        fr.recs[i].slot = i;
    }
    bin64(*f, fr, margin, tileStride == 0 ? 1 : tileStride, tileOffset);
    blend64(*f, fr, colour, depth, nearDecision, margin, tileStride == 0 ? 1 : tileStride, tileOffset, threads);
}

void orc_render_params_f64(const orc_frame64* f, uint32_t count, const double* means, const double* logScales,
                           const double* quats, const double* logits, const double* shs, uint32_t shDegree,
                           double* colour, double* depth, int threads) {
    Frame64 fr;
    fr.recs.resize(count);
    for (uint32_t i = 0; i < count; ++i) {
        Gauss64 g{};
        for (int k = 0; k < 3; ++k) {
            g.p[k] = means[i * 3 + k];
            g.scale[k] = std::exp(logScales[i * 3 + k]);
        }
        g.opacity = sigmoid(logits[i]);
        const double* q = quats + (size_t)i * 4;   // w x y z
        const double n = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
        g.q[0] = q[1] / n;
        g.q[1] = q[2] / n;
        g.q[2] = q[3] / n;
        g.q[3] = q[0] / n;
        const double* c = shs + (size_t)i * 48;
        for (int k = 0; k < 3; ++k) g.base[k] = 0.5 + kSH0 * c[k];
        for (int b = 0; b < 15; ++b)
            for (int ch = 0; ch < 3; ++ch) g.rest[b][ch] = c[3 + b * 3 + ch];
        g.degree = shDegree;
        fr.recs[i] = project64(*f, g, 0.0);
        fr.recs[i].slot = i;
    }
    bin64(*f, fr, 0.0, 1, 0);
    blend64(*f, fr, colour, depth, nullptr, 0.0, 1, 0, threads);
}

void orc_render_params_sampled_f64(const orc_frame64* f, uint32_t count, const float* means, const float* scales,
                                   const float* quats, const float* sh, uint32_t shStride, uint32_t shDegree,
                                   double* colour, double* depth, uint8_t* nearDecision, double margin,
                                   uint32_t tileStride, uint32_t tileOffset, int threads) {
    // Only the records whose rect reaches a sampled tile are kept (a cloud of
    // tens of millions fits this way), in slot order, each with its slot.
    const uint32_t stride = tileStride == 0 ? 1 : tileStride;
    const uint32_t tilesX = (f->width + kTile - 1) / kTile;
    const auto reachesSample = [&](const Rec64& r) {
        if (!r.live && !r.faintNear) return false;
        const double x1 = r.cx - r.ex, x2 = r.cx + r.ex, y1 = r.cy - r.ey, y2 = r.cy + r.ey;
        if (x2 < 0 || y2 < 0 || x1 >= f->width || y1 >= f->height) return false;
        if (stride == 1) return true;
        const uint32_t tx0 = (uint32_t)std::max(x1, 0.0) / kTile, ty0 = (uint32_t)std::max(y1, 0.0) / kTile;
        const uint32_t tx1 = (uint32_t)std::min(x2, f->width - 1.0) / kTile,
                       ty1 = (uint32_t)std::min(y2, f->height - 1.0) / kTile;
        for (uint32_t ty = ty0; ty <= ty1; ++ty) {
            const uint32_t first = ty * tilesX + tx0;
            const uint32_t gap = (tileOffset + stride - first % stride) % stride;   // to the next sampled tile
            if (gap <= tx1 - tx0) return true;
        }
        return false;
    };
    constexpr uint32_t kChunk = 1u << 16;
    const uint32_t chunks = (count + kChunk - 1) / kChunk;
    std::vector<std::vector<Rec64>> kept(chunks);
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads > 0 ? threads : omp_get_max_threads())
    for (int64_t cc = 0; cc < (int64_t)chunks; ++cc) {
        const uint32_t end = std::min<uint32_t>(count, (uint32_t)(cc + 1) * kChunk);
        for (uint32_t i = (uint32_t)cc * kChunk; i < end; ++i) {
            Gauss64 g{};
            for (int k = 0; k < 3; ++k) {
                g.p[k] = means[(size_t)i * 4 + k];
                g.scale[k] = std::exp((double)scales[(size_t)i * 4 + k]);
            }
            g.opacity = sigmoid(means[(size_t)i * 4 + 3]);
            const float* q = quats + (size_t)i * 4;   // w x y z
            const double qw = q[0], qx = q[1], qy = q[2], qz = q[3];
            const double n = std::sqrt(qw * qw + qx * qx + qy * qy + qz * qz);
            g.q[0] = qx / n;
            g.q[1] = qy / n;
            g.q[2] = qz / n;
            g.q[3] = qw / n;
            const float* c = sh + (size_t)i * shStride;
            for (int k = 0; k < 3; ++k) g.base[k] = 0.5 + kSH0 * (double)c[k];
            const uint32_t bases = shDegree >= 3 ? 15 : shDegree == 2 ? 8 : shDegree == 1 ? 3 : 0;
            for (uint32_t b = 0; b < bases && 3 + b * 3 + 2 < shStride; ++b)
                for (int ch = 0; ch < 3; ++ch) g.rest[b][ch] = c[3 + b * 3 + ch];
            g.degree = shDegree;
            Rec64 r = project64(*f, g, margin);
            r.slot = i;
            if (reachesSample(r)) kept[cc].push_back(r);
        }
    }
    Frame64 fr;
    size_t total = 0;
    for (const auto& v : kept) total += v.size();
    fr.recs.reserve(total);
    for (auto& v : kept) {
        fr.recs.insert(fr.recs.end(), v.begin(), v.end());
        std::vector<Rec64>().swap(v);
    }
    bin64(*f, fr, margin, stride, tileOffset);
    blend64(*f, fr, colour, depth, nearDecision, margin, stride, tileOffset, threads);
}

}   // extern "C"

// ---------------------------------------------------------------------------
// Central finite differences of the mean-L2 loss in double, with the blend's
// decisions frozen at the base parameters: which records each pixel blends
// (power within the cutoff, alpha at least 1/255) and where its walk stops.
// Those decisions are piecewise constant, so the derivative the analytic
// backward computes is the derivative of the frozen walk; differencing the
// unfrozen image instead would count every pixel a footprint's edge crosses.
// ---------------------------------------------------------------------------
namespace {

constexpr int kParamsPerGaussian = 59;   // means 3, logit 1, log scales 3, quat 4 (w x y z), sh 48

struct ParamSet {
    const double *means, *logScales, *quats, *logits, *shs;
    uint32_t degree;
};

Gauss64 gaussOf(const ParamSet& P, uint32_t i, int perturbed, double delta) {
    double v[kParamsPerGaussian];
    v[0] = P.means[i * 3 + 0]; v[1] = P.means[i * 3 + 1]; v[2] = P.means[i * 3 + 2];
    v[3] = P.logits[i];
    v[4] = P.logScales[i * 3 + 0]; v[5] = P.logScales[i * 3 + 1]; v[6] = P.logScales[i * 3 + 2];
    for (int k = 0; k < 4; ++k) v[7 + k] = P.quats[i * 4 + k];
    for (int k = 0; k < 48; ++k) v[11 + k] = P.shs[(size_t)i * 48 + k];
    if (perturbed >= 0) v[perturbed] += delta;
    Gauss64 g{};
    for (int k = 0; k < 3; ++k) {
        g.p[k] = v[k];
        g.scale[k] = std::exp(v[4 + k]);
    }
    g.opacity = sigmoid(v[3]);
    const double n = std::sqrt(v[7] * v[7] + v[8] * v[8] + v[9] * v[9] + v[10] * v[10]);
    g.q[0] = v[8] / n;
    g.q[1] = v[9] / n;
    g.q[2] = v[10] / n;
    g.q[3] = v[7] / n;
    for (int k = 0; k < 3; ++k) g.base[k] = 0.5 + kSH0 * v[11 + k];
    for (int b = 0; b < 15; ++b)
        for (int ch = 0; ch < 3; ++ch) g.rest[b][ch] = v[11 + 3 + b * 3 + ch];
    g.degree = P.degree;
    return g;
}

// A pixel's frozen walk: the records it blended, in order.
struct FrozenPixel {
    std::vector<uint32_t> slots;
};

double pixelColourWith(const orc_frame64& f, const FrozenPixel& fp, const std::vector<Rec64>& recs, uint32_t px,
                       uint32_t py, uint32_t overrideSlot, const Rec64* overrideRec, double out[3]) {
    const double pxc = px + 0.5, pyc = py + 0.5;
    double rgb[3] = {0, 0, 0}, T = 1.0;
    for (uint32_t s : fp.slots) {
        const Rec64& r = (s == overrideSlot && overrideRec) ? *overrideRec : recs[s];
        const double dx = pxc - r.cx, dy = pyc - r.cy;
        const double power = r.a * dx * dx + 2.0 * r.b * dx * dy + r.c * dy * dy;
        const double alpha = std::min(0.99, r.alpha * std::exp(-0.5 * power));
        const double w = T * alpha;
        for (int k = 0; k < 3; ++k) rgb[k] += w * r.colour[k];
        T *= 1.0 - alpha;
    }
    for (int k = 0; k < 3; ++k) out[k] = rgb[k] + T * f.bg[k];
    return T;
}

}   // namespace

extern "C" void orc_fd_gradients_f64(const orc_frame64* f, uint32_t count, const double* means,
                                     const double* logScales, const double* quats, const double* logits,
                                     const double* shs, uint32_t shDegree, const float* target, const uint32_t* which,
                                     uint32_t nWhich, double eps, double* out, double* lossOut, int threads) {
    const ParamSet P{means, logScales, quats, logits, shs, shDegree};
    Frame64 fr;
    fr.recs.resize(count);
#pragma omp parallel for schedule(static, 1024) num_threads(threads > 0 ? threads : omp_get_max_threads())
    for (int64_t i = 0; i < (int64_t)count; ++i) {
        fr.recs[i] = project64(*f, gaussOf(P, (uint32_t)i, -1, 0.0), 0.0);
        fr.recs[i].slot = (uint32_t)i;
    }
    bin64(*f, fr, 0.0, 1, 0);
    const uint32_t W = f->width, H = f->height;
    std::vector<FrozenPixel> frozen((size_t)W * H);
    std::vector<double> base((size_t)W * H * 3);
    double loss = 0.0;
    const double scale = 1.0 / (3.0 * (double)W * (double)H);
    const uint32_t tiles = fr.tilesX * fr.tilesY;
#pragma omp parallel for schedule(dynamic, 4) reduction(+ : loss) num_threads(threads > 0 ? threads : omp_get_max_threads())
    for (int64_t ti = 0; ti < (int64_t)tiles; ++ti) {
        const uint32_t t = (uint32_t)ti, tx = t % fr.tilesX, ty = t / fr.tilesX;
        for (uint32_t ly = 0; ly < kTile; ++ly)
            for (uint32_t lx = 0; lx < kTile; ++lx) {
                const uint32_t px = tx * kTile + lx, py = ty * kTile + ly;
                if (px >= W || py >= H) continue;
                const size_t at = (size_t)py * W + px;
                FrozenPixel& fp = frozen[at];
                double T = 1.0;
                for (uint32_t s : fr.lists[t]) {
                    const Rec64& r = fr.recs[s];
                    if (!r.live) continue;
                    const double dx = px + 0.5 - r.cx, dy = py + 0.5 - r.cy;
                    const double power = r.a * dx * dx + 2.0 * r.b * dx * dy + r.c * dy * dy;
                    if (power > r.cutoff) continue;
                    const double alpha = std::min(0.99, r.alpha * std::exp(-0.5 * power));
                    if (alpha < 1.0 / 255.0) continue;
                    fp.slots.push_back(s);
                    T *= 1.0 - alpha;
                    if (T < 1e-4) break;
                }
                double c[3];
                pixelColourWith(*f, fp, fr.recs, px, py, ~0u, nullptr, c);
                for (int k = 0; k < 3; ++k) {
                    base[at * 3 + k] = c[k];
                    const double e = c[k] - target[at * 3 + k];
                    loss += e * e * scale;
                }
            }
    }
    if (lossOut) *lossOut = loss;
    // the pixels each perturbed Gaussian reaches
    std::vector<std::vector<uint32_t>> reach(nWhich);
    {
        std::vector<int64_t> index(count, -1);
        for (uint32_t k = 0; k < nWhich; ++k) index[which[k]] = k;
        for (size_t at = 0; at < frozen.size(); ++at)
            for (uint32_t s : frozen[at].slots)
                if (index[s] >= 0) reach[index[s]].push_back((uint32_t)at);
    }
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads > 0 ? threads : omp_get_max_threads())
    for (int64_t kk = 0; kk < (int64_t)nWhich; ++kk) {
        const uint32_t g = which[kk];
        for (int j = 0; j < kParamsPerGaussian; ++j) {
            double d[2] = {0.0, 0.0};
            for (int sgn = 0; sgn < 2; ++sgn) {
                Rec64 rec = project64(*f, gaussOf(P, g, j, sgn == 0 ? eps : -eps), 1.0);
                double delta = 0.0;
                for (uint32_t at : reach[kk]) {
                    double c[3];
                    pixelColourWith(*f, frozen[at], fr.recs, at % W, at / W, g, &rec, c);
                    for (int k = 0; k < 3; ++k) {
                        const double e1 = c[k] - target[(size_t)at * 3 + k];
                        const double e0 = base[(size_t)at * 3 + k] - target[(size_t)at * 3 + k];
                        delta += (e1 * e1 - e0 * e0) * scale;
                    }
                }
                d[sgn] = delta;
            }
            out[(size_t)kk * kParamsPerGaussian + j] = (d[0] - d[1]) / (2.0 * eps);
        }
    }
}
