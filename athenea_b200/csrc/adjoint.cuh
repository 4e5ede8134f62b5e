// The projection's adjoint (splat/splat_project.slang:497-785 differentiated):
// dL/d(record) -> dL/d(parameters) for the FP32 training and the mixed layouts.
// Shared by the one-view backward (backward.cu) and the batched one (batch.cu).
#pragma once

#include <cstdint>

#include "gauss.cuh"
#include "raster_types.cuh"
#include "splat_math.cuh"

namespace ath {

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

// dL/dparameters of one Gaussian, kept in registers so a caller can sum it over views.
struct ParamGrad {
    float dp[3];        // means
    float dLogit;
    float dLogScale[3];
    float dQuat[4];     // w x y z
    float dSh[48];      // DC rgb, then the rest rgb per basis

    __device__ __forceinline__ void clear() {
#pragma unroll
        for (int k = 0; k < 3; ++k) dp[k] = dLogScale[k] = 0.0f;
        dLogit = 0.0f;
#pragma unroll
        for (int k = 0; k < 4; ++k) dQuat[k] = 0.0f;
#pragma unroll
        for (int k = 0; k < 48; ++k) dSh[k] = 0.0f;
    }

    // Added into the gradient arrays (ath_param_grads' layout).
    __device__ __forceinline__ void addTo(uint32_t i, uint32_t shStride, float4* gMeans, float4* gScales, float4* gQuats,
                                          float* gSh, bool overwrite = false) const {
        float4 m = overwrite ? make_float4(0, 0, 0, 0) : gMeans[i];
        m.x += dp[0]; m.y += dp[1]; m.z += dp[2]; m.w += dLogit;
        gMeans[i] = m;
        float4 s = overwrite ? make_float4(0, 0, 0, 0) : gScales[i];
        s.x += dLogScale[0]; s.y += dLogScale[1]; s.z += dLogScale[2];
        gScales[i] = s;
        float4 q = overwrite ? make_float4(0, 0, 0, 0) : gQuats[i];
        q.x += dQuat[0]; q.y += dQuat[1]; q.z += dQuat[2]; q.w += dQuat[3];
        gQuats[i] = q;
        float* row = gSh + (size_t)i * shStride;
        const uint32_t n = shStride < 48 ? shStride : 48;
#pragma unroll
        for (uint32_t k = 0; k < 48; ++k)
            if (k < n) row[k] = (overwrite ? 0.0f : row[k]) + dSh[k];
    }
};

// The projection's adjoint past the colour, for one Gaussian and one view, up
// to the covariance's factor M = R diag(s): dL/d(record) `gw` -> dL/d(position,
// opacity logit) into `acc`, and dL/dM into `dM`. `G` is projectGeometry's
// result for (F, I, g); `dp` holds what the colour's adjoint gave the position
// and ends, with the geometry's share, in `acc`. dL/dM is linear in the views,
// so a caller that sums it over views takes it to the scales and the
// quaternion once (shapeAdjoint).
__device__ __forceinline__ void geometryAdjointToM(const FrameConst& F, const InstanceConst& I, const Gauss& g,
                                                   const Geometry& G, const float gw[kGradWords], float dp[3],
                                                   ParamGrad& acc, float dM[3][3]) {
    const float* m = I.m;
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
    float da2, db, dc2;
    if (G.wide) {
        // the mixed path's FP64 conic (gauss.cuh wideCovariance), differentiated in FP64
        const WideCovariance W = wideCovariance(G.t3, G.u3, G.M);
        const double d2 = W.det * W.det;
        da2 = (float)(gA * (-W.c2 * W.c2 / d2) + gB * (W.b * W.c2 / d2) + gC * (1.0 / W.det - W.a2 * W.c2 / d2));
        db = (float)(gA * (2.0 * W.b * W.c2 / d2) + gB * (-1.0 / W.det - 2.0 * W.b * W.b / d2) +
                     gC * (2.0 * W.a2 * W.b / d2));
        dc2 = (float)(gA * (1.0 / W.det - W.c2 * W.a2 / d2) + gB * (W.b * W.a2 / d2) + gC * (-W.a2 * W.a2 / d2));
    } else {
        da2 = gA * (-c2 * c2 / det2) + gB * (b * c2 / det2) + gC * (1.0f / det - a2 * c2 / det2);
        db = gA * (2.0f * b * c2 / det2) + gB * (-1.0f / det - 2.0f * b * b / det2) + gC * (2.0f * a2 * b / det2);
        dc2 = gA * (1.0f / det - c2 * a2 / det2) + gB * (b * a2 / det2) + gC * (-a2 * a2 / det2);
    }
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
    float dt3[3], du3[3];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        dt3[r] = G.M[r][0] * dax[0] + G.M[r][1] * dax[1] + G.M[r][2] * dax[2];
        du3[r] = G.M[r][0] * day[0] + G.M[r][1] * day[1] + G.M[r][2] * day[2];
#pragma unroll
        for (int col = 0; col < 3; ++col) dM[r][col] = G.t3[r] * dax[col] + G.u3[r] * day[col];
    }

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

    acc.dp[0] += dp[0]; acc.dp[1] += dp[1]; acc.dp[2] += dp[2];
    acc.dLogit += dLogit;
}

// dL/dM (M = R diag(s), R the rotation projectGeometry builds from g.q) ->
// dL/d(log scales, raw quaternion), added into `acc`.
__device__ __forceinline__ void shapeAdjoint(const InstanceConst& I, uint32_t i, const Gauss& g, const float R[3][3],
                                             const float dM[3][3], ParamGrad& acc) {
    float dScale[3] = {0.0f, 0.0f, 0.0f}, dR[3][3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int col = 0; col < 3; ++col) {
            dScale[col] += dM[r][col] * R[r][col];
            dR[r][col] = dM[r][col] * g.scale[col];
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

#pragma unroll
    for (int k = 0; k < 3; ++k) acc.dLogScale[k] += dScale[k] * g.scale[k];
    acc.dQuat[0] += dQuat.x; acc.dQuat[1] += dQuat.y; acc.dQuat[2] += dQuat.z; acc.dQuat[3] += dQuat.w;
}

// The projection's adjoint past the colour, for one Gaussian and one view:
// dL/d(record) `gw` -> dL/d(position, opacity logit, log scales, quaternion).
template <uint32_t L>
__device__ __forceinline__ void geometryAdjoint(const FrameConst& F, const InstanceConst& I, uint32_t i, const Gauss& g,
                                                const Geometry& G, const float gw[kGradWords], float dp[3],
                                                ParamGrad& acc) {
    float dM[3][3];
    geometryAdjointToM(F, I, g, G, gw, dp, acc, dM);
    shapeAdjoint(I, i, g, G.R, dM, acc);
}

// The projection's adjoint for one Gaussian and one view: dL/d(record) `gw`
// (gradient words of raster_types.cuh) -> dL/dparameters, added into `acc`.
template <uint32_t L>
__device__ __forceinline__ void projectAdjoint(const FrameConst& F, const InstanceConst& I, uint32_t i,
                                               const float gw[kGradWords], ParamGrad& acc) {
    const Gauss g = loadGauss<L>(I, i);
    const Geometry G = projectGeometry<L == kLayoutMixed>(F, I, g, g.opacity);

    // ---- colour: c = decode(base + rest(dir)) ------------------------------
    float dp[3] = {0.0f, 0.0f, 0.0f};
    const uint32_t degree = min(degreeOf(I.restPerColour), F.shLimit);
    const float ex = g.px - I.eye[0], ey = g.py - I.eye[1], ez = g.pz - I.eye[2];
    const float len = sqrtf((ex * ex + ey * ey) + ez * ez);
    const float dir[3] = {ex / len, ey / len, ez / len};
    float Y[15], dY[15][3];
    shBasis(degree, dir[0], dir[1], dir[2], Y, dY);
    const uint32_t bases = degree == 3 ? 15 : degree == 2 ? 8 : degree == 1 ? 3 : 0;
    float dDir[3] = {0.0f, 0.0f, 0.0f};
    const float gc[3] = {gw[kGradR], gw[kGradG], gw[kGradB]};
#pragma unroll
    for (int ch = 0; ch < 3; ++ch) {
        float v = g.base[ch];
#pragma unroll
        for (uint32_t k = 0; k < 15; ++k)
            if (k < bases) v += Y[k] * restAt<L>(I, i, k * 3 + (uint32_t)ch);
        float dcdv;
        if (I.linear != 0) {
            dcdv = v > 0.0f ? 1.0f : 0.0f;
        } else {
            dcdv = v <= 0.0f ? 0.0f : v <= 0.04045f ? 1.0f / 12.92f : (2.4f / 1.055f) * pow_f((v + 0.055f) / 1.055f, 1.4f);
        }
        const float dv = gc[ch] * dcdv;
        acc.dSh[ch] += kSH0 * dv;
#pragma unroll
        for (uint32_t k = 0; k < 15; ++k) {
            if (k >= bases) continue;
            acc.dSh[3 + k * 3 + ch] += Y[k] * dv;
            const float coef = restAt<L>(I, i, k * 3 + (uint32_t)ch) * dv;
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

    geometryAdjoint<L>(F, I, i, g, G, gw, dp, acc);
}


}   // namespace ath
