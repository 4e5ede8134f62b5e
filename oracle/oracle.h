/*
 * ORACLE -- TEST INFRASTRUCTURE ONLY.
 *
 * A CPU restatement of athenea's Gaussian-splat tile rasteriser (the plain
 * path of render::TileRasterizer and the Slang kernels it dispatches), written
 * from the reference's shader sources and used as the checker for the CUDA
 * product. Nothing in the product links, loads or calls this code: only
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg do.
 *
 * Parity status: the reference cannot run here (it needs Slang, slang-rhi and a
 * GPU). The restatement is pinned against the reference's own known-answer
 * tests (tests/render/test_splat_render.cpp:130-206, :1831-1917,
 * tests/scene/test_loading.cpp:91-166, tests/gpu/test_algo.cpp:347-379), which
 * the test suite re-runs against it. Bit-level parity with the Slang build is
 * unpinned where Slang maps exp/log/pow to a vendor library: this restatement
 * uses its own exp/log (Cody-Waite reduction, Taylor and atanh series), and so
 * does the product, which is what makes keys, rects, counts, ranges and images
 * comparable bit for bit between the two.
 *
 * Arithmetic rules (so the CUDA side can reproduce every bit): IEEE float32,
 * no contraction of a*b+c into fma (built with -ffp-contract=off), expressions
 * evaluated left to right exactly as the Slang source writes them.
 */
#ifndef ATHENEA_ORACLE_H
#define ATHENEA_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* common/edit.slang:23-36 (EditParams). */
typedef struct {
    uint32_t active, shape, mode, invert;
    float centre[3];
    float size[3];
    float tint[3];
    float saturation, brightness, opacity, minOpacity, maxScale;
} orc_edit;

/* The subset of splat/frame.slang:51-230 (FrameParams) the plain path reads,
 * as setFrame/setObject/setCloudSpace fill it (modules/render/src/FrameParams.h:32-117). */
typedef struct {
    uint32_t width, height, tilesX, tilesY;
    float focalX, focalY, centreX, centreY, nearZ, farZ;
    uint32_t orthographic, antialias;
    float paidAt;
    uint32_t surfels;
    float m[12];      /* object -> view, rows of a 3x4 */
    float eye[3];     /* the camera in the cloud's own space */
    uint32_t restPerColour, shWords, shLimit, linearCloud;
    uint32_t depthMode;
    float depthThreshold;
    float bg[4];
    orc_edit edit;
    uint32_t tile;    /* tile size: 16 (frame.slang:34) unless orc_frame_set_tile changed it */
} orc_frame;

/* 3DGS record layout (io::SplatEncoding) for the decode. Field indices into a
 * record of `stride` floats; rest coefficients colour-outer (r..., g..., b...). */
typedef struct {
    uint32_t stride;
    uint32_t x, y, z, opacity, scale0, scale1, scale2, rotW, rotX, rotY, rotZ, dc0, dc1, dc2;
    uint32_t restBase, filePerColour, keepPerColour;
} orc_encoding;

/* ---- scalar helpers the product must agree with (exposed for unit tests) ---- */
float orc_exp(float x);
float orc_log(float x);
float orc_pow(float x, float y);
uint16_t orc_f32_to_f16(float v);
float orc_f16_to_f32(uint16_t h);
uint32_t orc_encode_quaternion(const float q[4]);
void orc_decode_quaternion(uint32_t word, float q[4]);

/* ---- decode: scene/splat_validate.slang + scene/splat_decode.slang ----
 * Records that fail validation are dropped and the rest compacted in file
 * order. Returns the number kept. shWords = keep == 0 ? 1 : (3 keep + 1) / 2. */
uint32_t orc_decode(const float* records, uint32_t count, const orc_encoding* e, float* positions,
                    uint32_t* shape, uint32_t* sh, uint32_t* origin);

/* ---- camera: modules/render/src/Camera.cpp:9-64 (double precision) ---- */
typedef struct {
    double cameraToWorld[16]; /* row-major, column vectors (p' = M p) */
    uint32_t orthographic;
    double focal, haperture, nearZ, farZ;
    double windowTranslate[2], windowScale[2], windowRoll;
} orc_camera;

typedef struct {
    double worldToView[16];
    double focalX, focalY, centreX, centreY, nearZ, farZ;
    uint32_t orthographic;
    double eyeWorld[3];
} orc_projection;

void orc_camera_looking_at(const double eye[3], const double target[3], const double up[3], orc_camera* out);
void orc_projection_for(const orc_camera* camera, uint32_t width, uint32_t height, orc_projection* out);
/* setFrame + setObject + setCloudSpace for one instance (FrameParams.h:32-117;
 * TileRasterizer.cpp:599-601). antialiased: -1 when the cloud's file says nothing. */
void orc_frame_for(const orc_projection* p, const double objectToWorld[16], uint32_t width, uint32_t height,
                   uint32_t antialias, int32_t antialiased, float madeSpread, uint32_t surfels,
                   uint32_t maxShDegree, uint32_t restPerColour, uint32_t shWords, uint32_t linearCloud,
                   const float bg[4], uint32_t depthMode, float depthThreshold, const orc_edit* edit,
                   orc_frame* out);

/* ---- (a) projection: splat/splat_project.slang:497-785,1080-1129 (projectSplat<0>) ----
 * Per slot base+i: record (12 floats: screen xyzw, conic xyzw, colour rgb + mark),
 * tile rect (4), tiles touched, depth key (or 0xFF000000 | cull reason), visible. */
void orc_project(const orc_frame* f, uint32_t count, uint32_t base, const float* positions,
                 const uint32_t* shape, const uint32_t* sh, float* records, uint32_t* rects,
                 uint32_t* touched, uint32_t* depthKeys, uint32_t* visible, int threads);

/* The same projection from FP32 training parameters: means float4 (xyz, opacity
 * logit), scales float4 (log scales), quats float4 (w x y z, any length), sh
 * shStride floats (DC rgb, then rest rgb per basis). Decoded as an upload
 * would: sigmoid, exp, normalise, 0.5 + SH0 * DC. */
void orc_project_params(const orc_frame* f, uint32_t count, uint32_t base, const float* means, const float* scales,
                        const float* quats, const float* sh, uint32_t shStride, float* records, uint32_t* rects,
                        uint32_t* touched, uint32_t* depthKeys, uint32_t* visible, int threads);

/* ---- (b)+(c) binning, the reference's two-sort form (TileRasterizer.cpp:1088-1176):
 * compact -> stable 24-bit depth sort -> gather -> scan -> emit -> stable tile sort -> ranges.
 * pairTiles/pairSplats need `pairs` entries (the sum of touched); ranges 2 per tile.
 * Returns the number of pairs written. */
uint64_t orc_bin(const orc_frame* f, uint32_t slots, const float* records, const uint32_t* rects,
                 const uint32_t* touched, const uint32_t* depthKeys, const uint32_t* visible,
                 uint32_t* pairTiles, uint32_t* pairSplats, uint32_t* ranges, uint32_t* visibleCount);

/* The frame at another tile size (the batched path bins at 8, 16 or 32): the
 * tile rects, the tile test (frame.slang:374-402), the tile count and the
 * blends' tiles all follow it. */
void orc_frame_set_tile(orc_frame* f, uint32_t tile);

/* orc_bin writing only the pairs of tiles t with t % tileStride == tileOffset
 * (each such tile's pairs in the order orc_bin gives them): a sampled check of
 * a frame too large to bin whole. Returns the pairs written; ranges cover every tile.
 * With pairTiles NULL it only counts them (nothing else is written). */
uint64_t orc_bin_sampled(const orc_frame* f, uint32_t slots, const float* records, const uint32_t* rects,
                         const uint32_t* touched, const uint32_t* depthKeys, const uint32_t* visible,
                         uint32_t* pairTiles, uint32_t* pairSplats, uint32_t* ranges, uint32_t tileStride,
                         uint32_t tileOffset);

/* ---- (d) blend: splat/splat_blend.slang:236-578 (blendPixel<false,false,false>) ----
 * colour float4 and depth per pixel, bottom row first. finalT / lastContrib
 * (optional, may be NULL): the transmittance the walk ended with and one past
 * the index into the tile's pair range of the last record blended (0: none).
 * Returns the number of (pixel, record) evaluations the walks made. */
uint64_t orc_blend(const orc_frame* f, const uint32_t* ranges, const uint32_t* pairSplats,
                   const float* records, float* colour, float* depth, float* finalT, uint32_t* lastContrib,
                   int threads);

/* orc_blend over an opaque layer under the splats (TileRasterizer::render's
 * `under`, splat_blend.slang's composite path without points): underColour
 * float4 and underDepth float a pixel; a pixel whose underDepth > 0 stops its
 * walk at the first record at or behind that depth and takes the layer's
 * colour and depth behind what it blended. */
/* The Cryptomatte of a frame (splat_blend.slang's matte path): cryptoIds a
 * uint a slot; crypto 3 x pixels float4 out. underDepth / underCrypto may be
 * null (no under layer). */
void orc_blend_matte(const orc_frame* f, const uint32_t* ranges, const uint32_t* pairSplats, const float* records,
                     const uint32_t* cryptoIds, const float* underDepth, const uint32_t* underCrypto, float* crypto,
                     int threads);

void orc_blend_over(const orc_frame* f, const uint32_t* ranges, const uint32_t* pairSplats, const float* records,
                    const float* underColour, const float* underDepth, float* colour, float* depth, int threads);

/* contributionMode 4 (splat_blend.slang:381-398): per slot four signed words,
 * weight * dLdPixel.rgb in 1/256 with hash-dithered rounding, and the weight. */
void orc_colour_gradient(const orc_frame* f, const uint32_t* ranges, const uint32_t* pairSplats,
                         const float* records, const float* dLdPixel, int32_t* contribution);

/* The same sums unquantised, in double: gradient[slot*3 + c] = sum of weight * dLdPixel. */
void orc_colour_gradient_exact(const orc_frame* f, const uint32_t* ranges, const uint32_t* pairSplats,
                               const float* records, const float* dLdPixel, double* gradient);

/* contributionMode 1: the weight each slot blended with, in 1/4096 of a pixel. */
void orc_contribution_weight(const orc_frame* f, const uint32_t* ranges, const uint32_t* pairSplats,
                             const float* records, uint32_t* contribution);

/* contributionMode 2 (splat_blend.slang:366-380): per slot the squared colour
 * change taking it away would leave in each pixel, capped at one, in 2^-24,
 * against `wholeFrame` (float4 a pixel), added as a 64-bit sum into two words
 * (low, high). */
void orc_contribution_change(const orc_frame* f, const uint32_t* ranges, const uint32_t* pairSplats,
                             const float* records, const float* wholeFrame, uint32_t* contribution);

/* contributionMode 3 (splat_blend.slang:399-407): per slot two words, the
 * weight times liftMask (clamped to [0, 1]) and the weight, in 1/1024. */
void orc_contribution_lift(const orc_frame* f, const uint32_t* ranges, const uint32_t* pairSplats,
                           const float* records, const float* liftMask, uint32_t* contribution);

/* The matte summed by the blend (splat_blend.slang:423-435,536-539) from a
 * lift's two words a slot (weight x mask, weight): one float a pixel. */
void orc_matte_lift(const orc_frame* f, const uint32_t* ranges, const uint32_t* pairSplats, const float* records,
                    const uint32_t* liftSums, uint32_t hard, float threshold, float* matte);

/* The trace (splat_trace.slang): 11 planes of width*height words, as the
 * product writes them, for a frame with no layer under the splats. */
void orc_trace(const orc_frame* f, const uint32_t* ranges, const uint32_t* pairSplats, const float* records,
               uint32_t* trace);

/* P: usd/aov_position.slang:34-52; viewToWorld rows (3x4, float). */
void orc_position(uint32_t width, uint32_t height, uint32_t orthographic, float focalX, float focalY,
                  float centreX, float centreY, const float viewToWorld[12], const float* depth,
                  float* position);

/* ---- FP64 oracle ----
 * The same plain path evaluated in double from the same packed inputs (fp16
 * fields widened exactly), binned with the exact tile test, sorted per tile by
 * (view depth, slot) -- reference/reference_blend.slang's order -- and blended
 * in double. `near` (optional) receives, per pixel, 1 where a blend decision
 * (cutoff, 1/255, T < 1e-4) of some record lies within `margin` relative of
 * its threshold: a pixel where float rounding may legitimately decide
 * otherwise. One instance per call, as the FP32 path's orc_project. */
typedef struct {
    double focalX, focalY, centreX, centreY, nearZ, farZ;
    uint32_t width, height, orthographic, antialias;
    double paidAt;
    double m[12];
    double eye[3];
    uint32_t restPerColour, shWords, shLimit, linearCloud;
    double bg[4];
} orc_frame64;

void orc_frame64_from(const orc_projection* p, const double objectToWorld[16], uint32_t width, uint32_t height,
                      uint32_t antialias, uint32_t maxShDegree, uint32_t restPerColour, uint32_t shWords,
                      uint32_t linearCloud, const double bg[4], orc_frame64* out);

/* Renders `count` splats; only pixels whose tile index satisfies
 * tile % tileStride == tileOffset are written (a sampled check at scale);
 * others are left as they are. */
void orc_render_f64(const orc_frame64* f, uint32_t count, const float* positions, const uint32_t* shape,
                    const uint32_t* sh, double* colour, double* depth, uint8_t* nearDecision, double margin,
                    uint32_t tileStride, uint32_t tileOffset, int threads);

/* The same FP64 path from FP32 training parameters (means, log-scales,
 * quaternion wxyz unnormalised, opacity logit, 48 SH floats a splat rgb per
 * basis with the DC first): the function the gradients are checked against. */
void orc_render_params_f64(const orc_frame64* f, uint32_t count, const double* means, const double* logScales,
                           const double* quats, const double* logits, const double* shs, uint32_t shDegree,
                           double* colour, double* depth, int threads);

/* orc_render_params_f64 from the FP32 training layout as the GPU holds it
 * (means x y z logit, log scales, quaternion w x y z, each 4 floats a splat; SH
 * rows of `shStride` floats), with orc_render_f64's near-decision flags and
 * tile sampling: the image-error check of the mixed-precision path at scale. */
void orc_render_params_sampled_f64(const orc_frame64* f, uint32_t count, const float* means, const float* scales,
                                   const float* quats, const float* sh, uint32_t shStride, uint32_t shDegree,
                                   double* colour, double* depth, uint8_t* nearDecision, double margin,
                                   uint32_t tileStride, uint32_t tileOffset, int threads);

/* Central finite differences (step eps) of L = mean over pixels and r g b of
 * (colour - target)^2, in double, for the Gaussians `which`: out[k*59 + j] for
 * parameter j of which[k] in the order means x y z, logit, log scales x y z,
 * quat w x y z, sh[48]. The blend's decisions (which records each pixel blends
 * and where its walk stops) are frozen at the base parameters. target: float3
 * a pixel. *lossOut receives L at the base. */
void orc_fd_gradients_f64(const orc_frame64* f, uint32_t count, const double* means, const double* logScales,
                          const double* quats, const double* logits, const double* shs, uint32_t shDegree,
                          const float* target, const uint32_t* which, uint32_t nWhich, double eps, double* out,
                          double* lossOut, int threads);

#ifdef __cplusplus
}
#endif

#endif
