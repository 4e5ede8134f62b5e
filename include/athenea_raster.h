/*
 * athenea-b200: the Gaussian-splat tile rasteriser of athenea, for B200
 * (sm_100a), behind a C ABI.
 *
 * Each entry point replaces one member of the reference's
 * render::TileRasterizer (modules/render/include/athenea/render/TileRasterizer.h)
 * or of the camera helpers it is driven by (modules/render/src/Camera.cpp); the
 * comment above each names the interface and file:line it stands in for.
 *
 * Conventions (the reference's, splat/frame.slang:22-30): view +z forward, x
 * right, y up; images bottom row first; pixel centres at +0.5; colour is
 * premultiplied linear RGBA.
 *
 * Memory: every pointer a caller passes that a kernel reads or writes is device
 * memory the caller owns (GpuSplats and RenderTargets are the caller's in the
 * reference too). The rasteriser owns its scratch, grows it by half again when
 * a frame needs more (TileRasterizer.cpp:30-36) and gives it back on
 * ath_raster_release_scratch (:178-191).
 *
 * Errors: every function returns an ath_status; the message of the last failure
 * on the calling thread is ath_last_error_message(). Nothing throws across the
 * ABI. A handle is one camera's frame at a time and is not re-entrant
 * (TileRasterizer.h:316-317): use one handle per thread or stream.
 */
#ifndef ATHENEA_RASTER_H
#define ATHENEA_RASTER_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* core/Error.h:14-26 (ErrorCode), in its order, after ATH_OK; plus ATH_E_TIMEOUT
 * for a bounded device wait that gave up (the sort's look-back) and
 * ATH_E_CAPACITY for a frame or step whose pairs outgrew the pair buffers'
 * capacity (it is not valid; the next one grows them). */
typedef enum {
    ATH_OK = 0,
    ATH_E_UNKNOWN = 1,
    ATH_E_NOT_FOUND = 2,
    ATH_E_INVALID_ARGUMENT = 3,
    ATH_E_UNSUPPORTED = 4,
    ATH_E_IO_FAILURE = 5,
    ATH_E_DEVICE_FAILURE = 6,
    ATH_E_SHADER_FAILURE = 7,
    ATH_E_PLUGIN_FAILURE = 8,
    ATH_E_OUT_OF_MEMORY = 9,
    ATH_E_CANCELLED = 10,
    ATH_E_INTERNAL = 11,
    ATH_E_TIMEOUT = 12,
    ATH_E_CAPACITY = 13
} ath_status;

typedef struct ath_raster ath_raster;

/* Camera.h:89-117 (Lens) and :119-126 (Camera). Matrices are row-major 4x4
 * acting on column vectors (p' = M p). */
typedef struct {
    double camera_to_world[16];
    int32_t orthographic;
    double focal;             /* mm */
    double haperture;         /* mm */
    double near_z, far_z;
    double window_translate[2];
    double window_scale[2];
    double window_roll;       /* degrees, counter-clockwise */
} ath_camera;

/* Camera.h:129-155 (Projection): what the kernels need of a camera for one image size. */
typedef struct {
    double world_to_view[16]; /* +z forward */
    double focal_x, focal_y;  /* pixels per unit of x/z (perspective) or per world unit (ortho) */
    double centre_x, centre_y;
    double near_z, far_z;
    int32_t orthographic;
    double eye_world[3];
} ath_projection;

/* TileRasterizer.h:38-60 (SplatEdit); common/edit.slang. */
typedef struct {
    int32_t active;
    uint32_t shape;           /* 0 box, 1 sphere */
    uint32_t mode;            /* 0 keep inside, 1 remove inside, 2 grade inside */
    int32_t invert;
    float centre[3], size[3], tint[3];
    float saturation, brightness, opacity, min_opacity, max_scale;
} ath_edit;

/* scene::GpuSplats (scene/GpuClouds.h:44-52) with SplatInstance
 * (TileRasterizer.h:85-172): device pointers in the reference's packed layout
 * (common/packing.slang:5-27):
 *   positions  float4 a splat: xyz, opacity
 *   shape      uint4 a splat:  [0] 10-bit smallest-three quaternion, [1] f16 ln sx | ln sy,
 *                              [2] f16 ln sz | base r, [3] base g | base b
 *   sh         sh_words uint a splat: f16 rest coefficients, rgb per basis */
typedef struct {
    const float* positions;
    const uint32_t* shape;
    const uint32_t* sh;
    uint32_t count;
    uint32_t rest_per_colour;  /* 0, 3, 8 or 15 */
    uint32_t sh_words;         /* rest_per_colour == 0 ? 1 : (3 rest_per_colour + 1) / 2 */
    int32_t linear;            /* 1: colours are linear light; 0: sRGB, decoded per splat */
    int32_t antialiased;       /* what the cloud's file said: -1 nothing, 0 no, 1 yes */
    double object_to_world[16];
    ath_edit edit;
} ath_instance;

/* The plain-path subset of RenderSettings (TileRasterizer.h:248-371). */
typedef struct {
    uint32_t width, height;
    int32_t antialias;          /* default 1 */
    int32_t antialias_override; /* -1 none, else 0/1 */
    float made_spread;
    int32_t surfels;            /* default 1 */
    uint32_t max_sh_degree;     /* default 3 */
    float background[4];        /* premultiplied linear */
    uint32_t depth_mode;        /* 0 alpha-weighted mean, 1 first threshold crossing */
    float depth_threshold;      /* default 0.5 */
    int32_t time_stages;        /* wait after each stage and fill the *_ms stats */
    int32_t count_splats;       /* count culls by reason and clouds (ath_raster_latest_counters); does not wait */
    uint64_t counters_tag;
    /* What each splat gave the frame, added into `contribution` (device memory,
     * never cleared here, so frames from many cameras sum into it), in the
     * reference's contributionMode (TileRasterizer.h:351-367,
     * splat_blend.slang:364-407): 0 nothing; 1 a uint a slot, the transmittance
     * times alpha it blended with summed over its pixels, in 1/4096; 2 two
     * uint a slot (low, then high word of one 64-bit sum), the squared colour
     * change taking the splat away would leave in each pixel, capped at one, in
     * 2^-24, against `final_colour`, the frame drawn whole from the same camera
     * (float4 a pixel, as the colour target holds it); 3 two uint a slot, the
     * weight times `lift_mask` (one float a pixel, 0 to 1) and the weight, in
     * 1/1024; 4 four words a slot, three signed (the weight times
     * `final_colour`, here a loss's derivative at each pixel, float4 a pixel,
     * summed in 1/256 with hash-dithered rounding) and the weight in 1/256.
     * Slots are the instances' splats one after another. */
    uint32_t contribution_mode;
    uint32_t* contribution;
    const float* final_colour;
    /* Cryptomatte (splat_blend.slang:29-35,88-143,420-421,525-534): with
     * crypto_ids (a uint id a slot; 0 names nothing) and crypto (3 x width x
     * height float4, layer-major), each pixel keeps the 6 ids that covered it
     * most, ranked by coverage (weight summed a id) and written as (id bits as
     * float, coverage, id, coverage). under_crypto, optional, is the under
     * layer's id a pixel (ath_raster_render_over). */
    const uint32_t* crypto_ids;
    float* crypto;
    const uint32_t* under_crypto;
    const float* lift_mask;     /* contribution mode 3's mask: one float a pixel, 0 to 1 */
    /* The matte summed by the blend (TileRasterizer.h:319-326, splat_blend.slang:
     * 423-435,536-539): with matte_lift (two uint a slot, as contribution mode 3
     * wrote them: the weight times a mask and the weight) and matte (one float a
     * pixel), each blended splat that a lift saw adds its weight times its share
     * (inside / seen; 1 above matte_threshold and 0 below when matte_hard), one
     * it did not is counted at the pixel's known share, and the pixel's matte is
     * that sum clamped to [0, 1]. matte_threshold defaults to 0.5. */
    const uint32_t* matte_lift;
    float* matte;
    int32_t matte_hard;
    float matte_threshold;
    /* The trace (TileRasterizer.h:282-288, splat/splat_trace.slang): the four
     * splats that weighed most in each pixel, 11 planes of width*height uint:
     * their slots heaviest first (0xFFFFFFFF where a rank is empty), their view
     * depths as float bits, their weights as halves two a word, and the weight
     * the list had no room for with what closed the walk from behind (the under
     * layer) as halves; a pixel nothing reached has 0xFFFFFFFE in its first word
     * and nothing else written. NULL: no trace. */
    uint32_t* trace;
} ath_settings;

/* RenderTargets (TileRasterizer.h:421-450) plus the P layer
 * (usd/aov_position.slang): caller-owned device buffers of width*height,
 * bottom row first. position may be NULL. */
typedef struct {
    uint32_t width, height;
    float* colour;    /* float4, premultiplied linear */
    float* depth;     /* float, view z */
    float* position;  /* float4 world xyz, 1 (zeros where nothing drew); optional */
} ath_targets;

/* FrameStats (TileRasterizer.h:408-419). */
typedef struct {
    uint32_t splats, visible, pairs;
    double project_ms, counts_ms, depth_sort_ms, emit_ms, tile_sort_ms, blend_ms, total_ms;
} ath_frame_stats;

/* SplatCounters::Cloud (TileRasterizer.h:396-399): one instance's share. */
typedef struct {
    uint32_t visible, pairs;
} ath_cloud_counts;

/* SplatCounters (TileRasterizer.h:373-401); culled[] in splat/frame.slang:42-49's
 * numbering. clouds[] holds the first cloud_count instances of the counted frame,
 * in the order it was given them (at most 64, SplatCounters::kMaxClouds); later
 * instances are only in the totals. */
typedef struct {
    uint64_t tag;
    uint32_t slots, visible, pairs, max_tiles;
    uint32_t culled[7];
    uint32_t cloud_count;
    ath_cloud_counts clouds[64];
} ath_splat_counters;

/* ---- camera helpers ----------------------------------------------------- */

/* Camera::lookingAt (Camera.cpp:9-25). up may be NULL for +Y. */
ath_status ath_camera_looking_at(const double eye[3], const double target[3], const double up[3], ath_camera* out);
/* A camera with the reference's defaults (Camera.h:89-121): at the origin, looking down -Z. */
ath_status ath_camera_default(ath_camera* out);
/* projectionFor (Camera.cpp:32-64). */
ath_status ath_projection_for(const ath_camera* camera, uint32_t width, uint32_t height, ath_projection* out);
/* RenderSettings' defaults (TileRasterizer.h:248-371). */
ath_status ath_settings_default(ath_settings* out);

/* ---- the rasteriser ------------------------------------------------------ */

/* TileRasterizer::create (TileRasterizer.h:454). Binds the current CUDA device. */
ath_status ath_raster_create(ath_raster** out);
/* ~TileRasterizer: frees the scratch; the handle is gone. */
void ath_raster_destroy(ath_raster* r);
/* TileRasterizer::releaseScratch (TileRasterizer.h:482; TileRasterizer.cpp:178-191). */
ath_status ath_raster_release_scratch(ath_raster* r);

/* TileRasterizer::render(const Projection&, span<const SplatInstance>,
 * const RenderSettings&, RenderTargets&) (TileRasterizer.h:468-474;
 * TileRasterizer.cpp:296-1295). Enqueued on `stream` (a cudaStream_t; NULL:
 * the legacy default stream) with nothing read back and no wait, where the
 * reference waits once mid-frame for its visible and pair totals
 * (TileRasterizer.cpp:1093-1102): the pairs are sized from a capacity the
 * handle keeps, and the sort, ranges and blend take the pair count from the
 * device. The one exception is a handle's first frame (and its first after
 * ath_raster_release_scratch), which reads the pair total back once to size
 * that capacity. A frame whose pairs outgrow the capacity is not valid:
 * ath_raster_check reports it as ATH_E_CAPACITY, and the next frame grows the
 * capacity (to what the last finished frame needed). `stats`: splats always;
 * visible and pairs when the frame read them back (the sizing frame, or
 * time_stages, whose frame waits for its end and returns its own status),
 * else 0 -- ath_raster_check gives them. count_splats does not wait: the
 * counters come back through ath_raster_latest_counters. Targets must be
 * width x height of `settings`. */
ath_status ath_raster_render(ath_raster* r, const ath_projection* projection, const ath_instance* instances,
                             uint32_t instance_count, const ath_settings* settings, ath_targets* targets,
                             ath_frame_stats* stats, void* stream);

/* TileRasterizer::render with its `under` layer (TileRasterizer.h:468-474;
 * splat_blend.slang:249-251,329-333,516-523,555-575): the splats composited
 * over an opaque layer of the frame's size (colour float4, depth float a pixel,
 * depth 0 where it has nothing). A pixel's walk stops at the first splat at or
 * behind the layer; the layer takes what light is left, and the pixel's depth
 * and coverage count it. A layer of another size is ATH_E_INVALID_ARGUMENT. */
ath_status ath_raster_render_over(ath_raster* r, const ath_projection* projection, const ath_instance* instances,
                                  uint32_t instance_count, const ath_settings* settings, ath_targets* targets,
                                  const ath_targets* under, ath_frame_stats* stats, void* stream);

/* ---- differentiation (no counterpart in the reference's API: it only has
 * the colour gradient of splat_blend.slang:381-398, contributionMode 4) ------ */

/* A cloud as FP32 training parameters: one Gaussian a row of each array.
 * The projection decodes them as the reference's upload would: opacity =
 * sigmoid(logit), scale = exp(log scale), rotation = the unit quaternion,
 * base colour = 0.5 + SH0 * DC. */
typedef struct {
    const float* means;    /* float4: x y z, opacity logit (16-byte aligned) */
    const float* scales;   /* float4: log scale x y z, unused */
    const float* quats;    /* float4: w x y z, any length */
    const float* sh;       /* sh_stride floats: DC rgb, then the rest coefficients rgb per basis */
    uint32_t count;
    uint32_t sh_degree;    /* 0..3 */
    uint32_t sh_stride;    /* floats a Gaussian: at least 3 (1 + 3, 8 or 15 bases) */
    int32_t linear;        /* 1: colours are linear light; 0: sRGB, decoded per splat */
    double object_to_world[16];
} ath_params;

/* Gradients with respect to ath_params, in its layout (means' fourth float is
 * the opacity logit's). Added into: zero them before a batch. */
typedef struct {
    float* means;
    float* scales;
    float* quats;
    float* sh;
} ath_param_grads;

/* The forward of a differentiable frame: ath_raster_render for one cloud of
 * training parameters, keeping what the backward needs (per pixel the final
 * transmittance and one past the last record blended; the frame's pairs and
 * records). The backward must follow before the next render on this handle. */
ath_status ath_raster_render_params(ath_raster* r, const ath_projection* projection, const ath_params* params,
                                    const ath_settings* settings, ath_targets* targets, ath_frame_stats* stats,
                                    void* stream);

/* The backward of the last ath_raster_render_params: from dL/dcolour (float4 a
 * pixel, premultiplied rgba) and optionally dL/ddepth (a float a pixel, may be
 * NULL), adds dL/dparameters into `grads`. Reverse-order blend recomputed from
 * the stored transmittances, then the projection's adjoint. The targets and
 * parameters of the forward must be unchanged. */
ath_status ath_raster_backward(ath_raster* r, const float* dl_dcolour, const float* dl_ddepth, ath_param_grads* grads,
                               void* stream);

/* L = mean over pixels and the three colour channels of (colour - target)^2:
 * writes dL/dcolour (float4 a pixel, alpha 0) and adds L into *loss (device).
 * colour: float4 a pixel, target: float3 a pixel. */
ath_status ath_l2_loss(const float* colour, const float* target, uint32_t pixels, float* dl_dcolour, float* loss,
                       void* stream);

/* ---- the batched, mixed-precision training step (no counterpart in the
 * reference: it renders one camera a call, TileRasterizer.h:316-317) ------ */

/* A cloud in the mixed-precision layout: geometry FP32 as ath_params; the SH
 * DC and band 1 in BF16 (12 values: DC rgb, then band 1 rgb per basis), bands
 * 2-3 in FP8 e4m3 (36 values, rgb per basis) times a per-Gaussian FP32 scale. */
typedef struct {
    const float* means;     /* float4: x y z, opacity logit */
    const float* scales;    /* float4: log scales */
    const float* quats;     /* float4: w x y z */
    const void* sh_low;     /* 12 bf16 a Gaussian; 8-byte aligned */
    const void* sh_high;    /* 36 e4m3 a Gaussian; 4-byte aligned */
    const float* sh_scale;  /* 1 float a Gaussian */
    uint32_t count;
    uint32_t sh_degree;
    int32_t linear;
    double object_to_world[16];
} ath_mixed_params;

/* Converts ath_params' FP32 SH to the mixed layout (sh_low 12 x 2 bytes, sh_high
 * 36 bytes, sh_scale 4 bytes a Gaussian): the bands' scale is their largest
 * magnitude over e4m3's largest finite value, 448. */
ath_status ath_params_to_mixed(const ath_params* params, void* sh_low, void* sh_high, float* sh_scale, void* stream);

/* One view of a batch: a projection (ath_projection_for) and its image size. */
typedef struct {
    ath_projection projection;
    uint32_t width, height;
} ath_view;

typedef struct ath_batch ath_batch;

typedef struct {
    uint64_t pairs;        /* (tile, Gaussian) pairs of every view, the last step */
    uint64_t capacity;     /* pairs the buffers hold */
    uint32_t kept;         /* (view, Gaussian) records drawn */
    uint32_t tile, block_batch;
    float ms_per_step;     /* ath_batch_tune: the chosen setting's time */
    uint32_t degenerate;   /* records whose 2D conic was inverted in FP64 (det < 1e-6 trace^2) */
    /* The blends' work, counted by the step ath_batch_time_stages runs before its
     * timed one on the same inputs (neither the captured steps nor the timed step
     * count, to keep the counting out of their time). */
    uint64_t evaluated;    /* (pixel, record) evaluations of the forward blend */
    uint64_t blended;      /* of them, those that blended (inside the cutoff, alpha at least 1/255) */
    uint64_t adjoint_visited;  /* (pixel, record) evaluations of the blend adjoint (before the pixel's last contributor) */
    uint64_t adjoint_live;     /* of them, those that blended and whose gradient terms were summed */
    uint64_t warp_visits_forward;   /* (warp, record) visits of the forward walk (a warp: 64 pixels) */
    uint64_t warp_visits_adjoint;   /* (warp, record) visits of the adjoint walk */
    uint64_t warp_visits_adjoint_summed;  /* of them, those with a live pixel, whose sums the warp reduced */
    uint64_t records_staged;        /* records the blends' blocks loaded and box-tested for the forward walk */
} ath_batch_stats;

ath_status ath_batch_create(ath_batch** out);
void ath_batch_destroy(ath_batch* b);
/* The views every step draws (at most 256), and the frame settings they share
 * (background, max_sh_degree, antialias). Images are concatenated in view order:
 * view v's pixel (x, y) is at v's base + y * width + x; ath_batch_pixels gives the total. */
ath_status ath_batch_set_views(ath_batch* b, const ath_view* views, uint32_t count, const ath_settings* settings);
/* Tile size (8, 16 or 32) and records a block stages at once (64, 128, 256 or 512).
 * Images do not depend on either: a pixel blends the same records in the same
 * order whatever tile holds it. Default 16 and 256. */
ath_status ath_batch_set_tuning(ath_batch* b, uint32_t tile, uint32_t block_batch);
ath_status ath_batch_pixels(ath_batch* b, uint32_t* pixels);
/* How a step's (tile, Gaussian) pairs are keyed. 0 (default): one 64-bit word
 * (global tile | 24-bit depth key | Gaussian index), sorted keys-only, while
 * those bits fit in 64; else the packed word with the depth key's exponent byte
 * renumbered (below) while that fits; else the wide form. 1: always the packed
 * word with the 24-bit depth key (a step whose bits do not fit fails with
 * ATH_E_UNSUPPORTED). 2: the wide form, a 64-bit (global tile << 24 | depth key)
 * key and a 32-bit Gaussian index, sorted as key and value. 3: always the packed
 * word with the renumbered depth. Renumbered: the depth field is 16 mantissa bits
 * under the exponent byte less a base, in as few bits as the exponents a sizing
 * saw (with two to spare on each side) need; the order is the depth key's. A
 * step whose depths fall outside that range is reported by ath_batch_check as
 * ATH_E_CAPACITY (that step's order is not valid) and the next step plans again.
 * 50M Gaussians in 8 views of 3840x2160 take the renumbered form. The pairs'
 * order, and so the image, is the same in every form. */
ath_status ath_batch_set_key_mode(ath_batch* b, uint32_t mode);
/* One training step over every view, with nothing read back to the host:
 * project and emit every view's pairs (one launch), sort them all (one packed
 * 64-bit sort), blend every view's tiles (one persistent launch), the loss
 * (each view's mean L2 over its pixels and r g b against `target`, summed over
 * views, into *loss), and the backward, whose dL/dparameters overwrite `grads`
 * (FP32, ath_param_grads' layout, sh 48 floats a Gaussian). colour: float4 a
 * pixel, target: float3 a pixel, both concatenated. The first call sizes the
 * pair buffers (one host read) and captures the step into a CUDA graph; later
 * calls with the same pointers replay it. Up to four captured steps are kept,
 * keyed by the arrays they read and write, so a caller that alternates two
 * target (or colour) buffers, to upload one while the other is in use, replays
 * both after their first call. ath_batch_set_views, ath_batch_set_tuning and
 * ath_batch_set_key_mode may be called between steps, and the cloud may change
 * size: the next step grows the buffers and captures again. An empty cloud
 * (count 0) draws the background, and its gradient arrays may be null. */
ath_status ath_batch_train_step(ath_batch* b, const ath_mixed_params* params, const float* target, float* colour,
                                float* loss, ath_param_grads* grads, void* stream);
/* ath_batch_train_step with the target still arriving: the step's projection,
 * sort and ranges start at once, and only its blends wait for `target_ready` (a
 * cudaEvent_t the caller records after the target's upload, on any stream), so
 * that the upload overlaps them. The event is part of the captured step: one
 * event a target buffer, as for double-buffered uploads. */
ath_status ath_batch_train_step_after(ath_batch* b, const ath_mixed_params* params, const float* target,
                                      void* target_ready, float* colour, float* loss, ath_param_grads* grads,
                                      void* stream);
/* Gradient buckets, for a step whose gradients are summed over GPUs while it
 * still runs (no counterpart in the reference, which is single-device): with
 * `buckets` > 0, the step's projection adjoint runs bucket by bucket over
 * consecutive ranges of the `count` Gaussians (ath_gradient_bucket gives bucket
 * k's first Gaussian and size), writes bucket k's gradients into grads[k]'s four
 * arrays (rows of that bucket's Gaussians only, ath_param_grads' layout), and,
 * when `events` is given, records the cudaEvent_t events[k] on the step's stream
 * right after bucket k: a caller's stream that waits on it can start bucket k's
 * all-reduce while the later buckets are computed. ath_batch_train_step's
 * `grads` is then unused (may be NULL), and the cloud must have `count`
 * Gaussians. 0 buckets: the whole cloud into `grads` again. The next step
 * captures again. */
ath_status ath_batch_set_buckets(ath_batch* b, uint32_t count, uint32_t buckets, const ath_param_grads* grads,
                                 void* const* events);
/* Bucket k of `buckets` over `count` Gaussians: its first Gaussian and its size.
 * Consecutive ranges in whole blocks of 128 Gaussians, their sizes differing by
 * at most one block, covering every Gaussian once. */
ath_status ath_gradient_bucket(uint32_t count, uint32_t buckets, uint32_t k, uint32_t* first, uint32_t* n);

/* Every view's forward alone, for rendering many cameras at once, where the
 * reference's TileRasterizer::render draws one camera a call
 * (TileRasterizer.h:468-474): the same projection, sort and blend as a training
 * step, with no loss and no backward, into `colour` (float4 a pixel, views
 * concatenated; premultiplied linear, as ath_raster_render's colour target)
 * and, when not null, `depth` (float a pixel, views concatenated; the view-z
 * depth of ath_settings.depth_mode / depth_threshold as given to
 * ath_batch_set_views, as ath_raster_render's depth target). P is not written.
 * Sized and captured like a step, in a captured graph of its own. */
ath_status ath_batch_render(ath_batch* b, const ath_mixed_params* params, float* colour, float* depth, void* stream);
/* Waits for `stream` and reports the last step; ATH_E_CAPACITY when its pairs
 * outgrew the buffers (that step is not valid; the next one grows them). */
ath_status ath_batch_check(ath_batch* b, ath_batch_stats* out, void* stream);
/* The autotuner: times `repeats` steps for every tile size in {8, 16, 32} and
 * block batch in {64, 128, 256, 512}, keeps the fastest and reports it in `best`.
 * The pair buffers are then sized again for the setting kept. */
ath_status ath_batch_tune(ath_batch* b, const ath_mixed_params* params, const float* target, float* colour,
                          float* loss, ath_param_grads* grads, uint32_t repeats, ath_batch_stats* best, void* stream);

/* One step as ath_batch_train_step runs it, not captured, with events between
 * its stages, waited for: ms[] = project+emit (with the record gradients'
 * clearing), sort, ranges, blends (the forward blend, the loss and the blend
 * adjoint, one kernel), projection adjoint. For measurement. A step that counts
 * the blends' work (ath_batch_stats) runs first, untimed. */
ath_status ath_batch_time_stages(ath_batch* b, const ath_mixed_params* params, const float* target, float* colour,
                                 float* loss, ath_param_grads* grads, float ms[5], void* stream);

/* The last step's sorted pairs and tile ranges, for inspection: device
 * pointers the batch owns, valid until its next step. A packed pair is
 * (global tile << key_shift) | (depth field << slot_bits) | Gaussian; a wide
 * pair's key is (global tile << 24) | depth key (slot_bits 0, key_shift 24) with
 * its Gaussian in sorted_values. The depth field is the 24-bit depth key when
 * depth_bits is 24, else ((exponent byte - exp_base) << 16) | its 16 low bits.
 * View v's tiles start at tile_bases[v] (host array of `views` entries). */
typedef struct {
    uint64_t pairs;
    uint32_t key_shift, slot_bits, total_tiles, views;
    const uint64_t* sorted_pairs;
    const uint32_t* ranges;      /* 2 a global tile: [start, end) */
    const uint32_t* sorted_values; /* wide pairs: the Gaussian of each sorted pair; NULL when packed */
    const uint32_t* tile_bases;  /* host */
    uint32_t depth_bits, exp_base;
} ath_batch_buffers;

ath_status ath_batch_buffers_of(ath_batch* b, ath_batch_buffers* out, void* stream);

/* TileRasterizer::latestCounters (TileRasterizer.h:478; TileRasterizer.cpp:
 * 1356-1381): the newest frame drawn with count_splats that the device has
 * finished, read from pinned memory its counts were copied to behind an event
 * (a ring of three, as the reference's AsyncReadback). Never waits: right after
 * a frame it may still give an older one. A frame drawn without count_splats
 * leaves it as it was. ATH_E_NOT_FOUND until a counted frame has finished. */
ath_status ath_raster_latest_counters(ath_raster* r, ath_splat_counters* out);

/* The last frame's status, and its totals (splats, visible, pairs) into `out`
 * (may be NULL): waits for that frame (and for the ath_raster_backward after
 * it, when there is one) to finish. ATH_E_CAPACITY: its pairs outgrew the
 * handle's capacity (the frame is not valid; the next frame grows it).
 * ATH_E_TIMEOUT: a bounded look-back wait gave up. ATH_E_INTERNAL: an index
 * fell outside its buffer (skipped). ATH_E_NOT_FOUND: no frame yet. The
 * reference reports these from render itself, which waits mid-frame. */
ath_status ath_raster_check(ath_raster* r, ath_frame_stats* out);

/* The last frame's intermediate buffers, for inspection (what the reference's
 * tests read through its Buffer handles). Device pointers owned by the
 * rasteriser, valid until its next render or release_scratch:
 *   records    12 floats a slot: screen (centre xy, view z, cutoff), conic (a b c, alpha),
 *              colour (rgb, 0) -- splat/frame.slang:269-281's ProjRecord without the surfel
 *              word; written for kept slots only
 *   rects      2 words a slot: x0 | y0 << 16, x1 | y1 << 16 (inclusive tiles; kept slots)
 *   keys       a slot: the 24-bit depth key, or 0xFF000000 | cull reason (frame.slang:42-49)
 *   offsets    a slot: its first pair (exclusive scan of tiles touched)
 *   pair_keys, pair_splats   the sorted pairs: tile << 24 | depth key, and the slot
 *   ranges     2 a tile: [start, end) into the sorted pairs (splat_ranges.slang)
 *   grads      after ath_raster_backward, 10 floats a slot: dL/d(centre x y, conic a b c,
 *              alpha, colour r g b, view z) -- the colour part is contributionMode 4's sums */
typedef struct {
    uint32_t slots, pairs, tiles;
    const float* records;
    const uint32_t* rects;
    const uint32_t* keys;
    const uint32_t* offsets;
    const uint64_t* pair_keys;
    const uint32_t* pair_splats;
    const uint32_t* ranges;
    const float* grads;
} ath_frame_buffers;

ath_status ath_raster_frame_buffers(ath_raster* r, ath_frame_buffers* out);

/* ---- the radix sort: gpu::RadixSort (modules/gpu/include/athenea/gpu/algo/RadixSort.h;
 * RadixSort.cpp:95-261) ---------------------------------------------------- */

typedef struct ath_sorter ath_sorter;

/* RadixSort::create. Owns the sort's working memory (histograms, look-back words). */
ath_status ath_sorter_create(ath_sorter** out);
void ath_sorter_destroy(ath_sorter* s);

/* RadixSort::sort(batch, SortBuffers, count, keyBits): sorts the first `count`
 * (key, value) pairs stably by the low `key_bits` bits (1..64) of the key,
 * eight bits a pass. keys/values hold the input and receive the result; the
 * scratch pair (as SortBuffers' scratchKeys/scratchValues) holds count
 * entries each. An odd number of passes ends with a copy back. Enqueued on
 * `stream`, not waited for, and nothing is read back: what the sorts raise is
 * kept for ath_sorter_check. */
ath_status ath_sorter_sort(ath_sorter* s, uint64_t* keys, uint32_t* values, uint64_t* scratch_keys,
                           uint32_t* scratch_values, uint32_t count, uint32_t key_bits, void* stream);
/* Waits for the sorter's last sort and reports what its sorts raised since the
 * last check: ATH_E_TIMEOUT for a look-back wait that gave up (bounded spin),
 * ATH_E_INTERNAL for an index outside the buffers. Then clears it. */
ath_status ath_sorter_check(ath_sorter* s);

/* The same sort for callers that cannot allocate device memory while they
 * sort: a plugin whose host application owns the device memory and holds it to
 * a fixed budget mid-frame, or a real-time frame that cannot take the stall of
 * an allocation. It has no counterpart in the reference. The sort's own working
 * memory (histograms, look-back words, tickets, a status word) is a fixed 3.5 MiB
 * array every GPU that loads the library holds until exit; nothing is
 * allocated. At most 1,048,576 pairs a call (larger counts return
 * ATH_E_INVALID_ARGUMENT). The first call on a device (or the first status
 * query) finds that array's address and sets the kernel up: make it before any
 * stream capture. A call enqueues its work and returns: it reads nothing back
 * and does not wait. Every call shares the array, so calls that overlap on the
 * GPU race; keys/values and the scratch pair are as for ath_sorter_sort. */
ath_status ath_sort_pairs_static(uint64_t* keys, uint32_t* values, uint64_t* scratch_keys, uint32_t* scratch_values,
                                 uint32_t count, uint32_t key_bits, void* stream);
/* What the calls of ath_sort_pairs_static on this device raised since the last
 * query, when the caller chooses to look: waits for `stream`, then reports
 * ATH_E_TIMEOUT (a look-back wait gave up) or ATH_E_INTERNAL (an index outside
 * the buffers) and clears it. Allocates nothing. No counterpart in the reference. */
ath_status ath_sort_pairs_static_status(void* stream);

/* ---- decode: scene::CloudLoader::upload's kernels ------------------------ */

/* scene/splat_validate.slang:16-31 + scene/splat_decode.slang:45-173 for
 * 3DGS-encoded float records (io::SplatEncoding: logit opacity, log scale,
 * wxyz rotation, SH DC, rest colour-outer). `records` is device memory,
 * `count` records of `stride` floats; field indices as named. The valid
 * records are written compacted, in file order, to positions/shape/sh (room
 * for `count` splats); *kept receives how many (a device-to-host read). */
typedef struct {
    uint32_t stride;
    uint32_t x, y, z, opacity, scale0, scale1, scale2, rot_w, rot_x, rot_y, rot_z, dc0, dc1, dc2;
    uint32_t rest_base, file_per_colour, keep_per_colour;
} ath_encoding;

ath_status ath_decode_records(const float* records, uint32_t count, const ath_encoding* encoding, float* positions,
                              uint32_t* shape, uint32_t* sh, uint32_t* kept, void* stream);

/* ---- 3DGS PLY files (modules/io/src/SplatReaders.cpp:50-200, readSplatPly) --- */

/* A trained splat cloud's header: its vertex count and the encoding of its
 * records (stride = floats a record, one a vertex property in file order). Only
 * binary little-endian files are read, as by the reference: another format, a
 * list property, an unknown property type or harmonics that are not a whole
 * degree are ATH_E_UNSUPPORTED; a missing x y z / opacity / scale_0..2 /
 * rot_0..3 / f_dc_0..2 is ATH_E_INVALID_ARGUMENT; no file is ATH_E_NOT_FOUND. */
ath_status ath_ply_read_header(const char* path, uint32_t* count, ath_encoding* encoding);
/* The vertex element as count x stride floats into host memory `records`
 * (`capacity` floats), every property widened to float; then
 * ath_decode_records on a device copy gives the packed cloud. A file shorter
 * than its header says is ATH_E_IO_FAILURE. */
ath_status ath_ply_read(const char* path, float* records, uint64_t capacity, uint32_t* count,
                        ath_encoding* encoding);

/* ---- diagnostics --------------------------------------------------------- */

/* A device-memory budget for this library's scratch, in bytes (0: none), as
 * the reference's ATHENEA_GPU_BUDGET (modules/gpu/src/Device.cpp:434-449; the
 * same environment variable, in MiB, sets it at load): a frame whose scratch
 * would pass it fails with ATH_E_OUT_OF_MEMORY, and ath_raster_release_scratch
 * gives memory back (TileRasterizer.cpp:178-191). ath_memory_held reports the
 * bytes this library's buffers hold now and the budget. */
ath_status ath_set_memory_budget(uint64_t bytes);
ath_status ath_memory_held(uint64_t* bytes, uint64_t* budget);
/* Every device-side wait of this library spins a bounded number of times, then
 * sets a status bit and returns (ATH_E_TIMEOUT to the caller, the context
 * usable). This runs that wait on a flag set to `preset` (0: never set) with
 * at most `limit` spins, and reports how many it took: ATH_E_TIMEOUT when the
 * flag was never set. For failure-detection tests; no counterpart in the reference. */
ath_status ath_check_bounded_wait(uint32_t preset, uint32_t limit, uint32_t* spins, void* stream);

/* The current device's FP32 FMA rate (TFLOP/s, two a fused multiply-add) and
 * hardware base-2 exponential rate (G results/s), each the best of `repeats`
 * timed launches of a kernel that keeps every SM's pipe busy: the denominators
 * of the blends' arithmetic roofline. Waits for `stream`. No counterpart in the
 * reference. */
ath_status ath_measure_peaks(uint32_t repeats, double* fma_tflops, double* ex2_gops, void* stream);

/* The message of the last failure on this thread ("" when none). */
const char* ath_last_error_message(void);
/* Version of this library, "major.minor.patch". */
const char* ath_version(void);

#ifdef __cplusplus
}
#endif

#endif
