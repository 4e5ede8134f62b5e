// The rasteriser's host side behind the C ABI (include/athenea_raster.h): the
// B200 counterpart of render::TileRasterizer (modules/render/src/
// TileRasterizer.cpp) for its plain path, and of the camera helpers
// (modules/render/src/Camera.cpp) and FrameParams setters
// (modules/render/src/FrameParams.h) that feed it.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/athenea_raster.h"
#include "host_util.h"
#include "kernels.h"
#include "gauss.cuh"
#include "raster_types.cuh"

using namespace ath;

struct ath_raster {
    int device = 0;
    int sms = 148;
    bool tight = false;   // after release_scratch: grow to the need exactly
    uint32_t slotCapacity = 0, pairCapacity = 0, tileCapacity = 0, instanceCapacity = 0;
    DeviceBuffer recs, rects, keys, offsets, projectFlags, instances;
    DeviceBuffer pairKeys[2], pairVals[2], sortHist, sortFlags, ranges;
    DeviceBuffer words;          // kFrameWords
    PinnedBuffer wordsHost;      // kFrameWords: a frame that waits (its handle's first, or timed) reads them here
    PinnedBuffer instanceStage;  // InstanceConst staging for the H2D copy
    // The last frame's words, copied at its end behind `frameDone` (ath_raster_check,
    // and the next frame's capacity, read them once that event has passed).
    PinnedBuffer statusHost;
    cudaEvent_t frameDone = nullptr;
    bool frameRecorded = false;
    uint32_t frameSlots = 0;
    // Counted frames' words: a ring of kCountDepth copies behind events, as the
    // reference's AsyncReadback (TileRasterizer.cpp:1297-1381; depth 3), so that
    // ath_raster_latest_counters returns the newest finished one without waiting.
    static constexpr int kCountDepth = 3;
    PinnedBuffer countHost[kCountDepth];
    cudaEvent_t countDone[kCountDepth] = {};
    struct CountMeta {
        uint64_t seq = 0, tag = 0;
        uint32_t slots = 0, clouds = 0;
    } countMeta[kCountDepth];
    uint64_t countSeq = 0;
    bool haveCounters = false;
    uint64_t countersSeq = 0;   // the sequence number of `counters`
    ath_splat_counters counters{};
    cudaEvent_t marks[8] = {};
    uint32_t lastSlots = 0, lastTiles = 0, lastSorted = 0;   // what frame_buffers describes
    FrameConst lastFrame{};
    // the differentiable frame's state (ath_raster_render_params -> ath_raster_backward)
    DeviceBuffer finalT, lastContrib, grads;
    bool trainingValid = false;
    InstanceConst trainingInstance{};
    const float* trainingDepth = nullptr;
};

struct ath_sorter {
    int device = 0;
    DeviceBuffer hist, flags, words;   // words: 8 pass tickets, then the status, kept until ath_sorter_check
    PinnedBuffer wordsHost;
    cudaEvent_t done = nullptr;        // after the last sort
    bool recorded = false;
};

namespace {

uint32_t grow(uint32_t have, uint64_t need) {   // TileRasterizer.cpp:30-36
    uint64_t size = std::max<uint64_t>(have, 1024);
    while (size < need) size = size * 3 / 2;
    return (uint32_t)std::min<uint64_t>(size, 0xFFFFFFFFull);
}

uint32_t bitsFor(uint32_t values) {   // FrameParams.h:18-24
    uint32_t bits = 1;
    while (bits < 32 && (uint64_t{1} << bits) < values) ++bits;
    return bits;
}

void matMul4(const double* a, const double* b, double* out) {
    double r[16];
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) {
            double s = 0.0;
            for (int k = 0; k < 4; ++k) s += a[i * 4 + k] * b[k * 4 + j];
            r[i * 4 + j] = s;
        }
    std::memcpy(out, r, sizeof(r));
}

// The inverse of an affine 4x4 (aofx::xform::inverseAffine): the 3x3 inverted
// by cofactors, the translation by -A^-1 t.
void inverseAffine(const double* m, double* out) {
    const double a = m[0], b = m[1], c = m[2], d = m[4], e = m[5], f = m[6], g = m[8], h = m[9], i = m[10];
    const double A = e * i - f * h, B = -(d * i - f * g), C = d * h - e * g;
    const double det = a * A + b * B + c * C;
    const double inv[9] = {A / det, -(b * i - c * h) / det, (b * f - c * e) / det,
                           B / det, (a * i - c * g) / det, -(a * f - c * d) / det,
                           C / det, -(a * h - b * g) / det, (a * e - b * d) / det};
    for (int r = 0; r < 3; ++r) {
        out[r * 4 + 0] = inv[r * 3 + 0];
        out[r * 4 + 1] = inv[r * 3 + 1];
        out[r * 4 + 2] = inv[r * 3 + 2];
        out[r * 4 + 3] = -(inv[r * 3 + 0] * m[3] + inv[r * 3 + 1] * m[7] + inv[r * 3 + 2] * m[11]);
    }
    out[12] = out[13] = out[14] = 0.0;
    out[15] = 1.0;
}

struct DeviceGuard {
    int previous = -1;
    explicit DeviceGuard(int device) {
        if (cudaGetDevice(&previous) == cudaSuccess && previous != device) cudaSetDevice(device);
    }
    ~DeviceGuard() {
        int now = -1;
        if (previous >= 0 && cudaGetDevice(&now) == cudaSuccess && now != previous) cudaSetDevice(previous);
    }
};

ath_status validInstance(const ath_instance& in, uint32_t k) {
    if (in.count == 0) return ATH_OK;
    if (!in.positions || !in.shape || !in.sh)
        return fail(ATH_E_INVALID_ARGUMENT, "instance " + std::to_string(k) + ": a cloud needs positions, shape and sh");
    const uint32_t rpc = in.rest_per_colour;
    if (rpc != 0 && rpc != 3 && rpc != 8 && rpc != 15)
        return fail(ATH_E_INVALID_ARGUMENT, "instance " + std::to_string(k) + ": rest_per_colour must be 0, 3, 8 or 15");
    const uint32_t need = rpc == 0 ? 1 : (rpc * 3 + 1) / 2;
    if (in.sh_words < need)
        return fail(ATH_E_INVALID_ARGUMENT, "instance " + std::to_string(k) + ": sh_words too small for its harmonics");
    if ((reinterpret_cast<uintptr_t>(in.positions) & 15) || (reinterpret_cast<uintptr_t>(in.shape) & 15))
        return fail(ATH_E_INVALID_ARGUMENT, "instance " + std::to_string(k) + ": positions and shape must be 16-byte aligned");
    return ATH_OK;
}

}   // namespace

// ---- camera helpers ---------------------------------------------------------
extern "C" ath_status ath_camera_default(ath_camera* out) {
    if (!out) return fail(ATH_E_INVALID_ARGUMENT, "ath_camera_default: null output");
    std::memset(out, 0, sizeof(*out));
    for (int i = 0; i < 4; ++i) out->camera_to_world[i * 5] = 1.0;
    out->focal = 50.0;
    out->haperture = 24.576;
    out->near_z = 0.1;
    out->far_z = 10000.0;
    out->window_scale[0] = out->window_scale[1] = 1.0;
    return ATH_OK;
}

// Camera::lookingAt (Camera.cpp:9-25): a camera looking down its own -Z from
// `eye` at `target`; the near plane a thousandth of their distance.
extern "C" ath_status ath_camera_looking_at(const double eye[3], const double target[3], const double up[3],
                                            ath_camera* out) {
    if (!eye || !target || !out) return fail(ATH_E_INVALID_ARGUMENT, "ath_camera_looking_at: null argument");
    const double upY[3] = {0.0, 1.0, 0.0};
    const double* u = up ? up : upY;
    ath_camera_default(out);
    double z[3] = {eye[0] - target[0], eye[1] - target[1], eye[2] - target[2]};
    const double distance = std::sqrt(z[0] * z[0] + z[1] * z[1] + z[2] * z[2]);
    if (!(distance > 0.0)) return fail(ATH_E_INVALID_ARGUMENT, "ath_camera_looking_at: eye and target coincide");
    for (double& v : z) v /= distance;
    double x[3] = {u[1] * z[2] - u[2] * z[1], u[2] * z[0] - u[0] * z[2], u[0] * z[1] - u[1] * z[0]};
    const double xl = std::sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
    if (!(xl > 0.0)) return fail(ATH_E_INVALID_ARGUMENT, "ath_camera_looking_at: up is parallel to the view");
    for (double& v : x) v /= xl;
    const double y[3] = {z[1] * x[2] - z[2] * x[1], z[2] * x[0] - z[0] * x[2], z[0] * x[1] - z[1] * x[0]};
    for (int r = 0; r < 3; ++r) {
        out->camera_to_world[r * 4 + 0] = x[r];
        out->camera_to_world[r * 4 + 1] = y[r];
        out->camera_to_world[r * 4 + 2] = z[r];
        out->camera_to_world[r * 4 + 3] = eye[r];
    }
    out->near_z = std::max(distance * 1e-3, 1e-5);
    return ATH_OK;
}

// projectionFor (Camera.cpp:32-64) and viewFromCamera (:27-30).
extern "C" ath_status ath_projection_for(const ath_camera* c, uint32_t width, uint32_t height, ath_projection* out) {
    if (!c || !out) return fail(ATH_E_INVALID_ARGUMENT, "ath_projection_for: null argument");
    std::memset(out, 0, sizeof(*out));
    double inv[16];
    inverseAffine(c->camera_to_world, inv);
    const double flip[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, -1, 0, 0, 0, 0, 1};
    matMul4(flip, inv, out->world_to_view);
    if (std::fabs(c->window_roll) > 1e-12) {
        const double t = c->window_roll * 3.14159265358979323846 / 180.0;
        const double cs = std::cos(t), sn = std::sin(t);
        const double rz[16] = {cs, -sn, 0, 0, sn, cs, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};
        matMul4(rz, out->world_to_view, out->world_to_view);
    }
    const double w = (double)width, h = (double)height;
    const double focal = w * std::max(c->focal, 1e-9) / std::max(c->haperture, 1e-9);
    out->focal_x = focal * c->window_scale[0];
    out->focal_y = focal * c->window_scale[1];
    out->centre_x = w * 0.5 + c->window_translate[0] * w * 0.5;
    out->centre_y = h * 0.5 + c->window_translate[1] * w * 0.5;
    out->near_z = c->near_z;
    out->far_z = c->far_z;
    out->orthographic = c->orthographic;
    out->eye_world[0] = c->camera_to_world[3];
    out->eye_world[1] = c->camera_to_world[7];
    out->eye_world[2] = c->camera_to_world[11];
    return ATH_OK;
}

extern "C" ath_status ath_settings_default(ath_settings* out) {
    if (!out) return fail(ATH_E_INVALID_ARGUMENT, "ath_settings_default: null output");
    std::memset(out, 0, sizeof(*out));
    out->width = 1920;
    out->height = 1080;
    out->antialias = 1;
    out->antialias_override = -1;
    out->surfels = 1;
    out->max_sh_degree = 3;
    out->depth_threshold = 0.5f;
    out->matte_threshold = 0.5f;
    return ATH_OK;
}

// ---- frame constants (FrameParams.h:32-117) ---------------------------------
namespace ath {

FrameConst frameConstFor(const ath_projection& p, const ath_settings& s) {
    FrameConst F{};
    F.width = s.width;
    F.height = s.height;
    F.tilesX = (s.width + kTileSize - 1) / kTileSize;
    F.tilesY = (s.height + kTileSize - 1) / kTileSize;
    F.focalX = (float)p.focal_x;
    F.focalY = (float)p.focal_y;
    F.centreX = (float)p.centre_x;
    F.centreY = (float)p.centre_y;
    F.nearZ = (float)p.near_z;
    F.farZ = (float)p.far_z;
    F.orthographic = p.orthographic ? 1u : 0u;
    F.tileBits = bitsFor(F.tilesX * F.tilesY);
    F.shLimit = s.max_sh_degree;
    F.depthMode = s.depth_mode;
    F.depthThreshold = s.depth_threshold;
    for (int k = 0; k < 4; ++k) F.bg[k] = s.background[k];
    double v2w[16];
    inverseAffine(p.world_to_view, v2w);
    for (int k = 0; k < 12; ++k) F.viewToWorld[k] = (float)v2w[k];
    return F;
}

InstanceConst instanceConstFor(const ath_projection& p, const ath_settings& s, const ath_instance& in, uint32_t base) {
    InstanceConst I{};
    I.positions = reinterpret_cast<const float4*>(in.positions);
    I.shape = reinterpret_cast<const uint4*>(in.shape);
    I.sh = in.sh;
    I.count = in.count;
    I.base = base;
    I.restPerColour = in.rest_per_colour;
    I.shWords = in.sh_words;
    I.linear = in.linear ? 1u : 0u;
    // antialiasOf / setCloudSpace (FrameParams.h:103-117)
    const bool whole = s.antialias_override >= 0 ? s.antialias_override != 0
                       : in.antialiased >= 0     ? in.antialiased != 0
                                                 : s.antialias != 0;
    I.antialias = whole ? 1u : 0u;
    const float made = s.made_spread * s.made_spread;
    I.paidAt = !whole && made > 0.0f ? made / (made + 0.3f) : 0.0f;
    // setObject (FrameParams.h:84-95; TileRasterizer.cpp:599-601)
    double o2v[16];
    matMul4(p.world_to_view, in.object_to_world, o2v);
    for (int k = 0; k < 12; ++k) I.m[k] = (float)o2v[k];
    double w2o[16];
    inverseAffine(in.object_to_world, w2o);
    for (int r = 0; r < 3; ++r)
        I.eye[r] = (float)(w2o[r * 4 + 0] * p.eye_world[0] + w2o[r * 4 + 1] * p.eye_world[1] +
                           w2o[r * 4 + 2] * p.eye_world[2] + w2o[r * 4 + 3]);
    const ath_edit& e = in.edit;
    I.edit.active = e.active ? 1u : 0u;
    I.edit.shape = e.shape;
    I.edit.mode = e.mode;
    I.edit.invert = e.invert ? 1u : 0u;
    for (int k = 0; k < 3; ++k) {
        I.edit.centre[k] = e.centre[k];
        I.edit.size[k] = e.size[k];
        I.edit.tint[k] = e.tint[k];
    }
    I.edit.saturation = e.saturation;
    I.edit.brightness = e.brightness;
    I.edit.opacity = e.opacity;
    I.edit.minOpacity = e.min_opacity;
    I.edit.maxScale = e.max_scale;
    return I;
}

}   // namespace ath

// ---- the rasteriser ---------------------------------------------------------
extern "C" ath_status ath_raster_create(ath_raster** out) {
    if (!out) return fail(ATH_E_INVALID_ARGUMENT, "ath_raster_create: null output");
    *out = nullptr;
    ath_raster* r = new (std::nothrow) ath_raster();
    if (!r) return fail(ATH_E_OUT_OF_MEMORY, "ath_raster_create: host allocation failed");
    cudaError_t err = cudaGetDevice(&r->device);
    if (err == cudaSuccess) err = cudaDeviceGetAttribute(&r->sms, cudaDevAttrMultiProcessorCount, r->device);
    if (err == cudaSuccess) err = sortPrepare();
    if (err == cudaSuccess) err = r->words.reserve(kFrameWords * sizeof(uint32_t));
    if (err == cudaSuccess) err = r->wordsHost.reserve(kFrameWords * sizeof(uint32_t));
    if (err == cudaSuccess) err = r->statusHost.reserve(kFrameWords * sizeof(uint32_t));
    for (int k = 0; k < ath_raster::kCountDepth && err == cudaSuccess; ++k) {
        err = r->countHost[k].reserve(kFrameWords * sizeof(uint32_t));
        if (err == cudaSuccess) err = cudaEventCreateWithFlags(&r->countDone[k], cudaEventDisableTiming);
    }
    if (err == cudaSuccess) err = cudaEventCreateWithFlags(&r->frameDone, cudaEventDisableTiming);
    if (err == cudaSuccess) err = cudaMemset(r->words.ptr, 0, kFrameWords * sizeof(uint32_t));
    for (int k = 0; k < 8 && err == cudaSuccess; ++k) err = cudaEventCreate(&r->marks[k]);
    if (err != cudaSuccess) {
        ath_status s = failCuda(err, "ath_raster_create");
        ath_raster_destroy(r);
        return s;
    }
    *out = r;
    return ATH_OK;
}

extern "C" void ath_raster_destroy(ath_raster* r) {
    if (!r) return;
    DeviceGuard guard(r->device);
    for (cudaEvent_t& e : r->marks)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t& e : r->countDone)
        if (e) cudaEventDestroy(e);
    if (r->frameDone) cudaEventDestroy(r->frameDone);
    delete r;
}

extern "C" ath_status ath_raster_release_scratch(ath_raster* r) {
    if (!r) return fail(ATH_E_INVALID_ARGUMENT, "ath_raster_release_scratch: null handle");
    DeviceGuard guard(r->device);
    cudaDeviceSynchronize();
    r->tight = true;
    r->slotCapacity = r->pairCapacity = r->tileCapacity = r->instanceCapacity = 0;
    for (DeviceBuffer* b : {&r->recs, &r->rects, &r->keys, &r->offsets, &r->projectFlags, &r->instances,
                            &r->pairKeys[0], &r->pairKeys[1], &r->pairVals[0], &r->pairVals[1], &r->sortHist,
                            &r->sortFlags, &r->ranges, &r->finalT, &r->lastContrib, &r->grads})
        b->release();
    r->trainingValid = false;
    r->frameRecorded = false;
    r->instanceStage.release();
    return ATH_OK;
}

namespace {

// A counted frame's words as SplatCounters (TileRasterizer.cpp:1356-1381).
ath_splat_counters countersOf(const uint32_t* w, const ath_raster::CountMeta& m) {
    ath_splat_counters c{};
    c.tag = m.tag;
    c.slots = m.slots;
    c.visible = w[kWordVisible];
    c.pairs = w[kWordPairsLo];
    c.max_tiles = w[kWordMaxTiles];
    for (int k = 0; k < 7; ++k) c.culled[k] = w[kWordCulled + k];
    c.cloud_count = std::min(m.clouds, kMaxClouds);
    for (uint32_t k = 0; k < c.cloud_count; ++k) {
        c.clouds[k].visible = w[kWordClouds + 2 * k];
        c.clouds[k].pairs = w[kWordClouds + 2 * k + 1];
    }
    return c;
}

// The newest counted frame the device has finished, into r->counters; never waits.
void pollCounters(ath_raster* r) {
    int newest = -1;
    for (int k = 0; k < ath_raster::kCountDepth; ++k) {
        const ath_raster::CountMeta& m = r->countMeta[k];
        if (m.seq == 0 || m.seq <= r->countersSeq) continue;
        if (cudaEventQuery(r->countDone[k]) != cudaSuccess) continue;
        if (newest < 0 || m.seq > r->countMeta[newest].seq) newest = k;
    }
    cudaGetLastError();   // a not-ready query leaves cudaErrorNotReady as the last error
    if (newest < 0) return;
    r->counters = countersOf(static_cast<const uint32_t*>(r->countHost[newest].ptr), r->countMeta[newest]);
    r->countersSeq = r->countMeta[newest].seq;
    r->haveCounters = true;
}

}   // namespace

// latestCounters (TileRasterizer.h:478; TileRasterizer.cpp:1356-1381): the newest
// counted frame the device has finished, read from pinned memory its copy
// landed in; never waits. A frame drawn without count_splats leaves it as it was.
extern "C" ath_status ath_raster_latest_counters(ath_raster* r, ath_splat_counters* out) {
    if (!r || !out) return fail(ATH_E_INVALID_ARGUMENT, "ath_raster_latest_counters: null argument");
    pollCounters(r);
    if (!r->haveCounters) return fail(ATH_E_NOT_FOUND, "no counted frame has finished yet");
    *out = r->counters;
    return ATH_OK;
}

namespace {

ath_status reserveSlots(ath_raster* r, uint32_t slots) {   // reserveSplats (TileRasterizer.cpp:193-226)
    if (slots <= r->slotCapacity && r->recs.bytes) return ATH_OK;
    const uint32_t n = r->tight ? slots : grow(r->slotCapacity, slots);
    cudaError_t err = r->recs.reserve((size_t)n * 48);
    if (err == cudaSuccess) err = r->rects.reserve((size_t)n * 8);
    if (err == cudaSuccess) err = r->keys.reserve((size_t)n * 4);
    if (err == cudaSuccess) err = r->offsets.reserve((size_t)n * 4);
    if (err == cudaSuccess) err = r->projectFlags.reserve((size_t)projectBlocks(n) * 8);
    if (err != cudaSuccess) return failCuda(err, "reserving the splats' scratch");
    r->slotCapacity = n;
    return ATH_OK;
}

ath_status reservePairs(ath_raster* r, uint32_t pairs, uint32_t bits) {   // reservePairs (:228-247)
    if (pairs > r->pairCapacity || !r->pairKeys[0].bytes) {
        const uint32_t n = r->tight ? pairs : grow(r->pairCapacity, pairs);
        cudaError_t err = cudaSuccess;
        for (int k = 0; k < 2 && err == cudaSuccess; ++k) {
            err = r->pairKeys[k].reserve((size_t)n * 8);
            if (err == cudaSuccess) err = r->pairVals[k].reserve((size_t)n * 4);
        }
        if (err != cudaSuccess) return failCuda(err, "reserving the pairs");
        r->pairCapacity = n;
    }
    cudaError_t err = r->sortFlags.reserve(sortFlagWords(std::max(r->pairCapacity, pairs), std::max(bits, 8u)) * 8);
    if (err == cudaSuccess) err = r->sortHist.reserve(sortHistWords() * sizeof(uint32_t));
    if (err != cudaSuccess) return failCuda(err, "reserving the sort's scratch");
    return ATH_OK;
}

}   // namespace

namespace {

ath_status checkFrame(const ath_settings& s, const ath_targets& targets) {
    // TileRasterizer.cpp:302-325
    if (s.width == 0 || s.height == 0) return fail(ATH_E_INVALID_ARGUMENT, "a frame needs a size");
    if (s.width > 0xFFFFu * kTileSize || s.height > 0xFFFFu * kTileSize)
        return fail(ATH_E_UNSUPPORTED, "a frame wider or taller than 65535 tiles");
    if (targets.width != s.width || targets.height != s.height)
        return fail(ATH_E_INVALID_ARGUMENT, "the targets are not the frame's size");
    if (!targets.colour || !targets.depth) return fail(ATH_E_INVALID_ARGUMENT, "the targets need colour and depth");
    if (s.contribution_mode > 4)
        return fail(ATH_E_UNSUPPORTED, "contribution modes are 0 to 4 (TileRasterizer.h:357-366)");
    if (s.contribution_mode != 0 && !s.contribution)
        return fail(ATH_E_INVALID_ARGUMENT, "a contribution mode needs its contribution buffer");
    if (s.contribution_mode == 2 && !s.final_colour)
        return fail(ATH_E_INVALID_ARGUMENT, "contribution mode 2 needs final_colour (the frame drawn whole)");
    if (s.contribution_mode == 3 && !s.lift_mask)
        return fail(ATH_E_INVALID_ARGUMENT, "contribution mode 3 needs lift_mask (a float a pixel)");
    if (s.contribution_mode == 4 && !s.final_colour)
        return fail(ATH_E_INVALID_ARGUMENT, "contribution mode 4 needs final_colour (dL/dpixel)");
    if ((s.crypto != nullptr) != (s.crypto_ids != nullptr))
        return fail(ATH_E_INVALID_ARGUMENT, "a Cryptomatte needs both its ids and its layers");
    if ((s.matte_lift != nullptr) != (s.matte != nullptr))
        return fail(ATH_E_INVALID_ARGUMENT, "a lifted matte needs both the lift's sums and the matte target");
    return ATH_OK;
}

// The status bits of a frame's words as a status: the frame is not valid when any is set.
ath_status frameStatusOf(const uint32_t* w) {
    const uint32_t bits = w[kWordStatus] | w[kWordSticky];
    if (bits & kStatusLookbackTimeout)
        return fail(ATH_E_TIMEOUT, "a look-back wait gave up (bounded spin); the frame is not valid");
    if (bits & kStatusPairOverflow)
        return fail(ATH_E_CAPACITY, "the frame's pairs outgrew the pair buffers; the frame is not valid "
                                    "(the next frame grows them)");
    if (bits & kStatusIndexRange)
        return fail(ATH_E_INTERNAL, "the frame met an index outside its buffers (skipped, not written)");
    return ATH_OK;
}

uint64_t pairsOf(const uint32_t* w) { return (uint64_t)w[kWordPairsLo] | ((uint64_t)w[kWordPairsHi] << 32); }

// What the last frame asked of the pairs, once the device has finished it (never
// waits): the capacity the next frame needs.
uint64_t lastFrameNeed(ath_raster* r) {
    if (!r->frameRecorded) return 0;
    if (cudaEventQuery(r->frameDone) != cudaSuccess) {
        cudaGetLastError();   // not ready
        return 0;
    }
    return pairsOf(static_cast<const uint32_t*>(r->statusHost.ptr));
}

// One frame: project (scan fused), emit, sort, ranges, blend, with nothing read
// back in between. The pairs are sized from a capacity: a handle's first frame
// (and its first after release_scratch) reads the pair total back once and sizes
// them exactly, as the reference does every frame (TileRasterizer.cpp:1093-1102);
// later frames use the capacity the earlier ones needed. A frame whose pairs
// outgrow it raises an overflow status (ath_raster_check reports ATH_E_CAPACITY)
// and the next frame grows the pairs. The sort, the ranges and the blends take
// the pair count from the device. At its end the frame's words are copied to
// pinned memory behind an event (its status, for ath_raster_check), and, when it
// counts, to the counters' ring. `staged` is the instance table in host memory
// (pinned staging). `training` also keeps, per pixel, the final transmittance
// and the last record blended, for the backward.
ath_status drawFrame(ath_raster* r, const FrameConst& F, InstanceConst* staged, uint32_t instanceCount,
                     uint32_t slots, uint32_t layout, const ath_settings& s, ath_targets* targets,
                     ath_frame_stats* stats, cudaStream_t stream, bool training, const ath_targets* under = nullptr) {
    const auto frameStart = std::chrono::steady_clock::now();
    const uint32_t tiles = F.tilesX * F.tilesY;
    const uint32_t bits = 24 + F.tileBits;
    ath_status st = reserveSlots(r, std::max(slots, 1u));
    if (st != ATH_OK) return st;
    if (tiles > r->tileCapacity || !r->ranges.bytes) {
        if (cudaError_t err = r->ranges.reserve((size_t)tiles * 8); err != cudaSuccess)
            return failCuda(err, "reserving the tiles' ranges");
        r->tileCapacity = tiles;
    }
    if (training) {
        const size_t pixels = (size_t)F.width * F.height;
        cudaError_t err = r->finalT.reserve(pixels * 4);
        if (err == cudaSuccess) err = r->lastContrib.reserve(pixels * 4);
        if (err != cudaSuccess) return failCuda(err, "reserving the backward's per-pixel state");
    }
    // The pairs an earlier frame needed, if the device has finished it: grow to them.
    if (const uint64_t need = lastFrameNeed(r); need > r->pairCapacity) {
        if (need > 0xFFFFFFFFull) return fail(ATH_E_UNSUPPORTED, "more than 2^32 (tile, splat) pairs in one frame");
        if ((st = reservePairs(r, (uint32_t)std::min<uint64_t>(need + need / 7 + 4096, 0xFFFFFFFFull), bits)) != ATH_OK)
            return st;
    }
    uint32_t* words = static_cast<uint32_t*>(r->words.ptr);
    uint32_t* wordsHost = static_cast<uint32_t*>(r->wordsHost.ptr);
    const bool timed = s.time_stages != 0;
    const bool sizing = r->pairCapacity == 0 || !r->pairKeys[0].bytes;   // no capacity yet: read the total once
    auto mark = [&](int k) { if (timed) cudaEventRecord(r->marks[k], stream); };

    // --- project, with the tiles-touched scan fused in --------------------
    mark(0);
    cudaError_t err = cudaMemsetAsync(words, 0, kFrameWords * sizeof(uint32_t), stream);
    if (err == cudaSuccess && slots)
        err = cudaMemsetAsync(r->projectFlags.ptr, 0, (size_t)projectBlocks(slots) * 8, stream);
    if (err == cudaSuccess && instanceCount)
        err = cudaMemcpyAsync(r->instances.ptr, staged, instanceCount * sizeof(InstanceConst), cudaMemcpyHostToDevice,
                              stream);
    if (err == cudaSuccess)
        err = launchProject(F, static_cast<const InstanceConst*>(r->instances.ptr), instanceCount, slots, layout,
                            s.count_splats != 0, static_cast<float4*>(r->recs.ptr), static_cast<uint2*>(r->rects.ptr),
                            static_cast<uint32_t*>(r->keys.ptr), static_cast<uint32_t*>(r->offsets.ptr),
                            static_cast<uint64_t*>(r->projectFlags.ptr), words, stream);
    mark(1);
    bool haveTotals = false;
    if (sizing && err == cudaSuccess) {
        // The handle's sizing read: the frame's pair total, to size the pairs exactly.
        err = cudaMemcpyAsync(wordsHost, words, kFrameWords * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream);
        if (err == cudaSuccess) err = cudaStreamSynchronize(stream);
        if (err != cudaSuccess) return failCuda(err, "projecting the splats");
        if (wordsHost[kWordStatus] & kStatusLookbackTimeout)
            return fail(ATH_E_TIMEOUT, "a look-back wait gave up (bounded spin); the frame is not valid");
        const uint64_t pairs64 = pairsOf(wordsHost);
        if (pairs64 > 0xFFFFFFFFull) return fail(ATH_E_UNSUPPORTED, "more than 2^32 (tile, splat) pairs in one frame");
        // room for the next frames to vary without outgrowing it (a seventh over)
        const uint64_t plan = std::min<uint64_t>(std::max<uint64_t>(pairs64, 1) + pairs64 / 7, 0xFFFFFFFFull);
        if ((st = reservePairs(r, (uint32_t)plan, bits)) != ATH_OK) return st;
        haveTotals = true;
    }
    if (err != cudaSuccess) return failCuda(err, "projecting the splats");
    if ((st = reservePairs(r, r->pairCapacity, bits)) != ATH_OK) return st;   // the sort's scratch for this frame's bits
    mark(2);

    // --- emit, sort, ranges (the pair count on the device) ------------------
    const uint32_t capacity = r->pairCapacity;
    uint32_t* kept = words + kWordPairsKept;
    uint64_t* keysBuf[2] = {static_cast<uint64_t*>(r->pairKeys[0].ptr), static_cast<uint64_t*>(r->pairKeys[1].ptr)};
    uint32_t* valsBuf[2] = {static_cast<uint32_t*>(r->pairVals[0].ptr), static_cast<uint32_t*>(r->pairVals[1].ptr)};
    err = launchEmit(F, slots, static_cast<const float4*>(r->recs.ptr), static_cast<const uint2*>(r->rects.ptr),
                     static_cast<const uint32_t*>(r->keys.ptr), static_cast<const uint32_t*>(r->offsets.ptr), words,
                     capacity, keysBuf[0], valsBuf[0], stream);
    mark(3);
    if (err == cudaSuccess)
        err = launchSortDevice(keysBuf, valsBuf, capacity, kept, nullptr, 0, bits, static_cast<uint32_t*>(r->sortHist.ptr),
                               static_cast<uint64_t*>(r->sortFlags.ptr), words + kWordSortTickets, words + kWordSticky,
                               stream);
    const uint32_t sorted = sortPasses(bits) & 1u;
    if (err == cudaSuccess) err = cudaMemsetAsync(r->ranges.ptr, 0, (size_t)tiles * 8, stream);
    if (err == cudaSuccess)
        err = launchRanges(capacity, kept, tiles, keysBuf[sorted], static_cast<uint2*>(r->ranges.ptr),
                           words + kWordSticky, stream);
    mark(4);
    // --- blend ---------------------------------------------------------------
    if (err == cudaSuccess)
        err = launchBlend(F, capacity, slots, static_cast<const uint2*>(r->ranges.ptr), valsBuf[sorted],
                          static_cast<const float4*>(r->recs.ptr), reinterpret_cast<float4*>(targets->colour),
                          targets->depth, reinterpret_cast<float4*>(targets->position),
                          training ? static_cast<float*>(r->finalT.ptr) : nullptr,
                          training ? static_cast<uint32_t*>(r->lastContrib.ptr) : nullptr, words + kWordSticky, stream,
                          Contribution{s.contribution_mode, s.contribution, s.final_colour, s.lift_mask},
                          under ? Under{under->colour, under->depth} : Under{},
                          Matte{s.crypto_ids, s.crypto, under ? s.under_crypto : nullptr, s.matte_lift, s.matte,
                                s.matte_hard != 0 ? 1u : 0u, s.matte_threshold, s.trace});
    mark(5);
    // --- the frame's words: its counters into the ring; its status behind an event
    // (last, so that a wait for the frame covers both)
    if (err == cudaSuccess && s.count_splats) {
        const int k = (int)(r->countSeq % ath_raster::kCountDepth);
        r->countMeta[k] = ath_raster::CountMeta{};   // not readable until its new copy has landed
        err = cudaMemcpyAsync(r->countHost[k].ptr, words, kFrameWords * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream);
        if (err == cudaSuccess) err = cudaEventRecord(r->countDone[k], stream);
        if (err == cudaSuccess) r->countMeta[k] = ath_raster::CountMeta{++r->countSeq, s.counters_tag, slots, instanceCount};
    }
    if (err == cudaSuccess)
        err = cudaMemcpyAsync(r->statusHost.ptr, words, kFrameWords * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream);
    if (err == cudaSuccess) err = cudaEventRecord(r->frameDone, stream);
    if (err != cudaSuccess) return failCuda(err, "drawing the frame");
    r->frameRecorded = true;
    r->frameSlots = slots;
    r->lastSlots = slots;
    r->lastTiles = tiles;
    r->lastSorted = sorted;
    r->lastFrame = F;

    ath_frame_stats out{};
    out.splats = slots;
    if (haveTotals) {
        out.visible = wordsHost[kWordVisible];
        out.pairs = (uint32_t)pairsOf(wordsHost);
    }
    if (timed) {
        // A frame that asks for its stage times waits for its end, and so reports its own status.
        if ((err = cudaEventSynchronize(r->frameDone)) != cudaSuccess) return failCuda(err, "timing the frame");
        const uint32_t* w = static_cast<const uint32_t*>(r->statusHost.ptr);
        if ((st = frameStatusOf(w)) != ATH_OK) return st;
        out.visible = w[kWordVisible];
        out.pairs = (uint32_t)pairsOf(w);
        auto ms = [&](int a, int b) {
            float v = 0.0f;
            cudaEventElapsedTime(&v, r->marks[a], r->marks[b]);
            return (double)v;
        };
        out.project_ms = ms(0, 1);
        out.counts_ms = ms(1, 2);
        out.emit_ms = ms(2, 3);
        out.tile_sort_ms = ms(3, 4);
        out.blend_ms = ms(4, 5);
    }
    out.total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - frameStart).count();
    if (stats) *stats = out;
    return ATH_OK;
}

ath_status reserveInstances(ath_raster* r, uint32_t instanceCount) {
    if (instanceCount > r->instanceCapacity || !r->instances.bytes) {
        const uint32_t n = std::max(instanceCount, 4u);
        cudaError_t err = r->instances.reserve((size_t)n * sizeof(InstanceConst));
        if (err == cudaSuccess) err = r->instanceStage.reserve((size_t)n * sizeof(InstanceConst));
        if (err != cudaSuccess) return failCuda(err, "reserving the instance table");
        r->instanceCapacity = n;
    }
    return ATH_OK;
}

}   // namespace

namespace {

ath_status renderPacked(ath_raster* r, const ath_projection* projection, const ath_instance* instances,
                        uint32_t instanceCount, const ath_settings* settings, ath_targets* targets,
                        const ath_targets* under, ath_frame_stats* stats, void* streamPtr) {
    if (!r || !projection || !settings || !targets || (instanceCount && !instances))
        return fail(ATH_E_INVALID_ARGUMENT, "ath_raster_render: null argument");
    const ath_settings& s = *settings;
    ath_status st = checkFrame(s, *targets);
    if (st != ATH_OK) return st;
    // TileRasterizer.cpp:320-322
    if (under && (under->width != s.width || under->height != s.height))
        return fail(ATH_E_INVALID_ARGUMENT, "the under-layer is not the frame's size");
    if (under && (!under->colour || !under->depth))
        return fail(ATH_E_INVALID_ARGUMENT, "the under-layer needs colour and depth");
    uint64_t total = 0;
    for (uint32_t k = 0; k < instanceCount; ++k) {
        const ath_status v = validInstance(instances[k], k);
        if (v != ATH_OK) return v;
        total += instances[k].count;
    }
    if (total > 0xFFFFFFFFull) return fail(ATH_E_UNSUPPORTED, "more than 2^32 splats in one frame");
    DeviceGuard guard(r->device);
    if ((st = reserveInstances(r, instanceCount)) != ATH_OK) return st;
    InstanceConst* staged = static_cast<InstanceConst*>(r->instanceStage.ptr);
    uint32_t base = 0;
    for (uint32_t k = 0; k < instanceCount; ++k) {
        staged[k] = instanceConstFor(*projection, s, instances[k], base);
        base += instances[k].count;
    }
    r->trainingValid = false;
    return drawFrame(r, frameConstFor(*projection, s), staged, instanceCount, (uint32_t)total, kLayoutPacked, s,
                     targets, stats, static_cast<cudaStream_t>(streamPtr), false, under);
}

}   // namespace

extern "C" ath_status ath_raster_render(ath_raster* r, const ath_projection* projection, const ath_instance* instances,
                                        uint32_t instanceCount, const ath_settings* settings, ath_targets* targets,
                                        ath_frame_stats* stats, void* streamPtr) {
    return renderPacked(r, projection, instances, instanceCount, settings, targets, nullptr, stats, streamPtr);
}

extern "C" ath_status ath_raster_render_over(ath_raster* r, const ath_projection* projection,
                                             const ath_instance* instances, uint32_t instanceCount,
                                             const ath_settings* settings, ath_targets* targets,
                                             const ath_targets* under, ath_frame_stats* stats, void* streamPtr) {
    if (!under) return fail(ATH_E_INVALID_ARGUMENT, "ath_raster_render_over: null under-layer");
    return renderPacked(r, projection, instances, instanceCount, settings, targets, under, stats, streamPtr);
}

namespace ath {

// The training layout as an instance (setObject/setCloudSpace as for a packed cloud).
InstanceConst instanceConstForParams(const ath_projection& p, const ath_settings& s, const ath_params& in) {
    ath_instance packed{};
    packed.count = in.count;
    packed.rest_per_colour = in.sh_degree >= 3 ? 15 : in.sh_degree == 2 ? 8 : in.sh_degree == 1 ? 3 : 0;
    packed.sh_words = 1;
    packed.linear = in.linear;
    packed.antialiased = -1;
    std::memcpy(packed.object_to_world, in.object_to_world, sizeof(packed.object_to_world));
    InstanceConst I = instanceConstFor(p, s, packed, 0);
    I.positions = nullptr;
    I.shape = nullptr;
    I.sh = nullptr;
    I.means = in.means;
    I.scales = in.scales;
    I.quats = in.quats;
    I.shf = in.sh;
    I.shStride = in.sh_stride;
    return I;
}

}   // namespace ath

extern "C" ath_status ath_raster_render_params(ath_raster* r, const ath_projection* projection, const ath_params* params,
                                               const ath_settings* settings, ath_targets* targets,
                                               ath_frame_stats* stats, void* streamPtr) {
    if (!r || !projection || !params || !settings || !targets)
        return fail(ATH_E_INVALID_ARGUMENT, "ath_raster_render_params: null argument");
    const ath_settings& s = *settings;
    ath_status st = checkFrame(s, *targets);
    if (st != ATH_OK) return st;
    const ath_params& P = *params;
    if (P.count && (!P.means || !P.scales || !P.quats || !P.sh))
        return fail(ATH_E_INVALID_ARGUMENT, "ath_raster_render_params: a cloud needs means, scales, quats and sh");
    if (P.sh_degree > 3) return fail(ATH_E_INVALID_ARGUMENT, "ath_raster_render_params: sh_degree must be 0..3");
    const uint32_t rest = P.sh_degree >= 3 ? 15 : P.sh_degree == 2 ? 8 : P.sh_degree == 1 ? 3 : 0;
    if (P.sh_stride < 3 + 3 * rest) return fail(ATH_E_INVALID_ARGUMENT, "ath_raster_render_params: sh_stride too small");
    for (const float* ptr : {P.means, P.scales, P.quats})
        if (reinterpret_cast<uintptr_t>(ptr) & 15)
            return fail(ATH_E_INVALID_ARGUMENT, "ath_raster_render_params: means, scales and quats must be 16-byte aligned");
    DeviceGuard guard(r->device);
    if ((st = reserveInstances(r, 1)) != ATH_OK) return st;
    InstanceConst* staged = static_cast<InstanceConst*>(r->instanceStage.ptr);
    staged[0] = instanceConstForParams(*projection, s, P);
    r->trainingValid = false;
    st = drawFrame(r, frameConstFor(*projection, s), staged, 1, P.count, kLayoutParams, s, targets, stats,
                   static_cast<cudaStream_t>(streamPtr), true);
    if (st != ATH_OK) return st;
    r->trainingInstance = staged[0];
    r->trainingDepth = targets->depth;
    r->trainingValid = true;
    return ATH_OK;
}

extern "C" ath_status ath_raster_backward(ath_raster* r, const float* dlDcolour, const float* dlDdepth,
                                          ath_param_grads* grads, void* streamPtr) {
    if (!r || !dlDcolour || !grads || !grads->means || !grads->scales || !grads->quats || !grads->sh)
        return fail(ATH_E_INVALID_ARGUMENT, "ath_raster_backward: null argument");
    if (!r->trainingValid)
        return fail(ATH_E_INVALID_ARGUMENT, "ath_raster_backward: no ath_raster_render_params frame to differentiate");
    DeviceGuard guard(r->device);
    cudaStream_t stream = static_cast<cudaStream_t>(streamPtr);
    const FrameConst& F = r->lastFrame;
    const InstanceConst& I = r->trainingInstance;
    const uint32_t slots = r->lastSlots;
    cudaError_t err = r->grads.reserve((size_t)std::max(slots, 1u) * kGradWords * sizeof(float));
    if (err == cudaSuccess) err = cudaMemsetAsync(r->grads.ptr, 0, (size_t)slots * kGradWords * sizeof(float), stream);
    uint32_t* words = static_cast<uint32_t*>(r->words.ptr);
    if (err == cudaSuccess)
        err = launchBlendBackward(F, r->pairCapacity, slots, static_cast<const uint2*>(r->ranges.ptr),
                                  static_cast<const uint32_t*>(r->pairVals[r->lastSorted].ptr),
                                  static_cast<const float4*>(r->recs.ptr), static_cast<const float*>(r->finalT.ptr),
                                  static_cast<const uint32_t*>(r->lastContrib.ptr),
                                  reinterpret_cast<const float4*>(dlDcolour), dlDdepth, r->trainingDepth,
                                  static_cast<float*>(r->grads.ptr), words + kWordSticky, stream);
    if (err == cudaSuccess)
        err = launchProjectBackward(F, I, static_cast<const uint32_t*>(r->keys.ptr), static_cast<const float*>(r->grads.ptr),
                                    reinterpret_cast<float4*>(grads->means), reinterpret_cast<float4*>(grads->scales),
                                    reinterpret_cast<float4*>(grads->quats), grads->sh, stream);
    // the frame's words again, with what the backward raised, for ath_raster_check
    if (err == cudaSuccess)
        err = cudaMemcpyAsync(r->statusHost.ptr, words, kFrameWords * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream);
    if (err == cudaSuccess) err = cudaEventRecord(r->frameDone, stream);
    if (err != cudaSuccess) return failCuda(err, "the backward");
    return ATH_OK;
}

// The last frame (and the backward after it, if any): waits for its end and
// reports its status and totals.
extern "C" ath_status ath_raster_check(ath_raster* r, ath_frame_stats* out) {
    if (!r) return fail(ATH_E_INVALID_ARGUMENT, "ath_raster_check: null handle");
    if (!r->frameRecorded) return fail(ATH_E_NOT_FOUND, "no frame has been drawn on this handle");
    DeviceGuard guard(r->device);
    if (const cudaError_t err = cudaEventSynchronize(r->frameDone); err != cudaSuccess)
        return failCuda(err, "waiting for the frame");
    const uint32_t* w = static_cast<const uint32_t*>(r->statusHost.ptr);
    if (out) {
        *out = ath_frame_stats{};
        out->splats = r->frameSlots;
        out->visible = w[kWordVisible];
        out->pairs = (uint32_t)std::min<uint64_t>(pairsOf(w), 0xFFFFFFFFull);
    }
    return frameStatusOf(w);
}

extern "C" ath_status ath_l2_loss(const float* colour, const float* target, uint32_t pixels, float* dlDcolour,
                                  float* loss, void* streamPtr) {
    if (pixels && (!colour || !target || !dlDcolour || !loss))
        return fail(ATH_E_INVALID_ARGUMENT, "ath_l2_loss: null argument");
    const cudaError_t err = launchL2Loss(reinterpret_cast<const float4*>(colour), target, pixels,
                                         reinterpret_cast<float4*>(dlDcolour), loss, static_cast<cudaStream_t>(streamPtr));
    if (err != cudaSuccess) return failCuda(err, "ath_l2_loss");
    return ATH_OK;
}

extern "C" ath_status ath_raster_frame_buffers(ath_raster* r, ath_frame_buffers* out) {
    if (!r || !out) return fail(ATH_E_INVALID_ARGUMENT, "ath_raster_frame_buffers: null argument");
    if (!r->recs.ptr || !r->frameRecorded) return fail(ATH_E_NOT_FOUND, "no frame has been drawn since the scratch was made");
    DeviceGuard guard(r->device);
    // inspection: waits for the frame, whose pair count only the device knew
    if (const cudaError_t err = cudaEventSynchronize(r->frameDone); err != cudaSuccess)
        return failCuda(err, "waiting for the frame");
    out->slots = r->lastSlots;
    out->pairs = static_cast<const uint32_t*>(r->statusHost.ptr)[kWordPairsKept];
    out->tiles = r->lastTiles;
    out->records = static_cast<const float*>(r->recs.ptr);
    out->rects = static_cast<const uint32_t*>(r->rects.ptr);
    out->keys = static_cast<const uint32_t*>(r->keys.ptr);
    out->offsets = static_cast<const uint32_t*>(r->offsets.ptr);
    out->pair_keys = static_cast<const uint64_t*>(r->pairKeys[r->lastSorted].ptr);
    out->pair_splats = static_cast<const uint32_t*>(r->pairVals[r->lastSorted].ptr);
    out->ranges = static_cast<const uint32_t*>(r->ranges.ptr);
    out->grads = static_cast<const float*>(r->grads.ptr);
    return ATH_OK;
}

// ---- the radix sort (gpu::RadixSort) -----------------------------------------
extern "C" ath_status ath_sorter_create(ath_sorter** out) {
    if (!out) return fail(ATH_E_INVALID_ARGUMENT, "ath_sorter_create: null output");
    *out = nullptr;
    ath_sorter* s = new (std::nothrow) ath_sorter();
    if (!s) return fail(ATH_E_OUT_OF_MEMORY, "ath_sorter_create: host allocation failed");
    cudaError_t err = cudaGetDevice(&s->device);
    if (err == cudaSuccess) err = sortPrepare();
    if (err == cudaSuccess) err = s->hist.reserve(sortHistWords() * sizeof(uint32_t));
    if (err == cudaSuccess) err = s->words.reserve(16 * sizeof(uint32_t));
    if (err == cudaSuccess) err = s->wordsHost.reserve(16 * sizeof(uint32_t));
    if (err == cudaSuccess) err = cudaMemset(s->words.ptr, 0, 16 * sizeof(uint32_t));
    if (err == cudaSuccess) err = cudaEventCreateWithFlags(&s->done, cudaEventDisableTiming);
    if (err != cudaSuccess) {
        const ath_status st = failCuda(err, "ath_sorter_create");
        if (s->done) cudaEventDestroy(s->done);
        delete s;
        return st;
    }
    *out = s;
    return ATH_OK;
}

extern "C" void ath_sorter_destroy(ath_sorter* s) {
    if (!s) return;
    DeviceGuard guard(s->device);
    if (s->done) cudaEventDestroy(s->done);
    delete s;
}

extern "C" ath_status ath_sorter_sort(ath_sorter* s, uint64_t* keys, uint32_t* values, uint64_t* scratchKeys,
                                      uint32_t* scratchValues, uint32_t count, uint32_t keyBits, void* streamPtr) {
    if (!s) return fail(ATH_E_INVALID_ARGUMENT, "ath_sorter_sort: null handle");
    if (keyBits < 1 || keyBits > 64) return fail(ATH_E_INVALID_ARGUMENT, "ath_sorter_sort: key_bits must be 1..64");
    if (count > 1 && (!keys || !values || !scratchKeys || !scratchValues))
        return fail(ATH_E_INVALID_ARGUMENT, "ath_sorter_sort: null buffer");
    if (count <= 1) return ATH_OK;
    DeviceGuard guard(s->device);
    cudaStream_t stream = static_cast<cudaStream_t>(streamPtr);
    uint32_t* words = static_cast<uint32_t*>(s->words.ptr);
    cudaError_t err = s->flags.reserve(sortFlagWords(count, keyBits) * 8);
    if (err != cudaSuccess) return failCuda(err, "reserving the sort's look-back words");
    uint64_t* k[2] = {keys, scratchKeys};
    uint32_t* v[2] = {values, scratchValues};
    err = launchSort(k, v, count, keyBits, static_cast<uint32_t*>(s->hist.ptr), static_cast<uint64_t*>(s->flags.ptr),
                     words, words + 8, stream);
    if (err == cudaSuccess && sortResultIndex(count, keyBits) == 1) {
        // RadixSort.cpp:165-174: an odd number of passes copies back.
        err = cudaMemcpyAsync(keys, scratchKeys, (size_t)count * 8, cudaMemcpyDeviceToDevice, stream);
        if (err == cudaSuccess)
            err = cudaMemcpyAsync(values, scratchValues, (size_t)count * 4, cudaMemcpyDeviceToDevice, stream);
    }
    if (err == cudaSuccess) err = cudaEventRecord(s->done, stream);
    if (err != cudaSuccess) return failCuda(err, "sorting");
    s->recorded = true;
    return ATH_OK;
}

// Waits for the sorter's last sort and reports what its sorts since the last
// check raised (then clears it).
extern "C" ath_status ath_sorter_check(ath_sorter* s) {
    if (!s) return fail(ATH_E_INVALID_ARGUMENT, "ath_sorter_check: null handle");
    if (!s->recorded) return ATH_OK;
    DeviceGuard guard(s->device);
    uint32_t* words = static_cast<uint32_t*>(s->words.ptr);
    uint32_t* host = static_cast<uint32_t*>(s->wordsHost.ptr);
    cudaError_t err = cudaEventSynchronize(s->done);
    if (err == cudaSuccess) err = cudaMemcpy(host, words + 8, sizeof(uint32_t), cudaMemcpyDeviceToHost);
    const uint32_t bits = host[0];
    if (err == cudaSuccess && bits) err = cudaMemset(words + 8, 0, sizeof(uint32_t));
    if (err != cudaSuccess) return failCuda(err, "ath_sorter_check");
    if (bits & kStatusLookbackTimeout) return fail(ATH_E_TIMEOUT, "a look-back wait of a sort gave up (bounded spin)");
    if (bits) return fail(ATH_E_INTERNAL, "a sort met an index outside its buffers (skipped)");
    return ATH_OK;
}

// ---- decode -----------------------------------------------------------------
extern "C" ath_status ath_decode_records(const float* records, uint32_t count, const ath_encoding* encoding,
                                         float* positions, uint32_t* shape, uint32_t* sh, uint32_t* kept,
                                         void* streamPtr) {
    if (!encoding || !kept || (count && (!records || !positions || !shape || !sh)))
        return fail(ATH_E_INVALID_ARGUMENT, "ath_decode_records: null argument");
    const ath_encoding& e = *encoding;
    const uint32_t fields[] = {e.x, e.y, e.z, e.opacity, e.scale0, e.scale1, e.scale2, e.rot_w, e.rot_x, e.rot_y,
                               e.rot_z, e.dc0, e.dc1, e.dc2};
    for (uint32_t f : fields)
        if (f >= e.stride) return fail(ATH_E_INVALID_ARGUMENT, "ath_decode_records: a field lies outside the record");
    const uint32_t keep = e.keep_per_colour;
    if (keep > 15 || keep > e.file_per_colour ||
        (keep && (uint64_t)e.rest_base + 2ull * e.file_per_colour + keep > e.stride))
        return fail(ATH_E_INVALID_ARGUMENT, "ath_decode_records: the rest coefficients lie outside the record");
    if ((reinterpret_cast<uintptr_t>(positions) & 15) || (reinterpret_cast<uintptr_t>(shape) & 15))
        return fail(ATH_E_INVALID_ARGUMENT, "ath_decode_records: positions and shape must be 16-byte aligned");
    *kept = 0;
    if (count == 0) return ATH_OK;
    cudaStream_t stream = static_cast<cudaStream_t>(streamPtr);
    DeviceBuffer flags, words;
    PinnedBuffer host;
    cudaError_t err = flags.reserve((size_t)decodeBlocks(count) * 8);
    if (err == cudaSuccess) err = words.reserve(4 * sizeof(uint32_t));
    if (err == cudaSuccess) err = host.reserve(4 * sizeof(uint32_t));
    if (err == cudaSuccess) err = cudaMemsetAsync(flags.ptr, 0, (size_t)decodeBlocks(count) * 8, stream);
    if (err == cudaSuccess) err = cudaMemsetAsync(words.ptr, 0, 4 * sizeof(uint32_t), stream);
    if (err == cudaSuccess)
        err = launchDecode(records, count, e, reinterpret_cast<float4*>(positions), reinterpret_cast<uint4*>(shape), sh,
                           static_cast<uint64_t*>(flags.ptr), static_cast<uint32_t*>(words.ptr), stream);
    if (err == cudaSuccess)
        err = cudaMemcpyAsync(host.ptr, words.ptr, 4 * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream);
    if (err == cudaSuccess) err = cudaStreamSynchronize(stream);
    if (err != cudaSuccess) return failCuda(err, "decoding the records");
    const uint32_t* w = static_cast<const uint32_t*>(host.ptr);
    if (w[1] & kStatusLookbackTimeout) return fail(ATH_E_TIMEOUT, "the decode's compaction gave up waiting");
    if (w[1] & kStatusIndexRange) return fail(ATH_E_INTERNAL, "the decode's compaction went outside its buffers");
    *kept = w[2];
    return ATH_OK;
}

extern "C" const char* ath_version(void) { return "0.1.0"; }
