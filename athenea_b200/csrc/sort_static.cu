// The radix sort without allocation: ath_sort_pairs_static.
//
// Some callers cannot allocate device memory when they sort. A render
// delegate or an OpenFX node runs inside a host application's frame loop: the
// host owns the device memory and holds the plugin to a budget it must not
// grow mid-frame, and a real-time frame cannot afford the stall of an
// allocation (cudaMalloc synchronises the device). ath_sorter_sort allocates
// its look-back words on first use and whenever a larger sort needs more;
// this entry point instead keeps the sort's working memory (digit histograms,
// look-back words, tile tickets, a status word) in one fixed array that lives
// with the library on every GPU that loads it, and allocates nothing.
//
// The limit follows from that array's size: at most kStaticMaxCount pairs a
// call, 3.5 MiB of device memory a GPU for the library's lifetime. Every call
// shares the array and it keeps the last call's contents, so each call clears
// what must start at zero (histograms, look-back words, tickets); calls that
// overlap on the GPU (on different streams, or from different threads without
// ordering) race on it. A call neither reads anything back nor waits: what the
// calls raise collects in the array's status word until the caller asks for it
// with ath_sort_pairs_static_status, which waits for the stream.
#include <mutex>

#include <cuda_runtime.h>

#include "../../include/athenea_raster.h"
#include "host_util.h"
#include "kernels.h"
#include "raster_types.cuh"

namespace ath {
namespace {

constexpr uint32_t kStaticMaxCount = 1u << 20;              // pairs a call
constexpr uint32_t kStaticMaxPasses = 8;                    // 64-bit keys, 8 bits a pass
constexpr size_t kStaticTiles = kStaticMaxCount / kSortTileKeys;   // the onesweep's tiles
// look-back words (u64): a tile's words over every pass, at most 3584 (63 key bits
// sort in seven 9-bit passes of 512 digits; 64 bits in eight 8-bit passes of 256)
constexpr size_t kFlagWords = kStaticTiles * 7 * 512;
constexpr size_t kHistWords = kStaticMaxPasses * 512 / 2;               // 8 x 512 u32 histograms, as u64
constexpr size_t kCounterWords = 8;                                     // 16 u32: 8 pass tickets, status
constexpr size_t kScratchWords = kFlagWords + kHistWords + kCounterWords;

static __device__ __align__(256) uint64_t gSortScratch[kScratchWords];

// The array's device address, found once per device with that device current
// (in host code the symbol's name is only a host-side stand-in for it).
struct DeviceScratch {
    bool ready = false;
    uint64_t* ptr = nullptr;
};
constexpr int kMaxDevices = 64;
std::mutex gMutex;
DeviceScratch gPerDevice[kMaxDevices];

ath_status scratchOf(int device, uint64_t** out) {
    std::lock_guard<std::mutex> lock(gMutex);
    if (device < 0 || device >= kMaxDevices) return fail(ATH_E_UNSUPPORTED, "ath_sort_pairs_static: device ordinal too large");
    DeviceScratch& d = gPerDevice[device];
    if (!d.ready) {
        void* p = nullptr;
        cudaError_t err = cudaGetSymbolAddress(&p, gSortScratch);
        if (err != cudaSuccess) return failCuda(err, "ath_sort_pairs_static: finding the static working memory");
        err = sortPrepare();   // the onesweep kernel's shared-memory limit, once a device
        if (err != cudaSuccess) return failCuda(err, "ath_sort_pairs_static: preparing the sort");
        d.ptr = static_cast<uint64_t*>(p);
        d.ready = true;
    }
    *out = d.ptr;
    return ATH_OK;
}

}   // namespace
}   // namespace ath

using namespace ath;

extern "C" ath_status ath_sort_pairs_static(uint64_t* keys, uint32_t* values, uint64_t* scratchKeys,
                                            uint32_t* scratchValues, uint32_t count, uint32_t keyBits,
                                            void* streamPtr) {
    if (keyBits < 1 || keyBits > 64) return fail(ATH_E_INVALID_ARGUMENT, "ath_sort_pairs_static: key_bits must be 1..64");
    if (count > kStaticMaxCount)
        return fail(ATH_E_INVALID_ARGUMENT, "ath_sort_pairs_static: " + std::to_string(count) +
                                                " pairs exceed the static working memory's limit of " +
                                                std::to_string(kStaticMaxCount));
    if (count > 1 && (!keys || !values || !scratchKeys || !scratchValues))
        return fail(ATH_E_INVALID_ARGUMENT, "ath_sort_pairs_static: null buffer");
    if (count <= 1) return ATH_OK;
    int device = 0;
    cudaError_t err = cudaGetDevice(&device);
    if (err != cudaSuccess) return failCuda(err, "ath_sort_pairs_static");
    uint64_t* scratch = nullptr;
    const ath_status st = scratchOf(device, &scratch);
    if (st != ATH_OK) return st;
    cudaStream_t stream = static_cast<cudaStream_t>(streamPtr);
    uint64_t* flags = scratch;
    uint32_t* hist = reinterpret_cast<uint32_t*>(scratch + kFlagWords);
    uint32_t* counters = reinterpret_cast<uint32_t*>(scratch + kFlagWords + kHistWords);
    uint32_t* status = counters + 8;
    if (sortFlagWords(count, keyBits) > kFlagWords || sortHistWords() > 2 * kHistWords)
        return fail(ATH_E_INTERNAL, "ath_sort_pairs_static: the static working memory is too small for this sort");
    // The status word is not read here: the call enqueues its work and returns.
    // What a call raises (a look-back that gave up, an index outside the buffers)
    // stays in the word until ath_sort_pairs_static_status reads and clears it.
    // launchSort clears the histograms, the look-back words and the tickets it uses.
    uint64_t* k[2] = {keys, scratchKeys};
    uint32_t* v[2] = {values, scratchValues};
    err = launchSort(k, v, count, keyBits, hist, flags, counters, status, stream);
    if (err == cudaSuccess && sortResultIndex(count, keyBits) == 1) {
        err = cudaMemcpyAsync(keys, scratchKeys, (size_t)count * 8, cudaMemcpyDeviceToDevice, stream);
        if (err == cudaSuccess)
            err = cudaMemcpyAsync(values, scratchValues, (size_t)count * 4, cudaMemcpyDeviceToDevice, stream);
    }
    if (err != cudaSuccess) return failCuda(err, "ath_sort_pairs_static");
    return ATH_OK;
}

// The sorts' status, when the caller chooses to look: waits for `stream` (the
// stream the sorts were enqueued on), reads what the calls since the last look
// raised from the static array, and clears it. Allocates nothing: the word is
// read into a host variable by a plain copy.
extern "C" ath_status ath_sort_pairs_static_status(void* streamPtr) {
    int device = 0;
    cudaError_t err = cudaGetDevice(&device);
    if (err != cudaSuccess) return failCuda(err, "ath_sort_pairs_static_status");
    uint64_t* scratch = nullptr;
    const ath_status st = scratchOf(device, &scratch);
    if (st != ATH_OK) return st;
    cudaStream_t stream = static_cast<cudaStream_t>(streamPtr);
    uint32_t* status = reinterpret_cast<uint32_t*>(scratch + kFlagWords + kHistWords) + 8;
    uint32_t bits = 0;
    err = cudaStreamSynchronize(stream);
    if (err == cudaSuccess) err = cudaMemcpy(&bits, status, sizeof(bits), cudaMemcpyDeviceToHost);
    if (err == cudaSuccess && bits != 0) err = cudaMemset(status, 0, sizeof(uint32_t));
    if (err != cudaSuccess) return failCuda(err, "ath_sort_pairs_static_status");
    if (bits & kStatusLookbackTimeout)
        return fail(ATH_E_TIMEOUT, "ath_sort_pairs_static: a look-back wait of a sort gave up (bounded spin)");
    if (bits != 0) return fail(ATH_E_INTERNAL, "ath_sort_pairs_static: a sort met an index outside its buffers");
    return ATH_OK;
}
