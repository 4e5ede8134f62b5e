// Stage (c): a stable LSD radix sort of 64-bit keys with 32-bit values, eight
// (or nine) bits a pass, in the onesweep form (Adinets and Merrill, "Onesweep: A Faster
// Least Significant Digit Radix Sort for GPUs", 2022): one read of the keys
// makes every pass's digit histogram, then each pass is a single kernel whose
// tiles rank their keys in shared memory, find where each digit of theirs
// starts by a decoupled look-back over the tiles before them, and scatter.
//
// It replaces the reference's RadixSort (modules/gpu/src/algo/RadixSort.cpp:
// 95-261; shaders/athenea/algo/radix_*.slang), which the rasteriser runs twice
// (24-bit depth keys, then tile keys). Same contract: stable, so equal keys
// keep their input order (algo/radix_common.slang:18-22), and only the low
// `bits` of a key take part.
#include <cuda_runtime.h>

#include "kernels.h"
#include "raster_types.cuh"

namespace ath {
namespace {

constexpr uint32_t kMaxRadix = 512;     // a 9-bit pass's digits: the histograms' stride a pass
constexpr uint32_t kSortThreads = 512;
constexpr uint32_t kWarps = kSortThreads / 32;
constexpr uint32_t kItems = 16;
constexpr uint32_t kTileKeys = kSortThreads * kItems;   // 8192: fewer tiles for the look-back to walk
static_assert(kTileKeys == kSortTileKeys, "kernels.h states the sort's tile size");
// A warp ranks its items in independent chains (an 8-bit pass: items 0-7 and
// 8-15), each with its own digit counters, so the chains' shared-memory round
// trips overlap instead of queueing behind each other; the chains are ordered
// after each other like warps.
constexpr uint32_t kMaxPasses = 8;

// `nDevice`, when given, holds the key count (a count only the device knows, as
// in a step captured in a CUDA graph); `n` is then a bound on it.
__device__ __forceinline__ uint32_t countOf(uint32_t n, const uint32_t* nDevice) {
    return nDevice ? min(n, *nDevice) : n;
}

// Digit d's slot in a per-digit table in shared memory: d with its low five bits
// XORed with the next five (a permutation within each run of 32). A warp's keys
// often hold digits 32 or 64 apart and little else (a pass over an exponent byte's
// few values beside a tile index's low bits); unswizzled, those all fall in one
// bank and their counter reads serialise.
__device__ __forceinline__ uint32_t digitSlot(uint32_t d) { return d ^ ((d >> 5) & 31u); }

// A sort's passes: their digit widths (8 or 9 bits) over bits [firstBit, firstBit + bits).
struct SortPlan {
    uint32_t passes;
    uint32_t width[kMaxPasses];
    uint32_t shift[kMaxPasses];   // from firstBit
};

__global__ void __launch_bounds__(256)
    histogramKernel(const uint64_t* __restrict__ keys, uint32_t n, const uint32_t* __restrict__ nDevice,
                    uint32_t firstBit, const SortPlan plan, uint32_t* __restrict__ hist) {
    __shared__ uint32_t sHist[kMaxPasses * kMaxRadix];
    n = countOf(n, nDevice);
    for (uint32_t j = threadIdx.x; j < plan.passes * kMaxRadix; j += blockDim.x) sHist[j] = 0;
    __syncthreads();
    // eight keys a thread in flight before their counts (one load at a time left the
    // read latency-bound at a third of the bandwidth)
    constexpr uint32_t kBatch = 8;
    const uint64_t threads = (uint64_t)gridDim.x * blockDim.x, me = blockIdx.x * blockDim.x + threadIdx.x;
    for (uint64_t first = 0; first < n; first += kBatch * threads) {
        uint64_t key[kBatch];
#pragma unroll
        for (uint32_t k = 0; k < kBatch; ++k) {
            const uint64_t i = first + k * threads + me;
            key[k] = i < n ? keys[i] >> firstBit : 0ull;
        }
#pragma unroll
        for (uint32_t k = 0; k < kBatch; ++k) {
            if (first + k * threads + me >= n) break;
#pragma unroll
            for (uint32_t p = 0; p < kMaxPasses; ++p)
                if (p < plan.passes) {
                    const uint32_t d = (uint32_t)((key[k] >> plan.shift[p]) & ((1u << plan.width[p]) - 1u));
                    atomicAdd(&sHist[p * kMaxRadix + digitSlot(d)], 1u);
                }
        }
    }
    __syncthreads();
    for (uint32_t j = threadIdx.x; j < plan.passes * kMaxRadix; j += blockDim.x) {
        const uint32_t c = sHist[(j / kMaxRadix) * kMaxRadix + digitSlot(j % kMaxRadix)];
        if (c) atomicAdd(&hist[j], c);
    }
}

// Exclusive scan of one value a thread over the block (kSortThreads threads).
__device__ __forceinline__ uint32_t blockExclusiveScan(uint32_t v, uint32_t* sWarp) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    uint32_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t u = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= (uint32_t)o) incl += u;
    }
    if (lane == 31) sWarp[warp] = incl;
    __syncthreads();
    uint32_t base = 0;
#pragma unroll
    for (uint32_t w = 0; w < kWarps; ++w) base += w < warp ? sWarp[w] : 0u;
    __syncthreads();
    return base + incl - v;
}

// kBits: the pass's digit width, 8 or 9 (kRadixT digits, one thread each in the
// digit phase; a 9-bit pass ranks in one chain, so that its counters fit beside the keys).
template <bool kValues, uint32_t kBits>
__global__ void __launch_bounds__(kSortThreads, kValues ? 1 : 2)
    onesweepKernel(const uint64_t* __restrict__ keysIn, const uint32_t* __restrict__ valsIn,
                   uint64_t* __restrict__ keysOut, uint32_t* __restrict__ valsOut, uint32_t n, uint32_t shift,
                   uint32_t digitMask, const uint32_t* __restrict__ globalHist, uint64_t* __restrict__ flags,
                   uint32_t* __restrict__ ticket,
                   uint32_t* __restrict__ status, const uint32_t* __restrict__ nDevice,
                   const uint32_t* __restrict__ epochDevice) {
    constexpr uint32_t kRadix = 1u << kBits;
    constexpr uint32_t kChains = kBits == 8 ? 2 : 1;
    constexpr uint32_t kChainItems = kItems / kChains;
    constexpr uint32_t kCounters = kWarps * kChains;
    extern __shared__ __align__(16) unsigned char smem[];
    uint64_t* sKeys = reinterpret_cast<uint64_t*>(smem);
    uint32_t* sVals = reinterpret_cast<uint32_t*>(sKeys + kTileKeys);
    uint32_t* sWarpCnt = kValues ? sVals + kTileKeys : sVals;   // kCounters x kRadix
    __shared__ uint32_t sTile;
    __shared__ uint32_t sStart[kRadix];
    __shared__ uint32_t sAdjust[kRadix];
    __shared__ uint32_t sScan[kWarps];

    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    n = countOf(n, nDevice);
    // Look-back words are [epoch:30][status:2][value:32]; a word of another
    // epoch reads as not ready. Without an epoch (0) the caller clears them.
    const uint32_t epoch = epochDevice ? (*epochDevice & 0x3FFFFFFFu) : 0u;
    if (tid == 0) sTile = atomicAdd(ticket, 1u);
    __syncthreads();
    const uint32_t tile = sTile;
    const uint32_t base = tile * kTileKeys;
    if (base >= n) return;   // a tile past the keys (the grid was sized for a bound): out before any work
    for (uint32_t j = tid; j < kCounters * kRadix; j += kSortThreads) sWarpCnt[j] = 0;
    __syncthreads();
    const uint32_t ltMask = (1u << lane) - 1u;

    // Rank: warp `warp` owns keys [base + warp*32*kItems, +32*kItems), item k of
    // lane l being the (k*32 + l)-th; walking k then l is input order, so the
    // ranks are stable.
    uint64_t key[kItems];
    uint32_t val[kItems];
    uint32_t rank[kItems];
#pragma unroll
    for (uint32_t k = 0; k < kItems; ++k) {
        const uint32_t idx = base + warp * 32 * kItems + k * 32 + lane;
        const bool valid = idx < n;
        key[k] = valid ? keysIn[idx] : 0ull;
        if constexpr (kValues) val[k] = valid ? valsIn[idx] : 0u;
    }
#pragma unroll
    for (uint32_t i = 0; i < kChainItems; ++i) {
        uint32_t d[kChains], peers[kChains], before[kChains];
        bool valid[kChains];
#pragma unroll
        for (uint32_t c = 0; c < kChains; ++c) {
            const uint32_t k = c * kChainItems + i;
            valid[c] = base + warp * 32 * kItems + k * 32 + lane < n;
            d[c] = valid[c] ? (uint32_t)((key[k] >> shift) & digitMask) : kRadix + lane;
            peers[c] = __match_any_sync(0xFFFFFFFFu, d[c]);
        }
#pragma unroll
        for (uint32_t c = 0; c < kChains; ++c)
            before[c] = valid[c] ? sWarpCnt[(warp * kChains + c) * kRadix + digitSlot(d[c])] : 0u;
        __syncwarp();
#pragma unroll
        for (uint32_t c = 0; c < kChains; ++c)
            if (valid[c] && lane == (uint32_t)(__ffs(peers[c]) - 1))
                sWarpCnt[(warp * kChains + c) * kRadix + digitSlot(d[c])] = before[c] + __popc(peers[c]);
        __syncwarp();
#pragma unroll
        for (uint32_t c = 0; c < kChains; ++c) rank[c * kChainItems + i] = before[c] + __popc(peers[c] & ltMask);
    }
    __syncthreads();

    // One thread a digit (the first kRadix threads): the warps' counts to exclusive
    // offsets, the tile's count; every thread takes part in the block scans.
    const bool digit = tid < kRadix;
    const uint32_t t = digit ? tid : 0u;
    uint32_t count = 0;
    if (digit) {
#pragma unroll
        for (uint32_t w = 0; w < kCounters; ++w) {
            const uint32_t c = sWarpCnt[w * kRadix + digitSlot(t)];
            sWarpCnt[w * kRadix + digitSlot(t)] = count;
            count += c;
        }
    }
    // Where this tile's share of digit t starts in the output.
    uint64_t* flag = flags + (size_t)tile * kRadix + t;
    uint32_t exclusive = 0;
    const uint64_t tag = (uint64_t)epoch << 34;
    if (tile == 0) {
        exclusive = blockExclusiveScan(digit ? globalHist[t] : 0u, sScan);
        if (digit) storeRelaxed(flag, tag | (2ull << 32) | (uint64_t)(exclusive + count));
    } else if (digit) {
        storeRelaxed(flag, tag | (1ull << 32) | (uint64_t)count);
        uint64_t sum = 0;
        int64_t j = (int64_t)tile - 1;
        uint32_t spins = 0;
        while (j >= 0) {
            const uint64_t v = loadRelaxed(flags + (size_t)j * kRadix + t);
            const uint32_t st = (uint32_t)(v >> 34) == epoch ? (uint32_t)(v >> 32) & 3u : 0u;
            if (st == 0) {
                if (++spins > kSpinLimit || ((spins & 255u) == 0 && gaveUp(status))) {
                    atomicOr(status, kStatusLookbackTimeout);
                    break;
                }
                __nanosleep(32);
                continue;
            }
            sum += v & 0xFFFFFFFFull;
            if (st == 2) break;
            --j;
        }
        exclusive = (uint32_t)sum;
        storeRelaxed(flag, tag | (2ull << 32) | (uint64_t)(exclusive + count));
    }
    const uint32_t start = blockExclusiveScan(count, sScan);
    if (digit) {
        sStart[digitSlot(t)] = start;
        sAdjust[digitSlot(t)] = exclusive - start;
    }
    __syncthreads();

    // Scatter into shared memory in the tile's sorted order, then out.
#pragma unroll
    for (uint32_t k = 0; k < kItems; ++k) {
        const uint32_t idx = base + warp * 32 * kItems + k * 32 + lane;
        if (idx < n) {
            const uint32_t d = (uint32_t)((key[k] >> shift) & digitMask);
            const uint32_t at = digitSlot(d);
            const uint32_t s =
                sStart[at] + sWarpCnt[(warp * kChains + k / kChainItems) * kRadix + at] + rank[k];
            sKeys[s] = key[k];
            if constexpr (kValues) sVals[s] = val[k];
        }
    }
    __syncthreads();
    const uint32_t tileN = min(kTileKeys, n - base);
    for (uint32_t s = tid; s < tileN; s += kSortThreads) {
        const uint64_t k = sKeys[s];
        const uint32_t dst = sAdjust[digitSlot((uint32_t)((k >> shift) & digitMask))] + s;
        if (dst < n) {
            keysOut[dst] = k;
            if constexpr (kValues) valsOut[dst] = sVals[s];
        } else {
            atomicOr(status, kStatusIndexRange);
        }
    }
}

// A pass's dynamic shared memory: its keys (and values) and its chains' digit counters.
constexpr size_t onesweepSmem(bool values, uint32_t bits) {
    return (size_t)kTileKeys * 8 + (values ? (size_t)kTileKeys * 4 : 0) +
           (size_t)kWarps * (bits == 8 ? 2 : 1) * ((size_t)1 << bits) * 4;
}

// The passes of a sort of `bits` bits: eight bits a pass, or, where that takes a
// pass fewer, nine bits in as many passes as needed and eight in the rest
// (34 bits: 9 + 9 + 8 + 8 in four passes, not five).
SortPlan planSort(uint32_t bits) {
    SortPlan p{};
    const uint32_t eights = (bits + 7) / 8, nines = (bits + 8) / 9;
    p.passes = nines < eights ? nines : eights;
    const uint32_t wide = nines < eights ? (bits > 8 * p.passes ? bits - 8 * p.passes : 0) : 0;
    uint32_t at = 0;
    for (uint32_t k = 0; k < p.passes && k < kMaxPasses; ++k) {
        p.width[k] = k < wide ? 9u : 8u;
        p.shift[k] = at;
        at += p.width[k];
    }
    return p;
}

}   // namespace

uint32_t sortPasses(uint32_t bits) { return planSort(bits).passes; }
uint32_t sortTiles(uint32_t n) { return (n + kTileKeys - 1) / kTileKeys; }
size_t sortFlagWords(uint32_t n, uint32_t bits) {
    const SortPlan p = planSort(bits);
    size_t words = 0;
    for (uint32_t k = 0; k < p.passes; ++k) words += (size_t)sortTiles(n) << p.width[k];
    return words;
}

cudaError_t sortPrepare() {
    cudaError_t err = cudaFuncSetAttribute(onesweepKernel<true, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)onesweepSmem(true, 8));
    if (err == cudaSuccess)
        err = cudaFuncSetAttribute(onesweepKernel<false, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)onesweepSmem(false, 8));
    if (err == cudaSuccess)
        err = cudaFuncSetAttribute(onesweepKernel<true, 9>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)onesweepSmem(true, 9));
    if (err == cudaSuccess)
        err = cudaFuncSetAttribute(onesweepKernel<false, 9>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)onesweepSmem(false, 9));
    return err;
}

// keys/vals[0] hold the input; the sorted result lands in keys/vals[passes & 1]
// (the caller reads sortResultIndex). vals may be null (keys only). The passes
// sort bits [firstBit, firstBit + bits) of the keys, eight or nine at a time
// (planSort). hist: kMaxPasses * kSortHistStride words, flags: sortFlagWords
// words, tickets: one word a pass; all three are zeroed here.
cudaError_t launchSortDevice(uint64_t* keys[2], uint32_t* vals[2], uint32_t n, const uint32_t* nDevice,
                             const uint32_t* epochDevice, uint32_t firstBit, uint32_t bits, uint32_t* hist,
                             uint64_t* flags, uint32_t* tickets, uint32_t* status, cudaStream_t stream) {
    if (n <= 1 && !nDevice) return cudaSuccess;
    const SortPlan plan = planSort(bits);
    const uint32_t passes = plan.passes;
    if (passes > kMaxPasses || firstBit + bits > 64) return cudaErrorInvalidValue;
    const uint32_t tiles = sortTiles(n);
    cudaError_t err = cudaMemsetAsync(hist, 0, sizeof(uint32_t) * kMaxRadix * passes, stream);
    if (err != cudaSuccess) return err;
    if (!epochDevice) {
        err = cudaMemsetAsync(flags, 0, sizeof(uint64_t) * sortFlagWords(n, bits), stream);
        if (err != cudaSuccess) return err;
    }
    err = cudaMemsetAsync(tickets, 0, sizeof(uint32_t) * passes, stream);
    if (err != cudaSuccess) return err;
    int device = 0, sms = 148;
    cudaGetDevice(&device);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const uint32_t hblocks = min((n + 255) / 256, (uint32_t)sms * 4);
    histogramKernel<<<hblocks, 256, 0, stream>>>(keys[0], n, nDevice, firstBit, plan, hist);
    const bool withValues = vals != nullptr && vals[0] != nullptr;
    size_t flagAt = 0;
    for (uint32_t p = 0; p < passes; ++p) {
        const uint32_t in = p & 1u, out = in ^ 1u;
        const uint32_t shift = firstBit + plan.shift[p];
        const uint32_t* h = hist + p * kMaxRadix;
        const uint32_t digitMask = (1u << plan.width[p]) - 1u;
        uint64_t* f = flags + flagAt;
        flagAt += (size_t)tiles << plan.width[p];
#define ATH_PASS(V_, W_)                                                                                          \
    onesweepKernel<V_, W_><<<tiles, kSortThreads, onesweepSmem(V_, W_), stream>>>(                             \
        keys[in], V_ ? vals[in] : nullptr, keys[out], V_ ? vals[out] : nullptr, n, shift, digitMask, h, f,         \
        tickets + p, status, nDevice, epochDevice)
        if (withValues && plan.width[p] == 9) ATH_PASS(true, 9);
        else if (withValues) ATH_PASS(true, 8);
        else if (plan.width[p] == 9) ATH_PASS(false, 9);
        else ATH_PASS(false, 8);
#undef ATH_PASS
    }
    return cudaGetLastError();
}

cudaError_t launchSortBits(uint64_t* keys[2], uint32_t* vals[2], uint32_t n, uint32_t firstBit, uint32_t bits,
                           uint32_t* hist, uint64_t* flags, uint32_t* tickets, uint32_t* status, cudaStream_t stream) {
    return launchSortDevice(keys, vals, n, nullptr, nullptr, firstBit, bits, hist, flags, tickets, status, stream);
}

cudaError_t launchSort(uint64_t* keys[2], uint32_t* vals[2], uint32_t n, uint32_t bits, uint32_t* hist,
                       uint64_t* flags, uint32_t* tickets, uint32_t* status, cudaStream_t stream) {
    return launchSortBits(keys, vals, n, 0, bits, hist, flags, tickets, status, stream);
}

uint32_t sortResultIndex(uint32_t n, uint32_t bits) { return n <= 1 ? 0u : (sortPasses(bits) & 1u); }
uint32_t sortHistWords() { return kMaxPasses * kMaxRadix; }

}   // namespace ath
