// Diagnostics: failure detection without a fault, and the arithmetic peaks.
//
// Failure detection without a fault. Every device-side wait in this library
// (the decoupled look-backs of the projection's scan, of the sort and of the
// batched step, and the persistent tile queues' tickets) spins a bounded number
// of times; past it the kernel sets a status bit and returns, and the host
// reports ATH_E_TIMEOUT with the context still usable. ath_check_bounded_wait
// runs that same shape of wait on a flag the caller may leave unset, so that a
// test can make the wait run out and see the status come back.
#include <algorithm>

#include <cuda_runtime.h>

#include "../../include/athenea_raster.h"
#include "host_util.h"
#include "raster_types.cuh"

using namespace ath;

namespace {

__global__ void boundedWaitKernel(const uint32_t* flag, uint32_t limit, uint32_t* status, uint32_t* spinsOut) {
    uint32_t spins = 0;
    while (*reinterpret_cast<const volatile uint32_t*>(flag) == 0u) {
        if (++spins > limit) {
            atomicOr(status, kStatusLookbackTimeout);
            break;
        }
        __nanosleep(32);
    }
    *spinsOut = spins;
}

// ---- the arithmetic peaks a blend's roofline is taken against ---------------
// Eight independent FMA chains a thread, so that every SM's FMA pipes have work
// every cycle; the chains converge to b / (1 - a) and stay normal.
constexpr int kPeakChains = 8;
constexpr int kPeakUnroll = 16;

__global__ void __launch_bounds__(256) fmaPeakKernel(float* out, uint32_t iters, float a, float b) {
    float x[kPeakChains];
#pragma unroll
    for (int k = 0; k < kPeakChains; ++k) x[k] = 1e-3f * (float)(threadIdx.x + k);
    for (uint32_t i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < kPeakUnroll; ++u)
#pragma unroll
            for (int k = 0; k < kPeakChains; ++k) x[k] = fmaf(x[k], a, b);
    }
    float sum = 0.0f;
#pragma unroll
    for (int k = 0; k < kPeakChains; ++k) sum += x[k];
    if (sum == -1.0f) out[blockIdx.x] = sum;   // never true; keeps the chains live
}

// Eight independent chains of the hardware base-2 exponential (the blends'
// ex2.approx), x -> 2^-x, which stays in (0.5, 1].
__global__ void __launch_bounds__(256) ex2PeakKernel(float* out, uint32_t iters) {
    float x[kPeakChains];
#pragma unroll
    for (int k = 0; k < kPeakChains; ++k) x[k] = 1e-3f * (float)(threadIdx.x + k);
    for (uint32_t i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < kPeakUnroll; ++u)
#pragma unroll
            for (int k = 0; k < kPeakChains; ++k) asm volatile("ex2.approx.ftz.f32 %0, %1;" : "=f"(x[k]) : "f"(-x[k]));
    }
    float sum = 0.0f;
#pragma unroll
    for (int k = 0; k < kPeakChains; ++k) sum += x[k];
    if (sum == -1.0f) out[blockIdx.x] = sum;
}

}   // namespace

// The FP32 FMA rate (TFLOP/s, two a fused multiply-add) and the hardware
// exponential's rate (G results/s) of the current device, each the best of
// `repeats` timed launches of a kernel that keeps every SM's pipe busy (eight
// blocks of 256 threads an SM, eight independent chains a thread). What a
// blend kernel's arithmetic rate is measured against.
extern "C" ath_status ath_measure_peaks(uint32_t repeats, double* fma_tflops, double* ex2_gops, void* streamPtr) {
    if (!fma_tflops || !ex2_gops || repeats == 0) return fail(ATH_E_INVALID_ARGUMENT, "ath_measure_peaks: bad argument");
    cudaStream_t stream = static_cast<cudaStream_t>(streamPtr);
    int device = 0, sms = 0;
    cudaError_t err = cudaGetDevice(&device);
    if (err == cudaSuccess) err = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (err != cudaSuccess) return failCuda(err, "ath_measure_peaks");
    const uint32_t blocks = (uint32_t)sms * 8, threads = 256;
    DeviceBuffer sink;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    err = sink.reserve((size_t)blocks * sizeof(float));
    if (err == cudaSuccess) err = cudaEventCreate(&e0);
    if (err == cudaSuccess) err = cudaEventCreate(&e1);
    const uint32_t fmaIters = 4096, ex2Iters = 512;
    double bestFma = 0.0, bestEx2 = 0.0;
    for (uint32_t r = 0; r <= repeats && err == cudaSuccess; ++r) {   // the first of each is a warm-up
        float ms = 0.0f;
        err = cudaEventRecord(e0, stream);
        fmaPeakKernel<<<blocks, threads, 0, stream>>>(static_cast<float*>(sink.ptr), fmaIters, 0.999f, 1e-3f);
        if (err == cudaSuccess) err = cudaEventRecord(e1, stream);
        if (err == cudaSuccess) err = cudaEventSynchronize(e1);
        if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, e0, e1);
        const double flops = 2.0 * kPeakChains * kPeakUnroll * (double)fmaIters * blocks * threads;
        if (err == cudaSuccess && r > 0 && ms > 0.0f) bestFma = std::max(bestFma, flops / (ms * 1e-3) / 1e12);
        if (err == cudaSuccess) err = cudaEventRecord(e0, stream);
        ex2PeakKernel<<<blocks, threads, 0, stream>>>(static_cast<float*>(sink.ptr), ex2Iters);
        if (err == cudaSuccess) err = cudaEventRecord(e1, stream);
        if (err == cudaSuccess) err = cudaEventSynchronize(e1);
        if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, e0, e1);
        const double ops = (double)kPeakChains * kPeakUnroll * (double)ex2Iters * blocks * threads;
        if (err == cudaSuccess && r > 0 && ms > 0.0f) bestEx2 = std::max(bestEx2, ops / (ms * 1e-3) / 1e9);
    }
    if (err == cudaSuccess) err = cudaGetLastError();
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (err != cudaSuccess) return failCuda(err, "ath_measure_peaks");
    *fma_tflops = bestFma;
    *ex2_gops = bestEx2;
    return ATH_OK;
}

extern "C" ath_status ath_check_bounded_wait(uint32_t preset, uint32_t limit, uint32_t* spins, void* streamPtr) {
    if (limit == 0 || limit > kSpinLimit)
        return fail(ATH_E_INVALID_ARGUMENT, "ath_check_bounded_wait: limit must be 1 .. the library's spin limit");
    cudaStream_t stream = static_cast<cudaStream_t>(streamPtr);
    DeviceBuffer words;
    cudaError_t err = words.reserve(4 * sizeof(uint32_t));
    uint32_t host[4] = {preset, 0, 0, 0};   // flag, status, spins
    if (err == cudaSuccess) err = cudaMemcpyAsync(words.ptr, host, sizeof(host), cudaMemcpyHostToDevice, stream);
    uint32_t* w = static_cast<uint32_t*>(words.ptr);
    if (err == cudaSuccess) {
        boundedWaitKernel<<<1, 1, 0, stream>>>(w, limit, w + 1, w + 2);
        err = cudaGetLastError();
    }
    if (err == cudaSuccess) err = cudaMemcpyAsync(host, words.ptr, sizeof(host), cudaMemcpyDeviceToHost, stream);
    if (err == cudaSuccess) err = cudaStreamSynchronize(stream);
    if (err != cudaSuccess) return failCuda(err, "ath_check_bounded_wait");
    if (spins) *spins = host[2];
    if (host[1] & kStatusLookbackTimeout) return fail(ATH_E_TIMEOUT, "the wait gave up after its limit");
    return ATH_OK;
}
