// Failure detection without a fault. Every device-side wait in this library
// (the decoupled look-backs of the projection's scan, of the sort and of the
// batched step, and the persistent tile queues' tickets) spins a bounded number
// of times; past it the kernel sets a status bit and returns, and the host
// reports ATH_E_TIMEOUT with the context still usable. ath_check_bounded_wait
// runs that same shape of wait on a flag the caller may leave unset, so that a
// test can make the wait run out and see the status come back.
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

}   // namespace

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
