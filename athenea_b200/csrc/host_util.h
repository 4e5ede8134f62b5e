// Host-side helpers of the C ABI: owned device and pinned buffers, and the
// thread-local error message every ath_status comes with.
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>

#include <cuda_runtime.h>

#include "../../include/athenea_raster.h"

namespace ath {

constexpr uint32_t kTileSize = 16;

// Records `message` as this thread's last error and returns `status`.
ath_status fail(ath_status status, const std::string& message);
// A CUDA error as an ath_status: out of memory, or a device failure.
ath_status failCuda(cudaError_t err, const char* what);

// Device memory that grows and never shrinks until released.
struct DeviceBuffer {
    void* ptr = nullptr;
    size_t bytes = 0;
    DeviceBuffer() = default;
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    ~DeviceBuffer() { release(); }
    cudaError_t reserve(size_t need) {
        if (need <= bytes && ptr) return cudaSuccess;
        release();
        const cudaError_t err = cudaMalloc(&ptr, need ? need : 16);
        if (err != cudaSuccess) {
            ptr = nullptr;
            cudaGetLastError();   // clear the sticky-free allocation error
            return err;
        }
        bytes = need;
        return cudaSuccess;
    }
    void release() {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
    }
};

// Page-locked host memory for the copies a frame waits on.
struct PinnedBuffer {
    void* ptr = nullptr;
    size_t bytes = 0;
    PinnedBuffer() = default;
    PinnedBuffer(const PinnedBuffer&) = delete;
    PinnedBuffer& operator=(const PinnedBuffer&) = delete;
    ~PinnedBuffer() { release(); }
    cudaError_t reserve(size_t need) {
        if (need <= bytes && ptr) return cudaSuccess;
        release();
        const cudaError_t err = cudaMallocHost(&ptr, need ? need : 16);
        if (err != cudaSuccess) {
            ptr = nullptr;
            cudaGetLastError();
            return err;
        }
        bytes = need;
        return cudaSuccess;
    }
    void release() {
        if (ptr) cudaFreeHost(ptr);
        ptr = nullptr;
        bytes = 0;
    }
};

}   // namespace ath
