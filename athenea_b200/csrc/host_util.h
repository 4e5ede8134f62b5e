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

// The library's device-memory budget (0: none) and what its buffers hold now:
// a buffer that would take the total past the budget fails as out of memory
// (the reference's ATHENEA_GPU_BUDGET, modules/gpu/src/Device.cpp:434-449).
uint64_t memoryBudget();
void memoryHeldAdd(int64_t bytes);
uint64_t memoryHeld();

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
        const size_t size = need ? need : 16;
        const uint64_t budget = memoryBudget();
        if (budget && memoryHeld() + size > budget) return cudaErrorMemoryAllocation;
        const cudaError_t err = cudaMalloc(&ptr, size);
        if (err != cudaSuccess) {
            ptr = nullptr;
            cudaGetLastError();   // clear the sticky-free allocation error
            return err;
        }
        bytes = need;
        memoryHeldAdd((int64_t)size);
        return cudaSuccess;
    }
    void release() {
        if (ptr) {
            cudaFree(ptr);
            memoryHeldAdd(-(int64_t)(bytes ? bytes : 16));
        }
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
