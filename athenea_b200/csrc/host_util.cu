// The thread-local error message behind ath_last_error_message, and the
// library's device-memory budget.
#include <atomic>
#include <cstdlib>
#include <string>

#include "host_util.h"

namespace {
thread_local std::string g_message;

std::atomic<uint64_t> g_held{0};

std::atomic<uint64_t>& budgetWord() {
    // ATHENEA_GPU_BUDGET, in MiB, read once (modules/gpu/src/Device.cpp:434-449)
    static std::atomic<uint64_t> budget{[] {
        const char* env = std::getenv("ATHENEA_GPU_BUDGET");
        if (!env || !*env) return uint64_t{0};
        char* end = nullptr;
        const unsigned long long mib = std::strtoull(env, &end, 10);
        return end && *end == '\0' && mib > 0 ? uint64_t{mib} << 20 : uint64_t{0};
    }()};
    return budget;
}
}   // namespace

namespace ath {

ath_status fail(ath_status status, const std::string& message) {
    g_message = message;
    return status;
}

ath_status failCuda(cudaError_t err, const char* what) {
    const ath_status status = err == cudaErrorMemoryAllocation ? ATH_E_OUT_OF_MEMORY : ATH_E_DEVICE_FAILURE;
    return fail(status, std::string(what) + ": " + cudaGetErrorName(err) + " (" + cudaGetErrorString(err) + ")");
}

uint64_t memoryBudget() { return budgetWord().load(std::memory_order_relaxed); }
void memoryHeldAdd(int64_t bytes) { g_held.fetch_add((uint64_t)bytes, std::memory_order_relaxed); }
uint64_t memoryHeld() { return g_held.load(std::memory_order_relaxed); }

}   // namespace ath

extern "C" const char* ath_last_error_message(void) { return g_message.c_str(); }

extern "C" ath_status ath_set_memory_budget(uint64_t bytes) {
    budgetWord().store(bytes, std::memory_order_relaxed);
    return ATH_OK;
}

extern "C" ath_status ath_memory_held(uint64_t* bytes, uint64_t* budget) {
    if (bytes) *bytes = ath::memoryHeld();
    if (budget) *budget = ath::memoryBudget();
    return ATH_OK;
}
