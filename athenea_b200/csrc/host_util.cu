// The thread-local error message behind ath_last_error_message.
#include <string>

#include "host_util.h"

namespace {
thread_local std::string g_message;
}

namespace ath {

ath_status fail(ath_status status, const std::string& message) {
    g_message = message;
    return status;
}

ath_status failCuda(cudaError_t err, const char* what) {
    const ath_status status = err == cudaErrorMemoryAllocation ? ATH_E_OUT_OF_MEMORY : ATH_E_DEVICE_FAILURE;
    return fail(status, std::string(what) + ": " + cudaGetErrorName(err) + " (" + cudaGetErrorString(err) + ")");
}

}   // namespace ath

extern "C" const char* ath_last_error_message(void) { return g_message.c_str(); }
