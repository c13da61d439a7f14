// errors.cu -- status strings and the per-thread text of the last failure.
#include <string>
#include <cstdio>
#include "common.cuh"

namespace flip {

static thread_local std::string g_error;

void set_error_text(const char* text) { g_error = text ? text : ""; }
const char* error_text() { return g_error.c_str(); }

int set_cuda_error(cudaError_t e, const char* what) {
    char buf[512];
    snprintf(buf, sizeof(buf), "%s failed: %s (%s)", what, cudaGetErrorName(e), cudaGetErrorString(e));
    g_error = buf;
    return e == cudaErrorMemoryAllocation ? FLIP_ERR_OOM : FLIP_ERR_CUDA;
}

}  // namespace flip

extern "C" const char* flip_version(void) { return "flip2_b200 0.1 (sm_100a)"; }

extern "C" const char* flip_status_string(int status) {
    switch (status) {
    case FLIP_OK: return "ok";
    case FLIP_ERR_ARG: return "bad argument";
    case FLIP_ERR_CUDA: return "CUDA error";
    case FLIP_ERR_OOM: return "out of device memory";
    case FLIP_ERR_TIMEOUT: return "bounded device wait timed out";
    case FLIP_ERR_STATE: return "call out of order";
    case FLIP_ERR_NOT_CONVERGED: return "pressure solve did not converge";
    case FLIP_ERR_DEVICE: return "no usable device";
    default: return "unknown status";
    }
}
