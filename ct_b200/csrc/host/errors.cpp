#include <string>

#include "../ctb_internal.h"

namespace ctb {

namespace {
thread_local std::string g_last_error;
}

void set_global_error(const std::string& msg) { g_last_error = msg; }
const std::string& global_error() { return g_last_error; }

int cuda_status(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return CTB_OK;
    g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
    if (e == cudaErrorMemoryAllocation) return CTB_ERR_ALLOC;
    return CTB_ERR_CUDA;
}

}  // namespace ctb
