#include <map>
#include <mutex>
#include <string>
#include <utility>

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

int ensure_dynamic_smem(const void* kernel, size_t bytes) {
    static std::mutex m;
    static std::map<std::pair<int, const void*>, size_t> set;
    int dev = 0;
    CTB_CUDA_TRY(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(m);
    size_t& cur = set[{dev, kernel}];
    if (bytes <= cur) return CTB_OK;
    CTB_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)));
    cur = bytes;
    return CTB_OK;
}

}  // namespace ctb
