// ctb_backproject_noalloc: the backprojection entry point for callers that
// cannot allocate device memory.
//
// Some host applications cannot let a library call cudaMalloc (or the
// stream-ordered cudaMallocAsync) while they run: an acquisition system that
// reserves all of its GPU memory once at start-up so that a scan in progress
// can never fail with out-of-memory or stall on an allocator, or a program
// whose device memory is entirely owned by another framework's caching
// allocator. ctb_backproject needs a little scratch memory of its own, the
// per-view geometry table ({sin, cos, height} per view, built in FP64 on the
// device from the caller's host arrays), which it allocates and frees on the
// stream at every call. This variant keeps that scratch in one file-scope
// device array instead, so the call itself allocates nothing; the caller still
// passes the filtered projections and the output volume.
//
// Limits and rules:
//  * at most CTB_NOALLOC_MAX_VIEWS views per call (larger calls are rejected
//    with CTB_ERR_UNSUPPORTED before any device work);
//  * the array, 256 KB, exists on every GPU that loads the library and stays
//    there until the process exits;
//  * the first call on a device looks up the array's device address with
//    cudaGetSymbolAddress (with that device current) and caches it. With
//    CUDA's lazy module loading that first lookup is also what loads this
//    library's kernels onto the device, which takes device memory once, so
//    make the first call at start-up, before the memory is handed out and
//    before any stream capture;
//  * the cached address belongs to the context it was looked up in: it is
//    kept together with that context's unique ID, and a call that finds a
//    different context current (after cudaDeviceReset, say) looks it up
//    again, which again belongs at start-up;
//  * every call shares the one array and overwrites the entries it uses, so
//    nothing has to start at zero, but calls whose work overlaps on the GPU
//    (different streams, or concurrent host threads on the same device) race
//    on it: serialise them.

#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <mutex>

#include "ctb_internal.h"

namespace ctb {
namespace {

constexpr int kMaxViews = CTB_NOALLOC_MAX_VIEWS;
constexpr size_t kScratchBytes = size_t(kMaxViews) * (2 * sizeof(double) + sizeof(float4));
constexpr int kMaxDevices = 64;

// [angles_deg: double x kMaxViews][heights_px: double x kMaxViews][views: float4 x kMaxViews]
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_addr_mtx;
void* g_addr[kMaxDevices] = {};
unsigned long long g_ctx_id[kMaxDevices] = {};

// Unique ID of the current context (0 when it cannot be told: no context
// current yet, or a driver without cuCtxGetId).
unsigned long long current_context_id() {
    using GetCurrent = CUresult (*)(CUcontext*);
    using GetId = CUresult (*)(CUcontext, unsigned long long*);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* a = nullptr;
        void* b = nullptr;
        cudaDriverEntryPointQueryResult qa, qb;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &a, cudaEnableDefault, &qa) == cudaSuccess &&
            qa == cudaDriverEntryPointSuccess &&
            cudaGetDriverEntryPoint("cuCtxGetId", &b, cudaEnableDefault, &qb) == cudaSuccess &&
            qb == cudaDriverEntryPointSuccess) {
            get_current = reinterpret_cast<GetCurrent>(a);
            get_id = reinterpret_cast<GetId>(b);
        } else {
            cudaGetLastError();
        }
    });
    CUcontext c = nullptr;
    unsigned long long id = 0;
    if (!get_current || get_current(&c) != CUDA_SUCCESS || !c || get_id(c, &id) != CUDA_SUCCESS) return 0;
    return id;
}

// Device address of the scratch array on the current device: looked up once
// per device (and again if the device's context was replaced).
int scratch_address(void** out) {
    int dev = 0;
    CTB_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) {
        set_global_error("ctb_backproject_noalloc: device index out of range");
        return CTB_ERR_UNSUPPORTED;
    }
    std::lock_guard<std::mutex> lk(g_addr_mtx);
    const unsigned long long id = current_context_id();
    if (!g_addr[dev] || (id != 0 && id != g_ctx_id[dev])) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            set_global_error(std::string("ctb_backproject_noalloc: cudaGetSymbolAddress failed: ") +
                             cudaGetErrorString(e));
            cudaGetLastError();
            return CTB_ERR_CUDA;
        }
        g_addr[dev] = p;
        g_ctx_id[dev] = current_context_id();   // the lookup made the context current if it was not
    }
    *out = g_addr[dev];
    return CTB_OK;
}

}  // namespace
}  // namespace ctb

extern "C" int ctb_backproject_noalloc(const void* filtered, int store_type, int n_views, const double* angles_deg,
                                       const double* height_offsets_px, const ctb_detector* det, const ctb_grid* grid,
                                       int z_begin, int z_end, float load_scale, float* vol, int accumulate,
                                       void* stream) {
    using namespace ctb;
    // the same checks, in the same order, as ctb_backproject
    if (!filtered || !vol || !angles_deg || n_views <= 0 || !valid_detector(det) || !valid_grid(grid)) {
        set_global_error("ctb_backproject_noalloc: invalid arguments");
        return CTB_ERR_ARG;
    }
    if (z_begin < 0 || z_end <= z_begin || z_end > grid->z_to - grid->z_from) {
        set_global_error("ctb_backproject_noalloc: invalid z range");
        return CTB_ERR_ARG;
    }
    if (det->radius <= 0) {
        set_global_error("ctb_backproject_noalloc: detector radius not set (use ctb_reference_grid)");
        return CTB_ERR_ARG;
    }
    if (n_views > kMaxViews) {
        set_global_error("ctb_backproject_noalloc: " + std::to_string(n_views) + " views exceed the limit of " +
                         std::to_string(kMaxViews) + " views per call; split the views into several calls with "
                         "accumulate = 1, or use ctb_backproject");
        return CTB_ERR_UNSUPPORTED;
    }
    void* base = nullptr;
    int st = scratch_address(&base);
    if (st != CTB_OK) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    double* d_ang = static_cast<double*>(base);
    double* d_h = d_ang + kMaxViews;
    float4* d_views = reinterpret_cast<float4*>(d_h + kMaxViews);
    CTB_CUDA_TRY(cudaMemcpyAsync(d_ang, angles_deg, sizeof(double) * n_views, cudaMemcpyHostToDevice, s));
    double hmax = 0;
    if (height_offsets_px) {
        CTB_CUDA_TRY(cudaMemcpyAsync(d_h, height_offsets_px, sizeof(double) * n_views, cudaMemcpyHostToDevice, s));
        for (int i = 0; i < n_views; ++i) hmax = std::max(hmax, std::fabs(height_offsets_px[i]));
    } else {
        CTB_CUDA_TRY(cudaMemsetAsync(d_h, 0, sizeof(double) * n_views, s));
    }
    st = view_table_build(d_ang, d_h, n_views, d_views, s);
    if (st != CTB_OK) return st;
    const ProjGeom g = proj_geom(*det, *grid, z_begin, z_end, load_scale);
    return backproject_launch(filtered, store_type, d_views, n_views, g, hmax, vol, accumulate, s);
}
