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
//    cudaGetSymbolAddress (with that device current) and caches it; make that
//    first call before any stream capture;
//  * every call shares the one array and overwrites the entries it uses, so
//    nothing has to start at zero, but calls whose work overlaps on the GPU
//    (different streams, or concurrent host threads on the same device) race
//    on it: serialise them.

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

// Device address of the scratch array on the current device (set up once per device).
int scratch_address(void** out) {
    int dev = 0;
    CTB_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) {
        set_global_error("ctb_backproject_noalloc: device index out of range");
        return CTB_ERR_UNSUPPORTED;
    }
    std::lock_guard<std::mutex> lk(g_addr_mtx);
    if (!g_addr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            set_global_error(std::string("ctb_backproject_noalloc: cudaGetSymbolAddress failed: ") +
                             cudaGetErrorString(e));
            cudaGetLastError();
            return CTB_ERR_CUDA;
        }
        g_addr[dev] = p;
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
    if (!filtered || !vol || !angles_deg || n_views <= 0 || !det || !grid || det->width <= 1 || det->height <= 1 ||
        !(det->fcd > float(det->width)) || det->radius <= 0 || grid->voxel_pitch <= 0 ||
        grid->x_to <= grid->x_from || grid->y_to <= grid->y_from || grid->z_to <= grid->z_from) {
        set_global_error("ctb_backproject_noalloc: invalid arguments");
        return CTB_ERR_ARG;
    }
    if (n_views > kMaxViews) {
        set_global_error("ctb_backproject_noalloc: " + std::to_string(n_views) + " views exceed the limit of " +
                         std::to_string(kMaxViews) + " views per call; split the views into several calls with "
                         "accumulate = 1, or use ctb_backproject");
        return CTB_ERR_UNSUPPORTED;
    }
    if (z_begin < 0 || z_end <= z_begin || z_end > grid->z_to - grid->z_from) {
        set_global_error("ctb_backproject_noalloc: invalid z range");
        return CTB_ERR_ARG;
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
