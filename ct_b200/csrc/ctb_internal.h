// Internal declarations shared by the kernels (.cu) and the host runtime (.cpp).
#pragma once

#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/ctb.h"

namespace ctb {

// ----------------------------------------------------------------- errors
// Thread-local message for context-free calls; contexts keep their own copy.
void set_global_error(const std::string& msg);
const std::string& global_error();

// Map a CUDA error to a status, recording the message. Returns CTB_OK on success.
int cuda_status(cudaError_t e, const char* what);

#define CTB_CUDA_TRY(expr)                                      \
    do {                                                        \
        int _st = ::ctb::cuda_status((expr), #expr);            \
        if (_st != CTB_OK) return _st;                          \
    } while (0)

// Raise a kernel's dynamic shared-memory allowance on the current device to
// at least `bytes`. The attribute is per device and shared by all host
// threads, so it is only ever raised: a launch prepared by one thread is never
// invalidated by another thread lowering it.
int ensure_dynamic_smem(const void* kernel, size_t bytes);

// Argument checks shared by the operator entry points.
inline bool valid_detector(const ctb_detector* d) {
    return d && d->width > 1 && d->height > 1 && d->fcd > float(d->width) && d->base_intensity != 0.0f;
}
inline bool valid_grid(const ctb_grid* g) {
    return g && g->x_size > 0 && g->y_size > 0 && g->z_size > 0 && g->x_from >= 0 && g->x_to > g->x_from &&
           g->y_from >= 0 && g->y_to > g->y_from && g->z_from >= 0 && g->z_to > g->z_from && g->voxel_pitch > 0;
}

// Diagnostic: the n-th device or host allocation of the facade from now on
// fails as if memory were exhausted (0 = off).
void fail_allocation_after(long n);

inline size_t store_bytes(int store_type) { return store_type == CTB_FP32 ? 4 : 2; }
inline size_t raw_bytes(int raw_type) { return raw_type == CTB_U8 ? 1 : raw_type == CTB_U16 ? 2 : 4; }

// ----------------------------------------------------------- filter (a)+(b)
// Largest supported transform: the FFT runs one row pair per group of M/8
// threads and a CTA has at most 1024 threads.
constexpr int kMaxFftLen = 8192;

struct FilterPlan {
    int W = 0, pad = 0, filter = -1, M = 0, logM = 0;
    float2* tw = nullptr;   // exp(-2 pi i k / M), k < M   (FP64-built, stored FP32)
    float* K = nullptr;     // real kernel spectrum, M entries (includes scaling)
};

// Transform length for a detector width and padding mode.
int filter_transform_length(int W, int pad);
// Build the twiddle and kernel-spectrum tables on the device (FP64 kernels).
// tw and K must hold M entries each. Stream-ordered.
int filter_build_tables(int W, int pad, int filter, int M, float2* tw, float* K, cudaStream_t s);

// Device tables of a (W, pad, filter) triple on the current device, built on
// first use and kept for the life of the process.
struct FilterTables {
    int M = 0, logM = 0;
    const float2* tw = nullptr;
    const float* K = nullptr;
};
int filter_tables(int W, int pad, int filter, cudaStream_t s, FilterTables* out);

struct FilterArgs {
    int W, H, M, logM;
    long long n_views;
    float alpha, beta, log_scale;   // convertTo alpha/beta and the log pre-scale
    float D, uPre, vPre;            // Feldkamp weight
    float store_scale;
    int out_pitch;                  // elements per filtered row (>= W; padding is left untouched)
    // optional table (device): the Feldkamp weight of every detector pixel;
    // null -> evaluated per pixel
    const float* wt = nullptr;
};

// Build that table (exactly the per-pixel operations, evaluated once).
int build_weight_table(const FilterArgs& a, float* t, cudaStream_t s);
// Process-wide cache of weight tables per device and geometry. With build = 0
// (inside a stream capture) only an existing table is returned; a missing one
// stays null and the filter evaluates the weight per pixel.
int pre_tables(FilterArgs* a, cudaStream_t s, bool build);

// Launch the fused load/log/weight/FFT/window/IFFT/store kernel over n_views.
int filter_launch(const void* raw, int raw_type, void* out, int store_type, const FilterArgs& a,
                  const float2* tw, const float* K, cudaStream_t s);

// Fill FilterArgs from detector geometry (reference preprocessing constants).
FilterArgs filter_args(const ctb_detector& det, int raw_type, int M, int logM, long long n_views,
                       float store_scale);

// --------------------------------------------------------- geometry (FP64)
// Per-view record used by the projector kernels: {sin, cos, heightOffset, 0}.
// sin/cos follow the reference: float angle_rad = (deg/180)*pi, then the sine
// of that float in double precision, rounded to float (Ct/CtVolume.cpp:953-955).
int view_table_build(const double* angles_deg_dev, const double* heights_dev, int n, float4* out,
                     cudaStream_t s);

// Constants of one backprojection / forward projection launch (slab-local).
struct ProjGeom {
    int W, H;
    int X, Y, Zs;
    float xPre, yPre, zPre;     // world = (index - pre) * vs ; zPre relative to slab start
    float vs;
    float D, uOff, r2;
    float lbU, ubU, lbV, ubV, uPre, vPre;
    int z_begin;                // first box z index of the slab
    float zpv;                  // zPre(box) * vs: row lines use box z indices, so a
                                // voxel's row coordinate does not depend on the slabbing
    float vi_hi;                // largest valid row coordinate: float(H - 1.1)
    float load_scale;
    int pitch;                  // elements per projection row (>= W)
    long long view_stride;      // elements between consecutive projections (H * pitch)
};

ProjGeom proj_geom(const ctb_detector& det, const ctb_grid& grid, int z_begin, int z_end, float load_scale);

// The band of detector rows r_lo .. r_lo + rows - 1 that the voxels of box
// slices [z_begin, z_end) reach in any view with the given height offsets
// (pixels), every column of the reconstruction cylinder, with their bilinear
// neighbours and a margin of a few rows; the whole detector when no tighter
// bound applies.
void row_band(const ctb_detector& det, const ctb_grid& grid, int z_begin, int z_end, const double* heights_px,
              int n_views, int* r_lo, int* rows);

// Backprojection of views [0, n) from `views` (device view table) into vol.
// hmax bounds |height offset| (pixels) over the views. Dispatches to the
// shared-memory (TMA) kernel when possible, else to the global-gather kernel.
int bp_pick_zc(int slab_slices);
// Launch shape of the shared-memory backprojector; 0 = the built-in choice.
struct BpConfig {
    int zc = 0;     // z voxels per thread (8, 16 or 32): the block tile's height
    int nbuf = 0;   // projection boxes staged per CTA (2, 3 or 4): views in flight
};
int backproject_launch(const void* proj, int store_type, const float4* views, int n_views,
                       const ProjGeom& g, double hmax, float* vol, int accumulate, cudaStream_t s,
                       BpConfig cfg = BpConfig());
int backproject_global_launch(const void* proj, int store_type, const float4* views, int n_views,
                              const ProjGeom& g, float* vol, int accumulate, cudaStream_t s);
// Returns CTB_ERR_UNSUPPORTED (nothing launched) when the geometry or layout
// does not suit the TMA kernel. zc: z voxels per thread (8, 16 or 32).
int backproject_tma_launch(const void* proj, int store_type, const float4* views, int n_views,
                           const ProjGeom& g, double hmax, float* vol, int accumulate, cudaStream_t s,
                           int zc = 16, int nbuf = 0);

// Persistent multi-scan backprojection: one launch takes (scan, tile) work
// items from a device counter until every scan of the batch is done.
struct BpBatchScan {
    const void* proj;       // filtered projections (row pitch g.pitch)
    const float4* views;    // device view table
    int n_views;
    ProjGeom g;
    double hmax;
    float* vol;             // X-fastest slab of the box
    int accumulate;
};
struct BpBatchPlan {
    int store_type = 0, zc = 16, nbuf = 3, buf_stride = 0, grid = 0;
    size_t smem = 0, desc_size = 0;
    long long total_tiles = 0;
    std::vector<unsigned char> desc;   // descriptors of the included scans (host copy, to be uploaded)
    std::vector<long long> tile_start; // included + 1 prefix sums of tiles
    std::vector<int> included;         // scans handled by the persistent kernel
    std::vector<int> excluded;         // scans whose footprint does not suit it (global-gather kernel)
};
// Builds descriptors (tensor maps, boxes, tile counts) and launch shape for
// every scan that suits the shared-memory kernel; lists the others.
int bp_batch_plan(int store_type, int zc, const BpBatchScan* scans, int n, BpBatchPlan* plan, int nbuf = 0);
// desc / tile_start: device copies of plan.desc / plan.tile_start; queue: a
// device counter that must be zero at launch.
int bp_batch_launch(const BpBatchPlan& plan, const void* desc, const long long* tile_start, int n,
                    unsigned long long* queue, cudaStream_t s);
// Diagnostic: from the next launch on, views whose index is a multiple of
// `every` read their texels through global memory, as views whose footprint
// exceeds the box do (0 = off). Results do not change.
void bp_force_overflow(int every);
// Bounds-checked build: out-of-range texel fetches recorded by the shared-memory
// (TMA) and global-gather backprojectors since the last reset; always 0 in the
// normal build.
int bounds_status_tma(unsigned* count, unsigned long long* first, int reset);
int bounds_status_gather(unsigned* count, unsigned long long* first, int reset);
// Number of CTAs whose bounded mbarrier waits gave up since the last reset.
int device_wait_timeouts(unsigned* count, int reset);
// Run a wait that can never complete with the given try limit (diagnostic of
// the bounded-wait path): CTB_ERR_TIMEOUT when it gave up, as it must.
int bounded_wait_probe_run(unsigned limit, cudaStream_t s);

int forward_launch(const float* vol, const float4* views, int n_views, const ProjGeom& g, float* proj,
                   int accumulate, cudaStream_t s);
// r = a - b (n floats); adds the sum of r^2 to *sumsq (device double)
int residual_launch(const float* a, const float* b, float* r, long long n, double* sumsq, cudaStream_t s);

// ----------------------------------------------------------------- layout
int layout_launch(const float* src, int x, int y, int zs, int index_order, int byte_order, void* dst,
                  cudaStream_t s);

// ---------------------------------------------------------------- phantom
int phantom_launch(const double* ell, int n_ell, const double* angles_deg_dev, const double* heights_mm_dev,
                   int n_views, int W, int H, double pix, double D, double uoff, double* out, cudaStream_t s);

}  // namespace ctb
