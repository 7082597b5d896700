// Kernel (c): voxel-driven FDK backprojection, and the FP64 per-view geometry.
//
// Reference semantics: reconstructionCore (Ct/CtVolume.cpp:923-1046, CPU, the
// parity target) and reconstructionKernel (Ct/cuda_ct.cu:201-292, GPU):
//   x,y,z world = index - pre            (updateBoundaries :1419-1421)
//   cylinder    x^2 + y^2 < radius^2     (:980)
//   t = -x sin + y cos + uOffset, s = x cos + y sin, U = D/(D - s), u = t U
//   u in [-W/2, W-1.1-W/2]               (:998, bounds :924-925)
//   v = (z + h) U in [1.1-H/2+..., H/2]  (:1008-1011, bounds :927-928)
//   bilinear at (u + W/2, -v + H/2), weight U^2, vol += U^2 * value
//
// Design (B200): one thread owns an (x, y) column of ZC consecutive z voxels
// and keeps their sums in registers across every view of the launch, so the
// volume is written once per launch instead of read-modify-written per view
// (the reference launches once per view). u, U and U^2 depend only on
// (x, y, view) and are computed once per view for the whole column; per voxel
// only v, the row index and the bilinear sample remain. The per-view table
// {sin, cos, h} is built in FP64 on the device and staged into shared memory
// once per CTA. Warps run along x, so each z row of stores is one coalesced
// 128-byte segment of the X-fastest slab.

#include <cuda_bf16.h>
#include <cstdlib>
#include <cstring>
#include <cuda_fp16.h>

#include "../ctb_internal.h"
#include "geom.cuh"

namespace ctb {

namespace {

__global__ void view_table_kernel(const double* __restrict__ ang, const double* __restrict__ h, int n,
                                  float4* __restrict__ out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    // float angle_rad = (angle / 180.0) * M_PI; sine = sin(angle_rad) (:953-955)
    const float angle_rad = float((ang[i] / 180.0) * 3.14159265358979323846);
    double s, c;
    sincos(double(angle_rad), &s, &c);
    out[i] = make_float4(float(s), float(c), float(h[i]), 0.0f);
}

template <typename T> __device__ __forceinline__ float ld(const T* p);
template <> __device__ __forceinline__ float ld<float>(const float* p) { return __ldg(p); }
template <> __device__ __forceinline__ float ld<__half>(const __half* p) { return __half2float(__ldg(p)); }
template <> __device__ __forceinline__ float ld<__nv_bfloat16>(const __nv_bfloat16* p) {
    return __bfloat162float(__ldg(p));
}

constexpr int kBX = 32, kBY = 4;
constexpr int kViewsPerStage = 1024;   // shared-memory view table capacity (16 KB)

template <typename T, int ZC>
__global__ void __launch_bounds__(kBX * kBY) bp_kernel(const T* __restrict__ proj,
                                                       const float4* __restrict__ views, int n_views,
                                                       ProjGeom g, float* __restrict__ vol, int accumulate) {
    __shared__ float4 sviews[kViewsPerStage];
    const int x = blockIdx.x * kBX + threadIdx.x;
    const int y = blockIdx.y * kBY + threadIdx.y;
    const int z0 = blockIdx.z * ZC;
    const int tid = threadIdx.y * kBX + threadIdx.x;

    const float xw = world_coord(x, g.xPre, g.vs);
    const float yw = world_coord(y, g.yPre, g.vs);
    const bool live = x < g.X && y < g.Y && in_cylinder(xw, yw, g.r2);

    float acc[ZC];
#pragma unroll
    for (int j = 0; j < ZC; ++j) acc[j] = 0.0f;

    for (int vb = 0; vb < n_views; vb += kViewsPerStage) {
        const int nv = min(kViewsPerStage, n_views - vb);
        __syncthreads();
        for (int i = tid; i < nv; i += kBX * kBY) sviews[i] = __ldg(&views[vb + i]);
        __syncthreads();
        if (!live) continue;
        const T* pv = proj + (long long)vb * g.view_stride;
        for (int iv = 0; iv < nv; ++iv, pv += g.view_stride) {
            const float4 q = sviews[iv];  // sin, cos, h
            float U, u;
            column_geom(xw, yw, q.x, q.y, g.D, g.uOff, &U, &u);
            if (!(u >= g.lbU && u <= g.ubU)) continue;
            const float w = __fmul_rn(__fmul_rn(U, U), g.load_scale);
            const float ui = __fadd_rn(u, g.uPre);
            const int u0 = int(ui);
            const float fu = __fsub_rn(ui, float(u0));
#ifdef CTB_BOUNDS_CHECK
            const T* col = pv + (CTB_FETCH_OK(u0, g.W - 1, 6) ? u0 : 0);
#else
            const T* col = pv + u0;
#endif
            const RowLine rl = row_line(U, q.z, g.zpv, g.vs, g.vPre);
#pragma unroll
            for (int j = 0; j < ZC; ++j) {
                const float vi = row_at(rl, g.z_begin + z0 + j);
                const float zw = __fmul_rn(__fsub_rn(float(z0 + j), g.zPre), g.vs);
                if (v_inside(zw, q.z, U, g.lbV, g.ubV)) {
                    int v0 = int(vi);
                    const float fv = __fsub_rn(vi, float(v0));
#ifdef CTB_BOUNDS_CHECK
                    if (!CTB_FETCH_OK(v0, g.H - 1, 7)) v0 = 0;
#endif
                    const T* r0 = col + (long long)v0 * g.pitch;
                    const float a = (1.0f - fu) * ld(r0) + fu * ld(r0 + 1);
                    const float b = (1.0f - fu) * ld(r0 + g.pitch) + fu * ld(r0 + g.pitch + 1);
                    acc[j] += w * ((1.0f - fv) * a + fv * b);
                }
            }
        }
    }
    if (x >= g.X || y >= g.Y) return;
    const long long plane = (long long)g.X * g.Y;
    float* out = vol + (long long)z0 * plane + (long long)y * g.X + x;
#pragma unroll
    for (int j = 0; j < ZC; ++j) {
        if (z0 + j < g.Zs) {
            float* p = out + j * plane;
            *p = accumulate ? (*p + acc[j]) : acc[j];
        }
    }
}

template <typename T>
int bp_launch_typed(const T* proj, const float4* views, int n_views, const ProjGeom& g, float* vol,
                    int accumulate, cudaStream_t s) {
    constexpr int ZC = 16;
    dim3 block(kBX, kBY, 1);
    dim3 grid((g.X + kBX - 1) / kBX, (g.Y + kBY - 1) / kBY, (g.Zs + ZC - 1) / ZC);
    if (grid.x == 0 || grid.y == 0 || grid.z == 0) return CTB_OK;
    if (grid.z > 65535 || grid.y > 65535) {
        set_global_error("backproject: grid too large");
        return CTB_ERR_UNSUPPORTED;
    }
    bp_kernel<T, ZC><<<grid, block, 0, s>>>(proj, views, n_views, g, vol, accumulate);
    return cuda_status(cudaGetLastError(), "bp_kernel launch");
}

}  // namespace

int bounds_status_gather(unsigned* count, unsigned long long* first, int reset) {
#ifdef CTB_BOUNDS_CHECK
    CTB_CUDA_TRY(cudaMemcpyFromSymbol(count, g_bounds_count, sizeof(unsigned)));
    CTB_CUDA_TRY(cudaMemcpyFromSymbol(first, g_bounds_first, sizeof(unsigned long long)));
    if (reset) {
        const unsigned z = 0;
        const unsigned long long zz = 0;
        CTB_CUDA_TRY(cudaMemcpyToSymbol(g_bounds_count, &z, sizeof z));
        CTB_CUDA_TRY(cudaMemcpyToSymbol(g_bounds_first, &zz, sizeof zz));
    }
#else
    (void)reset;
    *count = 0;
    *first = 0;
#endif
    return CTB_OK;
}

int view_table_build(const double* angles_deg_dev, const double* heights_dev, int n, float4* out,
                     cudaStream_t s) {
    if (n <= 0) return CTB_OK;
    view_table_kernel<<<(n + 127) / 128, 128, 0, s>>>(angles_deg_dev, heights_dev, n, out);
    return cuda_status(cudaGetLastError(), "view_table_kernel launch");
}

static inline float __fmul_rn_host(float a, float b) { return a * b; }

ProjGeom proj_geom(const ctb_detector& det, const ctb_grid& grid, int z_begin, int z_end, float load_scale) {
    ProjGeom g;
    g.W = det.width;
    g.H = det.height;
    g.X = grid.x_to - grid.x_from;
    g.Y = grid.y_to - grid.y_from;
    g.Zs = z_end - z_begin;
    // updateBoundaries :1419-1423 (double expressions stored as float)
    g.xPre = float(float(grid.x_size) / 2.0 - float(grid.x_from));
    g.yPre = float(float(grid.y_size) / 2.0 - float(grid.y_from));
    const float zPre = float(float(grid.z_size) / 2.0 - float(grid.z_from));
    g.zPre = zPre - float(z_begin);
    g.vs = grid.voxel_pitch;
    g.D = det.fcd;
    g.uOff = det.u_offset;
    g.r2 = det.radius * det.radius;
    g.uPre = float(double(det.width) / 2.0);
    g.vPre = float(double(det.height) / 2.0);
    // reconstructionCore :924-928
    g.lbU = 0.0f - g.uPre;
    g.ubU = float(double(det.width) - 1 - 0.1) - g.uPre;
    g.lbV = (-1) * float(double(det.height) - 1 - 0.1) + g.vPre;
    g.ubV = (-1) * 0.0f + g.vPre;
    g.z_begin = z_begin;
    g.zpv = __fmul_rn_host(zPre, g.vs);
    g.vi_hi = float(double(det.height) - 1 - 0.1);
    g.load_scale = load_scale;
    g.pitch = det.width;
    g.view_stride = (long long)det.width * det.height;
    return g;
}

// z voxels per thread of the shared-memory backprojector: 32 spreads each
// column's per-view geometry over twice the voxels of 16 (8% faster on the
// 128-slice slabs of a 1024^3 volume, with 3 instead of 4 CTAs per SM; 64
// at 2 CTAs per SM was slower again) when the slab holds whole tiles of 32
// with at most 1/8 padding; thinner slabs take 16, or 8 for 8 slices or fewer.
int bp_pick_zc(int Zs) {
    for (int zc : {32, 16}) {
        const int padded = (Zs + zc - 1) / zc * zc;
        if (Zs >= 2 * zc && (padded - Zs) * 8 <= padded) return zc;
    }
    return Zs <= 8 ? 8 : 16;
}

int backproject_launch(const void* proj, int store_type, const float4* views, int n_views,
                       const ProjGeom& g, double hmax, float* vol, int accumulate, cudaStream_t s, BpConfig cfg) {
    // shared-memory staged kernel when the footprint bound and the 16-byte TMA
    // stride rule allow it; the global-gather kernel otherwise.
    // CTB_BP_VARIANT=global|tma forces one of them (tma fails when ineligible).
    static const int variant = [] {
        const char* e = std::getenv("CTB_BP_VARIANT");
        if (!e) return 0;
        if (!std::strcmp(e, "global")) return 1;
        if (!std::strcmp(e, "tma")) return 2;
        return 0;
    }();
    // CTB_BP_ZC=8|16|32 fixes the z voxels per thread of the shared-memory kernel
    static const int zc_env = [] {
        const char* e = std::getenv("CTB_BP_ZC");
        const int v = e ? std::atoi(e) : 0;
        return (v == 8 || v == 16 || v == 32) ? v : 0;
    }();
    if (variant != 1) {
        const int zc = zc_env ? zc_env : cfg.zc ? cfg.zc : bp_pick_zc(g.Zs);
        int st = backproject_tma_launch(proj, store_type, views, n_views, g, hmax, vol, accumulate, s, zc, cfg.nbuf);
        // a taller tile's footprint may exceed the box limits where a shorter one fits
        if (st == CTB_ERR_UNSUPPORTED && !zc_env && zc > 16)
            st = backproject_tma_launch(proj, store_type, views, n_views, g, hmax, vol, accumulate, s, 16);
        if (st != CTB_ERR_UNSUPPORTED || variant == 2) return st;
    }
    return backproject_global_launch(proj, store_type, views, n_views, g, vol, accumulate, s);
}

int backproject_global_launch(const void* proj, int store_type, const float4* views, int n_views,
                              const ProjGeom& g, float* vol, int accumulate, cudaStream_t s) {
    switch (store_type) {
        case CTB_FP32: return bp_launch_typed((const float*)proj, views, n_views, g, vol, accumulate, s);
        case CTB_FP16: return bp_launch_typed((const __half*)proj, views, n_views, g, vol, accumulate, s);
        case CTB_BF16:
            return bp_launch_typed((const __nv_bfloat16*)proj, views, n_views, g, vol, accumulate, s);
    }
    set_global_error("backproject: unknown storage type");
    return CTB_ERR_ARG;
}

}  // namespace ctb
