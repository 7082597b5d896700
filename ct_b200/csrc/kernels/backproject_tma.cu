// Kernel (c), shared-memory staged variant: the view footprint of a CTA's
// voxel tile is brought into shared memory by one TMA box load per view,
// triple buffered behind mbarriers, and the bilinear texels are then read
// from shared memory instead of through L1 gathers.
//
// Tile: 32 (x) x 8 (y) columns x ZC (z) voxels per CTA, one column of ZC
// voxels per thread (sums in registers across all views, as in the global
// variant). For every view, warp 0 projects the 4 (x, y) corners of the tile
// at the two z extremes with the same arithmetic as the voxels (u is a
// linear-fractional function of (x, y), v is monotone in z and U, so the
// extremes sit at the corners), rounds the box origin down to a 16-byte
// aligned column, and lane 0 issues cp.async.bulk.tensor.3d for the box
// [u0, u0 + BU) x [v0, v0 + BV) of view iv. Boxes that reach outside the
// detector read zeros (TMA out-of-bounds fill) which no in-bounds voxel uses.
// A view whose footprint would not fit the box (BU, BV are host-side bounds
// with margins) is flagged and read through global memory instead.
//
// Every mbarrier wait is bounded; a CTA that gives up records the failure in a
// device counter (read by ctb_device_status) and stops issuing work.
// No multicast is used anywhere.

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cudaTypedefs.h>

#include <mutex>

#include "../ctb_internal.h"
#include "geom.cuh"

namespace ctb {

__device__ unsigned int g_wait_timeouts = 0;

namespace {

constexpr int kTX = 32, kTY = 8, kNBuf = 3;
constexpr unsigned kWaitLimit = 1u << 26;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int c0, int c1, int c2,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
        : "memory");
}

template <typename T> __device__ __forceinline__ float sval(T v);
template <> __device__ __forceinline__ float sval<float>(float v) { return v; }
template <> __device__ __forceinline__ float sval<__half>(__half v) { return __half2float(v); }
template <> __device__ __forceinline__ float sval<__nv_bfloat16>(__nv_bfloat16 v) { return __bfloat162float(v); }

template <typename T> __device__ __forceinline__ float gval(const T* p);
template <> __device__ __forceinline__ float gval<float>(const float* p) { return __ldg(p); }
template <> __device__ __forceinline__ float gval<__half>(const __half* p) { return __half2float(__ldg(p)); }
template <> __device__ __forceinline__ float gval<__nv_bfloat16>(const __nv_bfloat16* p) {
    return __bfloat162float(__ldg(p));
}

struct Box {
    int BU, BV;          // box columns / rows (elements)
    int buf_elems;       // elements per buffer (BU * BV rounded to 128 bytes)
    float vi_hi;         // upper bound of the row coordinate: float(H - 1.1)
};

template <typename T, int ZC>
__global__ void __launch_bounds__(kTX * kTY) bp_tma_kernel(const __grid_constant__ CUtensorMap map,
                                                           const T* __restrict__ proj,
                                                           const float4* __restrict__ views, int n_views,
                                                           ProjGeom g, Box bx, float* __restrict__ vol,
                                                           int accumulate) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t mbar[kNBuf];
    __shared__ int2 org[kNBuf];
    __shared__ int ovf[kNBuf];
    __shared__ int abort_flag;
    T* buf = reinterpret_cast<T*>(smem_raw);

    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * kTX + tx;
    const int warp = tid >> 5, lane = tid & 31;
    const int x0 = blockIdx.x * kTX, y0 = blockIdx.y * kTY, z0 = blockIdx.z * ZC;
    const int x = x0 + tx, y = y0 + ty;
    const float xw = world_coord(x, g.xPre, g.vs);
    const float yw = world_coord(y, g.yPre, g.vs);
    const bool live = x < g.X && y < g.Y && in_cylinder(xw, yw, g.r2);
    const int zl = min(ZC, g.Zs - z0);  // voxels of this tile in the slab

    float zw[ZC];
#pragma unroll
    for (int j = 0; j < ZC; ++j) zw[j] = world_coord(z0 + j, g.zPre, g.vs);
    float acc[ZC];
#pragma unroll
    for (int j = 0; j < ZC; ++j) acc[j] = 0.0f;

    if (tid == 0) {
        for (int i = 0; i < kNBuf; ++i) mbar_init(&mbar[i], 1);
        abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    // corner footprint of view iv -> box origin, then the TMA load (warp 0)
    // the whole ZC tile is evaluated (voxels past the slab end are discarded
    // at the store), so the footprint covers all ZC z positions
    const float zlo = zw[0], zhi = zw[ZC - 1];
    int issued = 0;  // views whose box load has been issued (tracked by warp 0)
    auto issue = [&](int iv) {
        const int b = iv % kNBuf;
        issued = iv + 1;
        float umin = 3.0e38f, umax = -3.0e38f, vmin = 3.0e38f, vmax = -3.0e38f;
        if (lane < 4) {
            const int cx = min(x0 + (lane & 1) * (kTX - 1), g.X - 1);
            const int cy = min(y0 + (lane >> 1) * (kTY - 1), g.Y - 1);
            const float4 q = __ldg(&views[iv]);
            float U, u;
            column_geom(world_coord(cx, g.xPre, g.vs), world_coord(cy, g.yPre, g.vs), q.x, q.y, g.D, g.uOff, &U,
                        &u);
            const float ui = __fadd_rn(u, g.uPre);
            float v;
            const float va = row_coord(zlo, q.z, U, g.vPre, &v);
            const float vb = row_coord(zhi, q.z, U, g.vPre, &v);
            umin = umax = ui;
            vmin = fminf(va, vb);
            vmax = fmaxf(va, vb);
        }
#pragma unroll
        for (int o = 1; o < 4; o <<= 1) {
            umin = fminf(umin, __shfl_xor_sync(0xffffffffu, umin, o));
            umax = fmaxf(umax, __shfl_xor_sync(0xffffffffu, umax, o));
            vmin = fminf(vmin, __shfl_xor_sync(0xffffffffu, vmin, o));
            vmax = fmaxf(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
        }
        if (lane == 0) {
            // clamp non-finite / huge values so the integer conversions stay defined
            umin = fminf(fmaxf(umin, -1.0e6f), 1.0e6f); umax = fminf(fmaxf(umax, -1.0e6f), 1.0e6f);
            vmin = fminf(fmaxf(vmin, -1.0e6f), 1.0e6f); vmax = fminf(fmaxf(vmax, -1.0e6f), 1.0e6f);
            const int uo = ((int(floorf(umin)) - 2) >> 3) << 3;   // 16-byte aligned column
            const int vo = int(floorf(vmin)) - 2;
            org[b] = make_int2(uo, vo);
            ovf[b] = (int(floorf(umax)) + 3 - uo > bx.BU) || (int(floorf(vmax)) + 3 - vo > bx.BV);
            mbar_expect_tx(&mbar[b], uint32_t(bx.BU) * bx.BV * sizeof(T));
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            tma_load_3d(buf + size_t(b) * bx.buf_elems, &map, uo, vo, iv, &mbar[b]);
        }
    };

    if (warp == 0)
        for (int i = 0; i < kNBuf - 1 && i < n_views; ++i) issue(i);

    int abort_iv = n_views;
    for (int iv = 0; iv < n_views; ++iv) {
        const int b = iv % kNBuf;
        if (warp == 0 && iv + kNBuf - 1 < n_views) issue(iv + kNBuf - 1);
        // bounded wait for the box of view iv
        unsigned tries = 0;
        while (!mbar_try_wait(&mbar[b], uint32_t((iv / kNBuf) & 1))) {
            if (++tries > kWaitLimit) {
                abort_flag = 1;
                break;
            }
        }
        if (live && !abort_flag) {
            const float4 q = __ldg(&views[iv]);
            float U, u;
            column_geom(xw, yw, q.x, q.y, g.D, g.uOff, &U, &u);
            if (u >= g.lbU && u <= g.ubU) {
                const float w = __fmul_rn(__fmul_rn(U, U), g.load_scale);
                const float ui = __fadd_rn(u, g.uPre);
                const int u0 = int(ui);
                const float fu = __fsub_rn(ui, float(u0));
                const int2 o = org[b];
                float v;
                const float vi_first = row_coord(zw[0], q.z, U, g.vPre, &v);
                const float vi_last = row_coord(zw[ZC - 1], q.z, U, g.vPre, &v);
                // strictly inside the row bounds (half-pixel margin): every voxel of the column passes the
                // per-voxel test, so the fast path and the checked path take the same decisions
                const bool all_rows =
                    fminf(vi_first, vi_last) >= 0.5f && fmaxf(vi_first, vi_last) <= bx.vi_hi - 0.5f;
                if (!ovf[b]) {
                    const T* col = buf + size_t(b) * bx.buf_elems + (u0 - o.x) - o.y * bx.BU;
#pragma unroll
                    for (int j = 0; j < ZC; ++j) {
                        const float vi = row_coord(zw[j], q.z, U, g.vPre, &v);
                        if (all_rows || (v >= g.lbV && v <= g.ubV)) {
                            const int v0 = int(vi);
                            const float fv = __fsub_rn(vi, float(v0));
                            const T* r0 = col + v0 * bx.BU;
                            const float p00 = sval(r0[0]), p01 = sval(r0[1]);
                            const float p10 = sval(r0[bx.BU]), p11 = sval(r0[bx.BU + 1]);
                            const float a = fmaf(fu, p01 - p00, p00);
                            const float c = fmaf(fu, p11 - p10, p10);
                            acc[j] = fmaf(w, fmaf(fv, c - a, a), acc[j]);
                        }
                    }
                } else {
                    const T* col = proj + (long long)iv * g.view_stride + u0;
#pragma unroll
                    for (int j = 0; j < ZC; ++j) {
                        const float vi = row_coord(zw[j], q.z, U, g.vPre, &v);
                        if (v >= g.lbV && v <= g.ubV) {
                            const int v0 = int(vi);
                            const float fv = __fsub_rn(vi, float(v0));
                            const T* r0 = col + (long long)v0 * g.W;
                            const float a = fmaf(fu, gval(r0 + 1) - gval(r0), gval(r0));
                            const float c = fmaf(fu, gval(r0 + g.W + 1) - gval(r0 + g.W), gval(r0 + g.W));
                            acc[j] = fmaf(w, fmaf(fv, c - a, a), acc[j]);
                        }
                    }
                }
            }
        }
        __syncthreads();
        if (abort_flag) {
            abort_iv = iv;
            break;
        }
    }
    if (abort_flag) {
        if (tid == 0) {
            atomicAdd(&g_wait_timeouts, 1u);
            // bounded drain of the boxes issued but not consumed (views abort_iv .. issued-1)
            // before the CTA's shared memory goes away
            for (int i = abort_iv; i < issued; ++i) {
                unsigned tries = 0;
                while (!mbar_try_wait(&mbar[i % kNBuf], uint32_t((i / kNBuf) & 1)) && ++tries < kWaitLimit) {
                }
            }
        }
        return;
    }
    if (x >= g.X || y >= g.Y) return;
    const long long plane = (long long)g.X * g.Y;
    float* out = vol + (long long)z0 * plane + (long long)y * g.X + x;
#pragma unroll
    for (int j = 0; j < ZC; ++j) {
        if (j < zl) {
            float* p = out + j * plane;
            *p = accumulate ? (*p + acc[j]) : acc[j];
        }
    }
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        else
            cudaGetLastError();
    });
    return fn;
}

// Host-side bound of the per-view footprint of one tile (with margins).
bool box_dims(const ProjGeom& g, int ZC, double hmax, int esize, Box* b) {
    const double D = g.D, vs = g.vs;
    // largest |(x, y)| of any grid column
    const double xa = std::max(std::fabs((0 - g.xPre) * vs), std::fabs((g.X - 1 - g.xPre) * vs));
    const double ya = std::max(std::fabs((0 - g.yPre) * vs), std::fabs((g.Y - 1 - g.yPre) * vs));
    const double R = std::sqrt(xa * xa + ya * ya);
    if (R >= 0.9 * D) return false;
    const double Umax = D / (D - R), dU = Umax * Umax / D;
    const double T = std::sqrt(std::pow((kTX - 1) * vs, 2) + std::pow((kTY - 1) * vs, 2));
    const double tmax = R + std::fabs(g.uOff);
    const double uext = Umax * T + tmax * dU * T;
    const double zabs =
        std::max(std::fabs((0 - g.zPre) * vs), std::fabs((g.Zs + ZC - 1 - g.zPre) * vs)) + hmax;
    const double vext = (ZC - 1) * vs * Umax + zabs * dU * T;
    int BU = int(std::ceil(uext)) + 12;
    BU = (BU + 7) / 8 * 8;
    const int BV = int(std::ceil(vext)) + 6;
    if (BU > 256 || BV > 256) return false;
    b->BU = BU;
    b->BV = BV;
    const int per128 = 128 / esize;
    b->buf_elems = (BU * BV + per128 - 1) / per128 * per128;
    b->vi_hi = float(double(g.H) - 1 - 0.1);
    return true;
}

template <typename T>
int launch_t(const T* proj, CUtensorMapDataType dt, const float4* views, int n_views, const ProjGeom& g,
             double hmax, float* vol, int accumulate, cudaStream_t s) {
    constexpr int ZC = 16;
    Box bx;
    if (!box_dims(g, ZC, hmax, sizeof(T), &bx)) return CTB_ERR_UNSUPPORTED;
    if ((g.W * sizeof(T)) % 16 != 0 || (reinterpret_cast<uintptr_t>(proj) & 15) != 0) return CTB_ERR_UNSUPPORTED;
    auto enc = encode_fn();
    if (!enc) return CTB_ERR_UNSUPPORTED;
    CUtensorMap map;
    const cuuint64_t dims[3] = {cuuint64_t(g.W), cuuint64_t(g.H), cuuint64_t(n_views)};
    const cuuint64_t strides[2] = {cuuint64_t(g.W) * sizeof(T), cuuint64_t(g.view_stride) * sizeof(T)};
    const cuuint32_t box[3] = {cuuint32_t(bx.BU), cuuint32_t(bx.BV), 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    if (enc(&map, dt, 3, const_cast<T*>(proj), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return CTB_ERR_UNSUPPORTED;
    const size_t smem = size_t(kNBuf) * bx.buf_elems * sizeof(T);
    auto kern = bp_tma_kernel<T, ZC>;
    if (smem > 200 * 1024) return CTB_ERR_UNSUPPORTED;
    CTB_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    dim3 block(kTX, kTY, 1);
    dim3 grid((g.X + kTX - 1) / kTX, (g.Y + kTY - 1) / kTY, (g.Zs + ZC - 1) / ZC);
    if (grid.y > 65535 || grid.z > 65535) return CTB_ERR_UNSUPPORTED;
    kern<<<grid, block, smem, s>>>(map, proj, views, n_views, g, bx, vol, accumulate);
    return cuda_status(cudaGetLastError(), "bp_tma_kernel launch");
}

}  // namespace

int backproject_tma_launch(const void* proj, int store_type, const float4* views, int n_views, const ProjGeom& g,
                           double hmax, float* vol, int accumulate, cudaStream_t s) {
    if (n_views <= 0) return CTB_ERR_UNSUPPORTED;
    switch (store_type) {
        case CTB_FP32:
            return launch_t((const float*)proj, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, views, n_views, g, hmax, vol,
                            accumulate, s);
        case CTB_FP16:
            return launch_t((const __half*)proj, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, views, n_views, g, hmax, vol,
                            accumulate, s);
        case CTB_BF16:
            return launch_t((const __nv_bfloat16*)proj, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, views, n_views, g, hmax,
                            vol, accumulate, s);
    }
    return CTB_ERR_UNSUPPORTED;
}

int device_wait_timeouts(unsigned* count, int reset) {
    CTB_CUDA_TRY(cudaMemcpyFromSymbol(count, g_wait_timeouts, sizeof(unsigned)));
    if (reset && *count) {
        const unsigned zero = 0;
        CTB_CUDA_TRY(cudaMemcpyToSymbol(g_wait_timeouts, &zero, sizeof(unsigned)));
    }
    return CTB_OK;
}

}  // namespace ctb
