// Kernel (c), shared-memory staged variant: the view footprint of a CTA's
// voxel tile is brought into shared memory by one TMA box load per view,
// triple buffered behind mbarriers, and the bilinear texels are then read
// from shared memory instead of through L1 gathers.
//
// Tile: 16 (x) x 16 (y) columns x ZC (z) voxels per CTA, one column of ZC
// voxels per consumer thread (sums in registers across all views, as in the
// global variant). A square tile's footprint on the detector is at most its
// diagonal wide whatever the view angle (a 32 x 8 tile's reaches its long
// side's length), so the box is a third narrower: a third less shared memory
// and TMA traffic per view (1440 views of 2048^2 into 1024^3: FP32 storage
// 11 % faster, FP16 1 %). For every view, a producer warp projects the 4 (x, y) corners of the tile
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

#include <algorithm>
#include <atomic>
#include <cstring>
#include <mutex>
#include <vector>

#include "../ctb_internal.h"
#include "geom.cuh"

namespace ctb {

__device__ unsigned int g_wait_timeouts = 0;

namespace {

// diagnostic: every k-th view reads through global memory (0 = off)
std::atomic<int> g_ovf_every{0};

constexpr int kTX = 16, kTY = 16;
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

// The fast column loop on pairs of voxels (j, j + 1) with the FP32x2
// instructions of sm_100 (one issue slot for two lanes' worth of FFMA/FADD).
// Same operations and roundings as the scalar loop, so the sums are
// bit-identical: the row floor is taken by adding 1.5 * 2^23 rounded toward
// zero (exact for 0 <= vi < 2^22; the caller guarantees vi >= 0.5), whose low
// bits are the row index and whose difference from the magic is float(v0);
// subtractions are FMAs with a -1 factor (one rounding, as a subtraction).
// Rows of the box relative to its origin row, for the bounds-checked build.
struct BoxRows {
    int oy, BV;
};

// float(b) - a for a stored texel b and an FP32 a. For the 16-bit types one
// mixed-precision instruction of sm_100 (sub.rn.f32.f16 / .bf16) converts b
// and subtracts: the same value as the conversion followed by the subtraction
// (the conversion is exact, one rounding), one instruction instead of a
// conversion and half an FP32x2 subtraction per texel (1440 views of 2048^2
// into 1024^3: FP16 storage 5 % faster, BF16 4 %; bit-identical sums).
template <typename T> __device__ __forceinline__ float sub_from(T b, float a);
template <> __device__ __forceinline__ float sub_from<float>(float b, float a) { return __fsub_rn(b, a); }
template <> __device__ __forceinline__ float sub_from<__half>(__half b, float a) {
    float d;
    asm("sub.rn.f32.f16 %0, %1, %2;" : "=f"(d) : "h"(__half_as_ushort(b)), "f"(a));
    return d;
}
template <> __device__ __forceinline__ float sub_from<__nv_bfloat16>(__nv_bfloat16 b, float a) {
    float d;
    asm("sub.rn.f32.bf16 %0, %1, %2;" : "=f"(d) : "h"(__bfloat16_as_ushort(b)), "f"(a));
    return d;
}

// KBU > 0: the box row stride as a compile-time constant (the loads of row
// v0 + 1 then take it as an immediate offset instead of an added register:
// 2-3 % faster for FP16, 4 % for FP32 on 1440 views of 2048^2 into 1024^3,
// bit-identical).
// The tile's first slice sits OFF slices into its block of 32 (geom.cuh), whose
// row origin is c0b: slice j's row is fma(OFF + j, mdv, c0b). IMM: OFF + j is
// an immediate operand and no register holds the slices' offsets (the freed
// registers let the compiler overlap voxel pairs: 4-6 % faster); otherwise
// the offsets zo[j] = OFF + j come from registers (the persistent batch
// kernel, whose extra state would otherwise spill), with the same values.
template <typename T, int ZC, int KBU, int OFF, bool IMM>
__device__ __forceinline__ void column_pairs(const T* col, const int BU_run, const float* zo, float c0b, float mdv,
                                             float fu, float w, float* acc, BoxRows br) {
    static_assert(OFF % ZC == 0 && OFF + ZC <= 32, "a tile lies inside one block of 32 slices");
    const int BU = KBU > 0 ? KBU : BU_run;
    constexpr float kMagic = 12582912.0f;   // 1.5 * 2^23
    const float2 fu2 = make_float2(fu, fu), w2 = make_float2(w, w);
    const float2 m1 = make_float2(-1.0f, -1.0f), mg = make_float2(kMagic, kMagic);
    const float2 mdv2 = make_float2(mdv, mdv), c0b2 = make_float2(c0b, c0b);
#pragma unroll
    for (int j = 0; j < ZC; j += 2) {
        float2 vi;
        if constexpr (IMM)
            vi = make_float2(fmaf(float(OFF + j), mdv, c0b), fmaf(float(OFF + j + 1), mdv, c0b));
        else
            vi = __ffma2_rn(make_float2(zo[j], zo[j + 1]), mdv2, c0b2);
        const float2 sm = __fadd2_rz(vi, mg);
        const float2 nfl = __ffma2_rn(sm, m1, mg);   // -float(floor(vi))
        const float2 fv = __fadd2_rn(vi, nfl);
        int rowa = __float_as_int(sm.x) - 0x4B400000, rowb = __float_as_int(sm.y) - 0x4B400000;
#ifdef CTB_BOUNDS_CHECK
        if (!CTB_FETCH_OK(rowa - br.oy, br.BV - 1, 1)) rowa = br.oy;
        if (!CTB_FETCH_OK(rowb - br.oy, br.BV - 1, 1)) rowb = br.oy;
#endif
        const T* ra = col + rowa * BU;
        const T* rb = col + rowb * BU;
        const float2 p00 = make_float2(sval(ra[0]), sval(rb[0]));
        const float2 p10 = make_float2(sval(ra[BU]), sval(rb[BU]));
        float2 d0, d1;   // p01 - p00, p11 - p10
        if constexpr (sizeof(T) == 4) {
            d0 = __ffma2_rn(p00, m1, make_float2(sval(ra[1]), sval(rb[1])));
            d1 = __ffma2_rn(p10, m1, make_float2(sval(ra[BU + 1]), sval(rb[BU + 1])));
        } else {
            d0 = make_float2(sub_from(ra[1], p00.x), sub_from(rb[1], p00.y));
            d1 = make_float2(sub_from(ra[BU + 1], p10.x), sub_from(rb[BU + 1], p10.y));
        }
        const float2 a = __ffma2_rn(fu2, d0, p00);
        const float2 c = __ffma2_rn(fu2, d1, p10);
        const float2 r = __ffma2_rn(fv, __ffma2_rn(a, m1, c), a);
        const float2 s = __ffma2_rn(w2, r, make_float2(acc[j], acc[j + 1]));
        acc[j] = s.x;
        acc[j + 1] = s.y;
    }
}

// column_pairs with the two most common row strides compiled in (box_dims
// gives 128 bytes times k plus 32: 80 or 144 texels of 16 bits, 72 or 40 of
// 32 bits for voxels of one to two detector pixels), any other at run time.
// An if-chain: a switch over more strides (a jump table) was 1 % slower.
template <typename T, int ZC, int OFF, bool IMM>
__device__ __forceinline__ void column_pairs_bu(const T* col, const int BU, const float* zo, float c0b, float mdv,
                                                float fu, float w, float* acc, BoxRows br) {
    constexpr int kA = sizeof(T) == 4 ? 72 : 80, kB = sizeof(T) == 4 ? 40 : 144;
    if (BU == kA) {
        column_pairs<T, ZC, kA, OFF, IMM>(col, BU, zo, c0b, mdv, fu, w, acc, br);
        return;
    }
    if (BU == kB) {
        column_pairs<T, ZC, kB, OFF, IMM>(col, BU, zo, c0b, mdv, fu, w, acc, br);
        return;
    }
    column_pairs<T, ZC, 0, OFF, IMM>(col, BU, zo, c0b, mdv, fu, w, acc, br);
}

// the pair loop for a tile at offset off (a multiple of ZC below 32) in its block
template <typename T, int ZC, bool IMM>
__device__ __forceinline__ void column_pairs_any(const T* col, const int BU, int off, const float* zo, float c0b,
                                                 float mdv, float fu, float w, float* acc, BoxRows br) {
    if constexpr (ZC >= 32 || !IMM) {
        column_pairs_bu<T, ZC, 0, IMM>(col, BU, zo, c0b, mdv, fu, w, acc, br);
    } else if constexpr (ZC == 16) {
        if (off == 0) column_pairs_bu<T, ZC, 0, IMM>(col, BU, zo, c0b, mdv, fu, w, acc, br);
        else column_pairs_bu<T, ZC, 16, IMM>(col, BU, zo, c0b, mdv, fu, w, acc, br);
    } else {
        if (off == 0) column_pairs_bu<T, ZC, 0, IMM>(col, BU, zo, c0b, mdv, fu, w, acc, br);
        else if (off == 8) column_pairs_bu<T, ZC, 8, IMM>(col, BU, zo, c0b, mdv, fu, w, acc, br);
        else if (off == 16) column_pairs_bu<T, ZC, 16, IMM>(col, BU, zo, c0b, mdv, fu, w, acc, br);
        else column_pairs_bu<T, ZC, 24, IMM>(col, BU, zo, c0b, mdv, fu, w, acc, br);
    }
}

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
    int ovf_every;       // diagnostic: views whose index is a multiple of this
                         // take the global-memory path as if they overflowed (0 = off)
};

// 8 consumer warps own the tile's columns; warp 8 is the producer that waits
// for a free buffer, projects the tile corners and issues the box load, so
// box loads run ahead of the compute independently of any consumer warp.
constexpr int kConsumerWarps = kTX * kTY / 32;
constexpr int kThreads = (kConsumerWarps + 1) * 32;

// Pipeline state in shared memory. Barrier phases are tracked through a
// running box sequence number, so one CTA can run many tiles (persistent
// kernel) through the same barriers.
template <int NBUF>
struct Pipe {
    uint64_t full[NBUF];    // box landed (TMA complete_tx)
    uint64_t empty[NBUF];   // every consumer warp finished reading the box
    int2 org[NBUF];         // box origin (column, row)
    float4 qv[NBUF];        // {sin, cos, h} of the view in each buffer
    int vv[NBUF];           // index of the view in each buffer
    int ovf[NBUF];          // footprint larger than the box: read global memory
    int abort_flag;         // a bounded wait gave up
    long long item;         // persistent kernel: current work item
};

template <int NBUF>
__device__ __forceinline__ void pipe_init(Pipe<NBUF>& p) {
    for (int i = 0; i < NBUF; ++i) {
        mbar_init(&p.full[i], 1);
        mbar_init(&p.empty[i], kConsumerWarps);
    }
    p.abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ bool aborted(const volatile int* f) { return *f != 0; }

// One tile (16 x 16 columns x ZC voxels of one slab) over every view.
// seq: box sequence number of this CTA (identical in all threads), advanced by
// n_views when the tile loads boxes. Returns false if a bounded wait gave up.
// rot: the tile visits the views in the order rot, rot + 1, ... (mod n_views);
// tiles that start later start further on, so the CTAs resident at one time
// read the same few views and share them in L2 (2.3x less DRAM traffic on a
// 1024^3 slab of 1440 views of 2048^2).
template <typename T, int ZC, int NBUF, bool IMM>
__device__ __forceinline__ void tile_pass(const CUtensorMap* map, const T* __restrict__ proj,
                                          const float4* __restrict__ views, int n_views, const ProjGeom& g,
                                          const Box& bx, int buf_stride, float* __restrict__ vol, int accumulate,
                                          int tile_x, int tile_y, int tile_z, Pipe<NBUF>& p, T* buf,
                                          unsigned& seq, int rot, int zshift) {
    volatile int* abort_flag = &p.abort_flag;
    // Consumer warp w covers an 8 (x) x 4 (y) patch of columns: its lanes then
    // sample a compact patch of the box (a few rows x ~12 words), which keeps
    // the shared-memory loads nearly free of bank conflicts even for voxels
    // larger than a detector pixel; stores remain full 32-byte sectors.
    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const bool producer = warp == kConsumerWarps;
    // z tiles start on multiples of ZC box slices (so each lies inside one block of
    // 32 slices, geom.cuh): zshift = z_begin mod ZC, and the first tile of a slab
    // that starts off such a multiple begins before the slab, its slices there
    // computed but not stored (the batch kernel's slabs start at 0: zshift 0)
    const int x0 = tile_x * kTX, y0 = tile_y * kTY, z0 = tile_z * ZC - zshift;
    constexpr int kWX = kTX / 8;   // warps along x
    const int x = x0 + (warp % kWX) * 8 + (lane & 7), y = y0 + (warp / kWX) * 4 + (lane >> 3);
    const int x1 = min(x0 + kTX, g.X) - 1, y1 = min(y0 + kTY, g.Y) - 1;
    const int zf = zshift > 0 ? max(0, -z0) : 0, zl = min(ZC, g.Zs - z0);  // voxels zf .. zl-1 are in the slab
    const long long plane = (long long)g.X * g.Y;

    // A tile whose closest column lies outside the reconstruction cylinder has
    // no voxel to update: write its zeros (unless accumulating) and leave.
    {
        const float ax = world_coord(x0, g.xPre, g.vs), bxw = world_coord(x1, g.xPre, g.vs);
        const float ay = world_coord(y0, g.yPre, g.vs), byw = world_coord(y1, g.yPre, g.vs);
        const float dx = fmaxf(0.0f, fmaxf(ax, -bxw)), dy = fmaxf(0.0f, fmaxf(ay, -byw));
        if (dx * dx + dy * dy > g.r2 * 1.0001f + 1.0f) {
            if (!producer && !accumulate && x < g.X && y < g.Y) {
                float* out = vol + (long long)y * g.X + x;
                for (int j = zf; j < zl; ++j) out[(long long)(z0 + j) * plane] = 0.0f;
            }
            return;
        }
    }
    const float xw = world_coord(x, g.xPre, g.vs);
    const float yw = world_coord(y, g.yPre, g.vs);
    const bool live = !producer && x < g.X && y < g.Y && in_cylinder(xw, yw, g.r2);

    // the tile's first box slice and its offset in its block of 32 slices
    // (a multiple of ZC: the tile lies inside the block)
    const int zt = g.z_begin + z0, zoff = zt & 31;
    const float fzoff = float(zoff);
    float zo[ZC];   // slice offsets in the block for the register form of the pair loop
#pragma unroll
    for (int j = 0; j < ZC; ++j) zo[j] = fzoff + float(j);

    if (producer) {
        // ------------------------------------------------------------ producer
        int iv = 0;
        for (; iv < n_views; ++iv) {
            const unsigned sq = seq + iv;
            const int b = sq % NBUF;
            // the buffer's previous box (sq - NBUF) must have been read by every consumer warp
            if (sq >= NBUF) {
                unsigned tries = 0;
                while (!mbar_try_wait(&p.empty[b], ((sq / NBUF) + 1) & 1)) {
                    if (++tries > kWaitLimit) {
                        *abort_flag = 1;
                        break;
                    }
                }
            }
            if (aborted(abort_flag)) break;
            // footprint of the whole ZC tile (voxels past the slab end are evaluated
            // too and dropped at the store): project the 4 (x, y) corners at both z ends
            float umin = 3.0e38f, umax = -3.0e38f, vmin = 3.0e38f, vmax = -3.0e38f;
            const int vv = rot ? (iv + rot) % n_views : iv;
            const float4 q = __ldg(&views[vv]);
            if (lane < 4) {
                const int cx = (lane & 1) ? x1 : x0;
                const int cy = (lane >> 1) ? y1 : y0;
                float U, u;
                column_geom(world_coord(cx, g.xPre, g.vs), world_coord(cy, g.yPre, g.vs), q.x, q.y, g.D, g.uOff,
                            &U, &u);
                const RowLine rl = row_line(U, q.z, g.zpv, g.vs, g.vPre);
                const float va = row_at(rl, zt), vb = row_at(rl, zt + ZC - 1);
                umin = umax = __fadd_rn(u, g.uPre);
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
                p.org[b] = make_int2(uo, vo);
                p.qv[b] = q;
                p.vv[b] = vv;
                p.ovf[b] = (int(floorf(umax)) + 3 - uo > bx.BU) || (int(floorf(vmax)) + 3 - vo > bx.BV) ||
                           (bx.ovf_every > 0 && vv % bx.ovf_every == 0);
                mbar_expect_tx(&p.full[b], uint32_t(bx.BU) * bx.BV * sizeof(T));
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                tma_load_3d(buf + size_t(b) * buf_stride, map, uo, vo, vv, &p.full[b]);
            }
            __syncwarp();
        }
        seq += iv;  // boxes issued (all of them unless a wait gave up)
        return;
    }

    // -------------------------------------------------------------- consumers
    float acc[ZC];
#pragma unroll
    for (int j = 0; j < ZC; ++j) acc[j] = 0.0f;
    for (int iv = 0; iv < n_views; ++iv) {
        const unsigned sq = seq + iv;
        const int b = sq % NBUF;
        // bounded wait for the box of view iv
        unsigned tries = 0;
        while (!mbar_try_wait(&p.full[b], (sq / NBUF) & 1)) {
            if (++tries > kWaitLimit) {
                *abort_flag = 1;
                break;
            }
        }
        if (aborted(abort_flag)) break;
        if (live) {
            const float4 q = p.qv[b];
            float U, u;
            column_geom(xw, yw, q.x, q.y, g.D, g.uOff, &U, &u);
            if (u >= g.lbU && u <= g.ubU) {
                const float w = __fmul_rn(__fmul_rn(U, U), g.load_scale);
                const float ui = __fadd_rn(u, g.uPre);
                const int u0 = int(ui);
                const float fu = __fsub_rn(ui, float(u0));
                const RowLine rl = row_line(U, q.z, g.zpv, g.vs, g.vPre);
                const float c0b = row_block(rl, zt - zoff);
                // row_at(rl, zt + j): slice j sits zoff + j < 32 slices into the block
                auto row_j = [&](int j) { return fmaf(fzoff + float(j), rl.mdv, c0b); };
                const float vf = row_j(0), vl = row_j(ZC - 1);
                if (!p.ovf[b]) {
                    const int2 o = p.org[b];
                    int cu = u0 - o.x;   // column of u0 in the box
#ifdef CTB_BOUNDS_CHECK
                    if (!CTB_FETCH_OK(cu, bx.BU - 1, 2)) cu = 0;
#endif
                    const T* col = buf + size_t(b) * buf_stride + cu - o.y * bx.BU;
                    const int BU = bx.BU;
                    // strictly inside the row bounds (half-pixel margin): every voxel of the column passes
                    // the per-voxel membership test, so this loop and the checked one take the same
                    // decisions
                    if (fminf(vf, vl) >= 0.5f && fmaxf(vf, vl) <= g.vi_hi - 0.5f) {
                        column_pairs_any<T, ZC, IMM>(col, BU, zoff, zo, c0b, rl.mdv, fu, w, acc,
                                                     BoxRows{o.y, bx.BV});
                    } else {
                        int ja, jb;
                        v_inside_run(z0, ZC, g.zPre, g.vs, q.z, U, g.lbV, g.ubV, &ja, &jb);
#pragma unroll
                        for (int j = 0; j < ZC; ++j) {
                            const float vi = row_j(j);
                            if (j >= ja && j <= jb) {
                                int v0 = int(vi);
                                const float fv = __fsub_rn(vi, float(v0));
#ifdef CTB_BOUNDS_CHECK
                                if (!CTB_FETCH_OK(v0 - o.y, bx.BV - 1, 1)) v0 = o.y;
#endif
                                const T* r0 = col + v0 * BU;
                                const float p00 = sval(r0[0]), p10 = sval(r0[BU]);
                                const float a = fmaf(fu, sub_from(r0[1], p00), p00);
                                const float c = fmaf(fu, sub_from(r0[BU + 1], p10), p10);
                                acc[j] = fmaf(w, fmaf(fv, c - a, a), acc[j]);
                            }
                        }
                    }
                } else {
                    // the view staged in this buffer (the tile's view order is rotated)
                    int gv = p.vv[b], gu = u0;
#ifdef CTB_BOUNDS_CHECK
                    if (!CTB_FETCH_OK(gv, n_views, 5)) gv = 0;
                    if (!CTB_FETCH_OK(gu, g.W - 1, 3)) gu = 0;
#endif
                    const T* col = proj + (long long)gv * g.view_stride + gu;
                    int ja, jb;
                    v_inside_run(z0, ZC, g.zPre, g.vs, q.z, U, g.lbV, g.ubV, &ja, &jb);
#pragma unroll
                    for (int j = 0; j < ZC; ++j) {
                        const float vi = row_j(j);
                        if (j >= ja && j <= jb) {
                            int v0 = int(vi);
                            const float fv = __fsub_rn(vi, float(v0));
#ifdef CTB_BOUNDS_CHECK
                            if (!CTB_FETCH_OK(v0, g.H - 1, 4)) v0 = 0;
#endif
                            const T* r0 = col + (long long)v0 * g.pitch;
                            const float a = fmaf(fu, gval(r0 + 1) - gval(r0), gval(r0));
                            const float c = fmaf(fu, gval(r0 + g.pitch + 1) - gval(r0 + g.pitch), gval(r0 + g.pitch));
                            acc[j] = fmaf(w, fmaf(fv, c - a, a), acc[j]);
                        }
                    }
                }
            }
        }
        // this warp is done with the box of view iv
        __syncwarp();
        if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&p.empty[b])) : "memory");
    }
    seq += n_views;
    if (aborted(abort_flag) || x >= g.X || y >= g.Y) return;
    // (slice z0 + j of column (x, y); z0 < 0 only for slices j < zf, which are not stored)
    float* out = vol + (long long)z0 * plane + (long long)y * g.X + x;
#pragma unroll
    for (int j = 0; j < ZC; ++j) {
        if (j >= zf && j < zl) {
            float* o = out + j * plane;
            *o = accumulate ? (*o + acc[j]) : acc[j];
        }
    }
}

// After an abort: bounded drain of the last NBUF issued boxes (those may still
// be in flight) before the CTA's shared memory goes away; count the failure.
template <int NBUF>
__device__ void pipe_abort_drain(Pipe<NBUF>& p, unsigned seq) {
    atomicAdd(&g_wait_timeouts, 1u);
    for (unsigned i = seq > NBUF ? seq - NBUF : 0; i < seq; ++i) {
        unsigned tries = 0;
        while (!mbar_try_wait(&p.full[i % NBUF], (i / NBUF) & 1) && ++tries < kWaitLimit) {
        }
    }
}

template <typename T, int ZC, int NBUF>
__global__ void __launch_bounds__(kThreads, ZC > 16 ? 3 : 4) bp_tma_kernel(const __grid_constant__ CUtensorMap map,
                                                          const T* __restrict__ proj,
                                                          const float4* __restrict__ views, int n_views,
                                                          ProjGeom g, Box bx, float* __restrict__ vol,
                                                          int accumulate, int resident) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ __align__(16) Pipe<NBUF> p;
    if (threadIdx.x == 0) pipe_init(p);
    __syncthreads();
    unsigned seq = 0;
    // CTAs start in launch order as earlier ones finish: the k-th starts about
    // k / resident of a tile's time after the first, so it starts that far on
    const long long k = blockIdx.x + (long long)gridDim.x * (blockIdx.y + (long long)gridDim.y * blockIdx.z);
    const int rot = int((k % resident) * n_views / resident);
    tile_pass<T, ZC, NBUF, true>(&map, proj, views, n_views, g, bx, bx.buf_elems, vol, accumulate, blockIdx.x,
                           blockIdx.y, blockIdx.z, p, reinterpret_cast<T*>(smem_raw), seq, rot, g.z_begin % ZC);
    __syncthreads();
    if (threadIdx.x == kConsumerWarps * 32 && p.abort_flag) pipe_abort_drain(p, seq);
}

// ----------------------------------------------------------------------------
// Persistent multi-scan kernel: every CTA takes (scan, tile) work items from
// an atomic counter until the batch is done. Scans may differ in detector
// size, view count, volume and voxel pitch; each has its own tensor map.
struct __align__(128) ScanDesc {
    CUtensorMap map;
    ProjGeom g;
    Box bx;
    const void* proj;
    const float4* views;
    float* vol;
    int n_views;
    int tiles_x, tiles_y, tiles_z;
    int accumulate;
};

template <typename T, int ZC, int NBUF>
__global__ void __launch_bounds__(kThreads, ZC > 16 ? 3 : 4) bp_batch_kernel(const ScanDesc* __restrict__ scans, int n_scans,
                                                            const long long* __restrict__ tile_start,
                                                            unsigned long long* queue, int buf_stride) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ __align__(16) Pipe<NBUF> p;
    // the current item's geometry lives in shared memory (read as needed)
    // rather than in every thread's registers
    __shared__ ProjGeom sg;
    __shared__ Box sbx;
    __shared__ int s_scan, s_tile[3];
    if (threadIdx.x == 0) pipe_init(p);
    __syncthreads();
    const long long total = tile_start[n_scans];
    unsigned seq = 0;
    while (true) {
        if (threadIdx.x == 0) {
            const long long item = (long long)atomicAdd(queue, 1ull);
            p.item = item;
            if (item < total) {
                int lo = 0, hi = n_scans - 1;  // scan of this item: last s with tile_start[s] <= item
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (tile_start[mid] <= item) lo = mid;
                    else hi = mid - 1;
                }
                const ScanDesc& d = scans[lo];
                const long long local = item - tile_start[lo];
                s_scan = lo;
                s_tile[0] = int(local % d.tiles_x);
                s_tile[1] = int((local / d.tiles_x) % d.tiles_y);
                s_tile[2] = int(local / ((long long)d.tiles_x * d.tiles_y));
                sg = d.g;
                sbx = d.bx;
            }
        }
        __syncthreads();
        if (p.item >= total || p.abort_flag) break;
        const ScanDesc& d = scans[s_scan];
        const int rot = int((p.item % gridDim.x) * d.n_views / gridDim.x);
        tile_pass<T, ZC, NBUF, false>(&d.map, static_cast<const T*>(d.proj), d.views, d.n_views, sg, sbx, buf_stride,
                               d.vol, d.accumulate, s_tile[0], s_tile[1], s_tile[2], p,
                               reinterpret_cast<T*>(smem_raw), seq, rot, 0);
        __syncthreads();
    }
    if (threadIdx.x == kConsumerWarps * 32 && p.abort_flag) pipe_abort_drain(p, seq);
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
    // only tiles that reach into the cylinder load boxes: their corners lie
    // within the cylinder radius plus one tile diagonal of the axis
    const double T0 = std::sqrt(std::pow((kTX - 1) * vs, 2) + std::pow((kTY - 1) * vs, 2));
    const double R = std::min(std::sqrt(xa * xa + ya * ya), double(std::sqrt(g.r2)) + T0);
    if (R >= 0.9 * D) return false;
    const double Umax = D / (D - R), dU = Umax * Umax / D;
    const double T = std::sqrt(std::pow((kTX - 1) * vs, 2) + std::pow((kTY - 1) * vs, 2));
    // Width: with a tile centre at (s, t) in a view's frame (t including the
    // detector offset), u = D t / (D - s) has gradient U (1, t U / D), U =
    // D / (D - s), so the tile's corners (diagonal T) span at most
    // T U sqrt(1 + (t U / D)^2) to first order; the second-order terms
    // (|u_ss| = 2 |t| U^3 / D^2, |u_st| = U^2 / D) add at most
    // (T/2)^2 (|u_ss| + 2 |u_st|) / 2. For each s the largest |t| within R
    // of the axis is the worst; s is scanned finely (the extent changes by
    // far less than 0.05 pixel between samples). Views whose footprint still
    // does not fit are read through global memory by the kernel.
    double uext = 0.0;
    for (int i = 0; i <= 4096; ++i) {
        const double s = R * (2.0 * i / 4096 - 1.0);
        const double t = std::sqrt(std::max(0.0, R * R - s * s)) + std::fabs(g.uOff);
        const double U = D / (D - s);
        const double first = T * U * std::sqrt(1.0 + (t * U / D) * (t * U / D));
        const double second = 0.125 * T * T * (2.0 * t * U * U * U / (D * D) + 2.0 * U * U / D);
        uext = std::max(uext, first + second);
    }
    uext += 0.05;
    const double zabs =
        std::max(std::fabs((-(ZC - 1) - g.zPre) * vs), std::fabs((g.Zs + ZC - 1 - g.zPre) * vs)) + hmax;
    const double vext = (ZC - 1) * vs * Umax + zabs * dU * T;
    // Row stride: 32 bytes more than a multiple of 128, so adjacent box rows
    // sit 8 banks apart and only rows four apart in one column share a bank;
    // the lanes of a warp (an 8 x 4 patch of columns) sample a few rows within
    // a few words of each other, so they rarely do. 1440 views of 2048^2 into
    // 1024^3 (boxes 80 texels wide, 72 for FP32): 2 % faster than 64 bytes past a multiple
    // of 128 for 16-bit texels, 1 % for FP32, 5-8 % faster than an odd number
    // of 16-byte chunks. Strides past 256 texels fall back to the odd-chunk
    // rule (consecutive rows start in different banks) to keep the box small.
    const int chunk = 16 / esize, per128 = 128 / esize, off = 32 / esize;
    int BU = int(std::ceil(uext)) + 12;
    const int bu32 = (BU - off + per128 - 1) / per128 * per128 + off;
    if (bu32 <= 256) {
        BU = bu32;
    } else {
        BU = (BU + chunk - 1) / chunk * chunk;
        if ((BU / chunk) % 2 == 0) BU += chunk;
    }
    const int BV = int(std::ceil(vext)) + 6;
    if (BU > 256 || BV > 256) return false;
    b->BU = BU;
    b->BV = BV;
    b->buf_elems = (BU * BV + per128 - 1) / per128 * per128;
    b->vi_hi = float(double(g.H) - 1 - 0.1);
    b->ovf_every = g_ovf_every.load();
    return true;
}

template <typename T> struct TmaType;
template <> struct TmaType<float> { static constexpr CUtensorMapDataType v = CU_TENSOR_MAP_DATA_TYPE_FLOAT32; };
template <> struct TmaType<__half> { static constexpr CUtensorMapDataType v = CU_TENSOR_MAP_DATA_TYPE_FLOAT16; };
template <> struct TmaType<__nv_bfloat16> {
    static constexpr CUtensorMapDataType v = CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
};

// Tensor map over [n_views][H][W] projections with row pitch g.pitch; columns
// W..pitch-1 and everything outside the detector read as zero.
template <typename T>
bool make_map(const T* proj, int n_views, const ProjGeom& g, const Box& bx, CUtensorMap* map) {
    if ((size_t(g.pitch) * sizeof(T)) % 16 != 0 || (reinterpret_cast<uintptr_t>(proj) & 15) != 0) return false;
    auto enc = encode_fn();
    if (!enc) return false;
    const cuuint64_t dims[3] = {cuuint64_t(g.W), cuuint64_t(g.H), cuuint64_t(n_views)};
    const cuuint64_t strides[2] = {cuuint64_t(g.pitch) * sizeof(T), cuuint64_t(g.view_stride) * sizeof(T)};
    const cuuint32_t box[3] = {cuuint32_t(bx.BU), cuuint32_t(bx.BV), 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    return enc(map, TmaType<T>::v, 3, const_cast<T*>(proj), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
               CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// three box buffers when three CTAs still fit an SM's shared memory, else two
int choose_nbuf(size_t per_buf) { return (3 * (3 * per_buf + 1024) <= 227 * 1024) ? 3 : 2; }

template <typename T, int ZC>
int launch_t(const T* proj, const float4* views, int n_views, const ProjGeom& g, double hmax, float* vol,
             int accumulate, cudaStream_t s, int nbuf_req) {
    Box bx;
    if (!box_dims(g, ZC, hmax, sizeof(T), &bx)) return CTB_ERR_UNSUPPORTED;
    CUtensorMap map;
    if (!make_map(proj, n_views, g, bx, &map)) return CTB_ERR_UNSUPPORTED;
    const size_t per_buf = size_t(bx.buf_elems) * sizeof(T);
    const int nbuf = (nbuf_req >= 2 && nbuf_req <= 4) ? nbuf_req : choose_nbuf(per_buf);
    const size_t smem = size_t(nbuf) * per_buf;
    if (smem > 200 * 1024) return CTB_ERR_UNSUPPORTED;
    auto kern = nbuf == 4 ? bp_tma_kernel<T, ZC, 4> : nbuf == 3 ? bp_tma_kernel<T, ZC, 3> : bp_tma_kernel<T, ZC, 2>;
    if (const int st = ensure_dynamic_smem(reinterpret_cast<const void*>(kern), smem)) return st;
    dim3 grid((g.X + kTX - 1) / kTX, (g.Y + kTY - 1) / kTY, (g.Zs + g.z_begin % ZC + ZC - 1) / ZC);
    if (grid.y > 65535 || grid.z > 65535) return CTB_ERR_UNSUPPORTED;
    int per_sm = 0, dev = 0, sms = 0;
    CTB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, smem));
    CTB_CUDA_TRY(cudaGetDevice(&dev));
    CTB_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    kern<<<grid, kThreads, smem, s>>>(map, proj, views, n_views, g, bx, vol, accumulate, std::max(1, per_sm * sms));
    return cuda_status(cudaGetLastError(), "bp_tma_kernel launch");
}

template <typename T>
int launch_zc(const void* proj, const float4* views, int n_views, const ProjGeom& g, double hmax, float* vol,
              int accumulate, int zc, cudaStream_t s, int nbuf) {
    if (zc == 8) return launch_t<T, 8>((const T*)proj, views, n_views, g, hmax, vol, accumulate, s, nbuf);
    if (zc == 32) return launch_t<T, 32>((const T*)proj, views, n_views, g, hmax, vol, accumulate, s, nbuf);
    return launch_t<T, 16>((const T*)proj, views, n_views, g, hmax, vol, accumulate, s, nbuf);
}

// ---------------------------------------------------------------- batch
template <typename T, int ZC>
int batch_plan_t(const BpBatchScan* scans, int n, BpBatchPlan* plan, int nbuf_req) {
    plan->desc.clear();
    plan->tile_start.assign(1, 0);
    plan->included.clear();
    plan->excluded.clear();
    int max_elems = 0;
    // longest items (most views) first, so the last items to finish are short
    std::vector<int> order(n);
    for (int i = 0; i < n; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return scans[a].n_views > scans[b].n_views; });
    for (int i : order) {
        const BpBatchScan& sc = scans[i];
        ScanDesc d;
        std::memset(&d, 0, sizeof d);
        // The persistent kernel sizes its buffers for the largest box of the batch;
        // a scan whose box would push it below its CTAs per SM (four, or three at
        // 32 z voxels per thread; three buffers each) runs through its own launch.
        constexpr size_t kBoxBudget = (227 * 1024 / (ZC > 16 ? 3 : 4) - 2048) / 3;
        // (its tiles start at slice 0 of the slab: a slab off a multiple of 32 runs on its own too)
        if (sc.g.z_begin % 32 != 0 || !box_dims(sc.g, ZC, sc.hmax, sizeof(T), &d.bx) ||
            size_t(d.bx.buf_elems) * sizeof(T) > kBoxBudget ||
            !make_map((const T*)sc.proj, sc.n_views, sc.g, d.bx, &d.map)) {
            plan->excluded.push_back(i);
            continue;
        }
        d.g = sc.g;
        d.proj = sc.proj;
        d.views = sc.views;
        d.vol = sc.vol;
        d.n_views = sc.n_views;
        d.tiles_x = (sc.g.X + kTX - 1) / kTX;
        d.tiles_y = (sc.g.Y + kTY - 1) / kTY;
        d.tiles_z = (sc.g.Zs + ZC - 1) / ZC;
        d.accumulate = sc.accumulate;
        max_elems = std::max(max_elems, d.bx.buf_elems);
        const size_t at = plan->desc.size();
        plan->desc.resize(at + sizeof(ScanDesc));
        std::memcpy(plan->desc.data() + at, &d, sizeof d);
        plan->tile_start.push_back(plan->tile_start.back() + (long long)d.tiles_x * d.tiles_y * d.tiles_z);
        plan->included.push_back(i);
    }
    plan->desc_size = sizeof(ScanDesc);
    plan->total_tiles = plan->tile_start.back();
    if (plan->included.empty()) return CTB_OK;
    plan->buf_stride = max_elems;
    const size_t per_buf = size_t(max_elems) * sizeof(T);
    plan->nbuf = (nbuf_req >= 2 && nbuf_req <= 4) ? nbuf_req : choose_nbuf(per_buf);
    plan->smem = size_t(plan->nbuf) * per_buf;
    if (plan->smem > 200 * 1024) return CTB_ERR_UNSUPPORTED;
    auto kern = plan->nbuf == 4 ? bp_batch_kernel<T, ZC, 4>
              : plan->nbuf == 3 ? bp_batch_kernel<T, ZC, 3> : bp_batch_kernel<T, ZC, 2>;
    if (const int st = ensure_dynamic_smem(reinterpret_cast<const void*>(kern), plan->smem)) return st;
    int per_sm = 0, dev = 0, sms = 0;
    CTB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, plan->smem));
    CTB_CUDA_TRY(cudaGetDevice(&dev));
    CTB_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    plan->grid = std::max(1, per_sm) * sms;
    return CTB_OK;
}

template <typename T>
int batch_plan_zc(const BpBatchScan* scans, int n, int zc, BpBatchPlan* plan, int nbuf) {
    if (zc == 8) return batch_plan_t<T, 8>(scans, n, plan, nbuf);
    if (zc == 32) return batch_plan_t<T, 32>(scans, n, plan, nbuf);
    return batch_plan_t<T, 16>(scans, n, plan, nbuf);
}

template <typename T, int ZC>
void batch_launch_t(const BpBatchPlan& plan, const void* desc, const long long* tile_start, int n,
                    unsigned long long* queue, cudaStream_t s) {
    auto kern = plan.nbuf == 4 ? bp_batch_kernel<T, ZC, 4>
              : plan.nbuf == 3 ? bp_batch_kernel<T, ZC, 3> : bp_batch_kernel<T, ZC, 2>;
    kern<<<plan.grid, kThreads, plan.smem, s>>>(static_cast<const ScanDesc*>(desc), n, tile_start, queue,
                                                plan.buf_stride);
}

template <typename T>
void batch_launch_zc(const BpBatchPlan& plan, const void* desc, const long long* tile_start, int n,
                     unsigned long long* queue, cudaStream_t s) {
    if (plan.zc == 8) batch_launch_t<T, 8>(plan, desc, tile_start, n, queue, s);
    else if (plan.zc == 32) batch_launch_t<T, 32>(plan, desc, tile_start, n, queue, s);
    else batch_launch_t<T, 16>(plan, desc, tile_start, n, queue, s);
}

}  // namespace

int backproject_tma_launch(const void* proj, int store_type, const float4* views, int n_views, const ProjGeom& g,
                           double hmax, float* vol, int accumulate, cudaStream_t s, int zc, int nbuf) {
    if (n_views <= 0) return CTB_ERR_UNSUPPORTED;
    switch (store_type) {
        case CTB_FP32: return launch_zc<float>(proj, views, n_views, g, hmax, vol, accumulate, zc, s, nbuf);
        case CTB_FP16: return launch_zc<__half>(proj, views, n_views, g, hmax, vol, accumulate, zc, s, nbuf);
        case CTB_BF16:
            return launch_zc<__nv_bfloat16>(proj, views, n_views, g, hmax, vol, accumulate, zc, s, nbuf);
    }
    return CTB_ERR_UNSUPPORTED;
}

int bp_batch_plan(int store_type, int zc, const BpBatchScan* scans, int n, BpBatchPlan* plan, int nbuf) {
    if (n <= 0) return CTB_ERR_ARG;
    plan->store_type = store_type;
    plan->zc = (zc == 8 || zc == 32) ? zc : 16;
    switch (store_type) {
        case CTB_FP32: return batch_plan_zc<float>(scans, n, plan->zc, plan, nbuf);
        case CTB_FP16: return batch_plan_zc<__half>(scans, n, plan->zc, plan, nbuf);
        case CTB_BF16: return batch_plan_zc<__nv_bfloat16>(scans, n, plan->zc, plan, nbuf);
    }
    return CTB_ERR_ARG;
}

int bp_batch_launch(const BpBatchPlan& plan, const void* desc, const long long* tile_start, int n,
                    unsigned long long* queue, cudaStream_t s) {
    if (n <= 0) return CTB_OK;
    switch (plan.store_type) {
        case CTB_FP32: batch_launch_zc<float>(plan, desc, tile_start, n, queue, s); break;
        case CTB_FP16: batch_launch_zc<__half>(plan, desc, tile_start, n, queue, s); break;
        case CTB_BF16: batch_launch_zc<__nv_bfloat16>(plan, desc, tile_start, n, queue, s); break;
        default: return CTB_ERR_ARG;
    }
    return cuda_status(cudaGetLastError(), "bp_batch_kernel launch");
}

namespace {
// Diagnostic: a barrier initialised for two arrivals that only ever gets one,
// waited on by a warp with the backprojector's bounded loop and the given
// limit. The wait must give up; it records that as the backprojector does.
__global__ void bounded_wait_probe(unsigned limit, int* gave_up) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 2);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&bar)) : "memory");
    unsigned tries = 0;
    bool done = false;
    while (!(done = mbar_try_wait(&bar, 0)) && ++tries <= limit) {
    }
    if (!done && threadIdx.x == 0) {
        atomicAdd(&g_wait_timeouts, 1u);
        *gave_up = 1;
    }
}
}  // namespace

int bounded_wait_probe_run(unsigned limit, cudaStream_t s) {
    int* d = nullptr;
    CTB_CUDA_TRY(cudaMallocAsync((void**)&d, sizeof(int), s));
    int st = cuda_status(cudaMemsetAsync(d, 0, sizeof(int), s), "probe flag");
    if (st == CTB_OK) {
        bounded_wait_probe<<<1, 32, 0, s>>>(limit, d);
        st = cuda_status(cudaGetLastError(), "bounded_wait_probe launch");
    }
    int h = 0;
    if (st == CTB_OK) st = cuda_status(cudaMemcpyAsync(&h, d, sizeof(int), cudaMemcpyDeviceToHost, s), "probe read");
    if (st == CTB_OK) st = cuda_status(cudaStreamSynchronize(s), "probe");
    cudaFreeAsync(d, s);
    if (st != CTB_OK) return st;
    if (h) {
        set_global_error("a bounded device wait gave up after " + std::to_string(limit) + " tries");
        return CTB_ERR_TIMEOUT;
    }
    return CTB_OK;
}

void bp_force_overflow(int every) { g_ovf_every.store(every > 0 ? every : 0); }

int bounds_status_tma(unsigned* count, unsigned long long* first, int reset) {
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

int device_wait_timeouts(unsigned* count, int reset) {
    CTB_CUDA_TRY(cudaMemcpyFromSymbol(count, g_wait_timeouts, sizeof(unsigned)));
    if (reset && *count) {
        const unsigned zero = 0;
        CTB_CUDA_TRY(cudaMemcpyToSymbol(g_wait_timeouts, &zero, sizeof(unsigned)));
    }
    return CTB_OK;
}

}  // namespace ctb
