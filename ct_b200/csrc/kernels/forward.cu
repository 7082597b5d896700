// Matched forward projector: the exact transpose of the voxel-driven
// backprojector in backproject.cu (no counterpart in the reference, which has
// no forward model). The shared-memory backprojector takes the same decisions
// but for rows whose coordinate lies within one unit in the last place of an
// integer (geom.cuh), so against it the transpose holds to that rounding.
//
// The backprojector adds, for every voxel and view,
//     w * [(1-fv)((1-fu) p[v0][u0] + fu p[v0][u0+1]) + fv((1-fu) p[v0+1][u0] + fu p[v0+1][u0+1])]
// with w = U^2 * load_scale, under the cylinder, u-bounds and v-bounds masks.
// Its transpose therefore gives detector pixel (r, c) of a view the sum over
// voxels with u0 in {c-1, c} and v0 in {r-1, r} of
//     w * (u0 == c ? 1-fu : fu) * (v0 == r ? 1-fv : fv) * vol.
//
// Ray-driven gather (deterministic, no atomics). A warp owns a strip of kK = 8
// adjacent detector columns c0 .. c0+7 and 256 rows (eight per lane) of one
// view; everything that depends only on (view, strip) -- which voxel columns
// can reach it -- is shared by the warp instead of being recomputed per lane:
//  1. the warp walks the in-plane axis that is most perpendicular to the ray,
//     32 positions at a time, one position per lane; each lane solves
//     u(x, y) = c0-1-W/2 and c0+8-W/2 for the other axis (u is a ratio of
//     linear functions) and gets a short range of candidate columns;
//  2. step by step through those ranges, each lane evaluates one candidate
//     column with the very same FP32 expressions as the backprojector (so the
//     discrete decisions u0, v0 and the masks agree bit for bit with the
//     gather kernel's), and for a
//     column that reaches the strip (u0 in c0-1 .. c0+7) its run of slices
//     inside the detector rows (the reference's v test, once per column);
//  3. the columns that reach the strip are broadcast one at a time (ballot +
//     shuffles); the lanes then walk that column's slices whose rows reach the
//     warp's 256 rows, one slice each, and add each slice's shares to rows v0,
//     v0+1 of detector columns u0, u0+1 (those inside the strip) in the warp's
//     accumulators in shared memory. Lanes that write in the same instruction
//     hold slices far enough apart that their rows differ, and the order of
//     the additions is fixed, so the result is deterministic.
// A voxel column is evaluated by one warp, or by two when u0 is the last
// column of a strip (the share of u0+1 belongs to the next strip): 1.125
// walks per voxel and view instead of the two of a warp per detector column.
// The volume is read in a z-fastest copy so that a warp's lanes (consecutive
// rows -> consecutive z) read contiguous memory.

#include <algorithm>
#include <type_traits>

#include "../ctb_internal.h"
#include "geom.cuh"

namespace ctb {

namespace {

// a CTA: kFC warps, each kK detector columns x kFR * kRPL rows (kRPL per lane)
constexpr int kFR = 32, kFC = 4, kK = 8, kRPL = 8;
constexpr int kRows = kFR * kRPL, kStride = kRows + 1;
constexpr unsigned kAll = 0xffffffffu;

__global__ void __launch_bounds__(kFR * kFC) fp_kernel(const float* __restrict__ volz,
                                                       const float4* __restrict__ views, ProjGeom g,
                                                       float* __restrict__ proj, int accumulate) {
    // per warp: columns c0 .. c0+7 of rows R .. R + 255, a column's rows
    // contiguous, columns kStride = 257 floats apart (the eight columns of a
    // row in eight banks for the write-out)
    __shared__ float s_rows[kFC][kK][kStride];
    const int lane = threadIdx.x;
    const int R = blockIdx.x * kRows;  // first row of the warp
    const int cs0 = (blockIdx.y * kFC + threadIdx.y) * kK;  // first column of the strip
    float(*sacc)[kStride] = s_rows[threadIdx.y];
    const int iv = blockIdx.z;
    if (cs0 >= g.W) return;  // whole warps leave together
    const float4 q = __ldg(&views[iv]);
    const float sn = q.x, cs = q.y, h = q.z;
    const float D = g.D;
    const double Tlo = double(cs0 - 1) - double(g.uPre), Thi = double(cs0 + kK) - double(g.uPre);
    const bool x_major = fabsf(cs) >= fabsf(sn);
    const int np = x_major ? g.X : g.Y;
    const int ns = x_major ? g.Y : g.X;
    const float ppre = x_major ? g.xPre : g.yPre;
    const float spre = x_major ? g.yPre : g.xPre;
#pragma unroll
    for (int k = 0; k < kK; ++k)
#pragma unroll
        for (int r = 0; r < kStride; r += kFR)
            if (r + lane < kStride) sacc[k][r + lane] = 0.0f;
    __syncwarp();
    for (int ip0 = 0; ip0 < np; ip0 += 32) {
        // (1) candidate range of this lane's position
        const int ip = ip0 + lane;
        int i0 = 0, cnt = 0;
        if (ip < np) {
            const float pw = (float(ip) - ppre) * g.vs;
            double s_a, s_b;
            if (x_major) {  // y = [T (D - x cs) + D (x sn - uOff)] / (D cs + T sn)
                s_a = (Tlo * (D - pw * cs) + D * (pw * sn - g.uOff)) / (D * cs + Tlo * sn);
                s_b = (Thi * (D - pw * cs) + D * (pw * sn - g.uOff)) / (D * cs + Thi * sn);
            } else {        // x = [T (D - y sn) - D (y cs + uOff)] / (T cs - D sn)
                s_a = (Tlo * (D - pw * sn) - D * (pw * cs + g.uOff)) / (Tlo * cs - D * sn);
                s_b = (Thi * (D - pw * sn) - D * (pw * cs + g.uOff)) / (Thi * cs - D * sn);
            }
            const double lo = fmin(s_a, s_b) / g.vs + spre, hi = fmax(s_a, s_b) / g.vs + spre;
            // (clamped to [-2, ns + 2] first: the int conversions stay in range
            // for rays nearly parallel to the secondary axis, NaN gives the full range)
            const double big = double(ns) + 2.0;
            i0 = int(fmax(0.0, floor(fmin(fmax(lo, -2.0), big)) - 1.0));
            const int i1 = int(fmin(double(ns - 1), ceil(fmax(fmin(hi, big), -2.0)) + 1.0));
            cnt = max(0, i1 - i0 + 1);
        }
        const int steps = __reduce_max_sync(kAll, cnt);
        for (int st = 0; st < steps; ++st) {
            // (2) this lane's candidate column for this step
            bool hit = false;
            float wa = 0.0f, wb = 0.0f, mdv = 0.0f, c0 = 0.0f, inv = 0.0f;
            int colidx = 0, ku = 0, ja = 0, jb = -1;
            if (st < cnt) {
                const int is = i0 + st;
                const int x = x_major ? ip : is, y = x_major ? is : ip;
                const float xw = world_coord(x, g.xPre, g.vs);
                const float yw = world_coord(y, g.yPre, g.vs);
                if (in_cylinder(xw, yw, g.r2)) {
                    float U, u;
                    column_geom(xw, yw, sn, cs, D, g.uOff, &U, &u);
                    if (u >= g.lbU && u <= g.ubU) {
                        const float ui = __fadd_rn(u, g.uPre);
                        const int u0 = int(ui);
                        const float fu = __fsub_rn(ui, float(u0));
                        if (u0 >= cs0 - 1 && u0 <= cs0 + kK - 1) {
                            v_inside_run(0, g.Zs, g.zPre, g.vs, h, U, g.lbV, g.ubV, &ja, &jb);
                            hit = ja <= jb;
                            const float w = __fmul_rn(__fmul_rn(U, U), g.load_scale);
                            wa = w * (1.0f - fu);  // to column u0
                            wb = w * fu;           // to column u0 + 1
                            const RowLine rl = row_line(U, h, g.zpv, g.vs, g.vPre);
                            mdv = rl.mdv;
                            c0 = rl.c0;
                            inv = 1.0f / -rl.mdv;
                            colidx = x * g.Y + y;
                            ku = u0 - cs0;
                        }
                    }
                }
            }
            // (3) every lane adds the voxels of each hit column that reach its rows
            unsigned mask = __ballot_sync(kAll, hit);
            while (mask) {
                const int j = __ffs(mask) - 1;
                mask &= mask - 1;
                const float jwa = __shfl_sync(kAll, wa, j);
                const float jwb = __shfl_sync(kAll, wb, j);
                const RowLine rl{__shfl_sync(kAll, mdv, j), __shfl_sync(kAll, c0, j)};
                const float jinv = __shfl_sync(kAll, inv, j);
                const int jcol = __shfl_sync(kAll, colidx, j);
                const int jku = __shfl_sync(kAll, ku, j);
                const int jja = __shfl_sync(kAll, ja, j);
                const int jjb = __shfl_sync(kAll, jb, j);
                // slices whose rows can reach R-1 .. R+255: box z in
                // ((c0-R-257)/dv, (c0-R+1)/dv], dv = -mdv > 0, widened by m for the
                // rounding of vi, of the quotients and of 1/dv (together below inv/16
                // for rows under 2^17); the exact row test below decides. Only the
                // slices inside the detector rows (ja .. jb) add.
                const float m = 0.08f * jinv + 0.01f;
                const float zbig = float(g.z_begin + g.Zs) + 2.0f;
                const float zlo = (rl.c0 - float(R + kRows) - 1.0f) * jinv - m;
                const float zhi = (rl.c0 - float(R) + 1.0f) * jinv + m;
                const int z0 = max(jja, int(floorf(fminf(fmaxf(zlo, -2.0f), zbig))) + 1 - g.z_begin);
                const int z1 = min(jjb, int(floorf(fmaxf(fminf(zhi, zbig), -2.0f))) - g.z_begin);
                // lanes st slices apart: their rows differ by st * dv > 1.02, more than
                // the rounding of two row coordinates (2^-6 for rows under 2^17), so
                // the lanes of one instruction never share a row (at st >= Zs only
                // lane 0 has a slice, so the cap keeps that true)
                const int sst = min(int(fminf(jinv, 1.0e7f) * 1.02f) + 1, max(1, g.Zs));
                const float* col = volz + (long long)jcol * g.Zs;
                const bool left = jku >= 0, right = jku + 1 < kK;
                // accumulators of column u0 + 1 (used only when right); column u0's
                // are kStride floats below (used only when left)
                float* const cb = &sacc[0][0] + (jku + 1) * kStride;
                if (z0 > z1) continue;
                const float2 jw2 = make_float2(jwa, jwb);
                constexpr float kMagic = 12582912.0f;  // 1.5 * 2^23: floor of a float in [0, 2^22) by one add
                auto add = [&](int z, float fo, float c0b, float vz) {
                    // computed for every lane; a lane past z1 writes nothing (lr = -2).
                    // The row as geom.cuh forms it: fo = z mod 32 (box slice z), c0b
                    // the row origin of z's block of 32 slices
                    const float vi = fmaf(fo, rl.mdv, c0b);
                    // int(vi) for vi > -1 (the rows of the slices walked here): the
                    // magic-number add floors max(vi, 0)
                    const float sm = __fadd_rz(fmaxf(vi, 0.0f), kMagic);
                    const int v0 = __float_as_int(sm) - __float_as_int(kMagic);
                    const float fv = __fsub_rn(vi, __fsub_rn(sm, kMagic));
                    const float2 vab = __fmul2_rn(jw2, make_float2(vz, vz));
                    const int lr = z <= z1 ? v0 - R : -2;
                    const float f1 = 1.0f - fv;
                    const float2 x0 = __fmul2_rn(make_float2(f1, f1), vab);  // row v0: columns u0, u0 + 1
                    const float2 x1 = __fmul2_rn(make_float2(fv, fv), vab);  // row v0 + 1
                    const bool in0 = unsigned(lr) < unsigned(kRows), in1 = unsigned(lr + 1) < unsigned(kRows);
                    if (left && in0) cb[lr - kStride] += x0.x;
                    if (right && in0) cb[lr] += x0.y;
                    __syncwarp();
                    if (left && in1) cb[lr + 1 - kStride] += x1.x;
                    if (right && in1) cb[lr + 1] += x1.y;
                    __syncwarp();
                };
                // slice of step st: z0 + lane s + (st / s) 32 s + st % s; the walk is
                // compiled for s = 1 and s = 2 (the divisions become shifts and the
                // preloaded steps' offsets constants) and for s at run time
                auto walk = [&](auto s_c) {
                    constexpr int S = decltype(s_c)::value;
                    const int s = S > 0 ? S : sst;
                    const int nsteps = ((z1 - z0) / (kFR * s) + 1) * s;
                    const int zl = z0 + lane * s;
                    auto off = [&](int st) { return (st / s) * kFR * s + st % s; };
                    // row arguments of step st: box slice za + off(st) = za + p + 32 s k
                    // (p = st % s, k = st / s) sits where za + p sits in its block of
                    // 32 slices, and that block starts 32 s k slices later
                    const int za = g.z_begin + zl;
                    const int zo0 = za & 31, zo1 = (za + 1) & 31;
                    const float fo0 = float(zo0), fb0 = float(za - zo0);
                    const float fo1 = float(zo1), fb1 = float(za + 1 - zo1);
                    auto rowarg = [&](int st, float& fo, float& c0b) {
                        if constexpr (S == 1) {
                            fo = fo0;
                            c0b = fmaf(fb0 + float(kFR * st), rl.mdv, rl.c0);
                        } else if constexpr (S == 2) {
                            const bool odd = st & 1;
                            fo = odd ? fo1 : fo0;
                            c0b = fmaf((odd ? fb1 : fb0) + float(2 * kFR * (st >> 1)), rl.mdv, rl.c0);
                        } else {
                            const int zz = za + off(st), zo = zz & 31;
                            fo = float(zo);
                            c0b = row_block(rl, zz - zo);
                        }
                    };
                    // the slice values of the first kPre steps are loaded before any
                    // is used (a 256-row band is about 8 steps at s = 1 and 10 at
                    // s = 2), later ones one step ahead
                    constexpr int kPre = 10;
                    float pre[kPre];
#pragma unroll
                    for (int st = 0; st < kPre; ++st) {
                        const int z = zl + off(st);
                        pre[st] = (st < nsteps && z <= z1) ? __ldg(&col[z]) : 0.0f;
                    }
#pragma unroll
                    for (int st = 0; st < kPre; ++st)
                        if (st < nsteps) {
                            float fo, c0b;
                            rowarg(st, fo, c0b);
                            add(zl + off(st), fo, c0b, pre[st]);
                        }
                    if (nsteps > kPre) {
                        int o = off(kPre);
                        float vz_next = zl + o <= z1 ? __ldg(&col[zl + o]) : 0.0f;
                        for (int st = kPre; st < nsteps; ++st) {
                            const float vz = vz_next;
                            const int on = off(st + 1);
                            if (st + 1 < nsteps) vz_next = zl + on <= z1 ? __ldg(&col[zl + on]) : 0.0f;
                            float fo, c0b;
                            rowarg(st, fo, c0b);
                            add(zl + o, fo, c0b, vz);
                            o = on;
                        }
                    }
                };
                if (sst == 1)
                    walk(std::integral_constant<int, 1>{});
                else if (sst == 2)
                    walk(std::integral_constant<int, 2>{});
                else
                    walk(std::integral_constant<int, 0>{});
            }
        }
    }
    __syncwarp();
    // rows R .. R+255 of columns cs0 .. cs0+7: a lane writes one column of a
    // row, a warp four rows of eight consecutive columns per step
    for (int idx = lane; idx < kK * kRows; idx += kFR) {
        const int k = idx % kK, r = idx / kK;
        const int rk = R + r, ck = cs0 + k;
        if (rk >= g.H || ck >= g.W) continue;
        float* out = proj + (long long)iv * g.view_stride + (long long)rk * g.W + ck;
        const float acc = sacc[k][r];
        *out = accumulate ? (*out + acc) : acc;
    }
}

}  // namespace

int forward_launch(const float* vol, const float4* views, int n_views, const ProjGeom& g, float* proj,
                   int accumulate, cudaStream_t s) {
    if (n_views <= 0) return CTB_OK;
    if (n_views > 65535) {
        set_global_error("forward projector: at most 65535 views per call");
        return CTB_ERR_UNSUPPORTED;
    }
    // z-fastest scratch copy of the slab
    float* volz = nullptr;
    const size_t n = size_t(g.X) * g.Y * g.Zs;
    CTB_CUDA_TRY(cudaMallocAsync((void**)&volz, sizeof(float) * n, s));
    int st = layout_launch(vol, g.X, g.Y, g.Zs, CTB_Z_FASTEST, CTB_LITTLE_ENDIAN, volz, s);
    if (st == CTB_OK) {
        dim3 block(kFR, kFC, 1);
        dim3 grid((g.H + kRows - 1) / kRows, (g.W + kFC * kK - 1) / (kFC * kK), n_views);
        cudaFuncSetAttribute(fp_kernel, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
        fp_kernel<<<grid, block, 0, s>>>(volz, views, g, proj, accumulate);
        st = cuda_status(cudaGetLastError(), "fp_kernel launch");
    }
    cudaFreeAsync(volz, s);
    return st;
}

namespace {
// r = a - b over n values; the sum of r^2 is added to *sumsq (double)
__global__ void residual_kernel(const float* __restrict__ a, const float* __restrict__ b, float* __restrict__ r,
                                long long n, double* __restrict__ sumsq) {
    double acc = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float d = a[i] - b[i];
        r[i] = d;
        acc += double(d) * double(d);
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    __shared__ double part[8];
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < int(blockDim.x >> 5); ++w) t += part[w];
        atomicAdd(sumsq, t);
    }
}
}  // namespace

int residual_launch(const float* a, const float* b, float* r, long long n, double* sumsq, cudaStream_t s) {
    if (n <= 0) return CTB_OK;
    int dev = 0, sms = 0;
    CTB_CUDA_TRY(cudaGetDevice(&dev));
    CTB_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const long long blocks = std::min<long long>((n + 255) / 256, 8LL * sms);
    residual_kernel<<<int(blocks), 256, 0, s>>>(a, b, r, n, sumsq);
    return cuda_status(cudaGetLastError(), "residual_kernel launch");
}

}  // namespace ctb
