// Matched forward projector: the exact transpose of the voxel-driven
// backprojector in backproject.cu (no counterpart in the reference, which has
// no forward model).
//
// The backprojector adds, for every voxel and view,
//     w * [(1-fv)((1-fu) p[v0][u0] + fu p[v0][u0+1]) + fv((1-fu) p[v0+1][u0] + fu p[v0+1][u0+1])]
// with w = U^2 * load_scale, under the cylinder, u-bounds and v-bounds masks.
// Its transpose therefore gives detector pixel (r, c) of a view the sum over
// voxels with u0 in {c-1, c} and v0 in {r-1, r} of
//     w * (u0 == c ? 1-fu : fu) * (v0 == r ? 1-fv : fv) * vol.
//
// Ray-driven gather (deterministic, no atomics). A warp owns 256 detector rows
// (eight per lane) of one detector column c of one view; everything that depends
// only on (view, c) -- which voxel columns can reach c -- is shared by the
// warp instead of being recomputed per lane:
//  1. the warp walks the in-plane axis that is most perpendicular to the ray,
//     32 positions at a time, one position per lane; each lane solves
//     u(x, y) = c-1-W/2 and c+1-W/2 for the other axis (u is a ratio of linear
//     functions) and gets a short range of candidate columns;
//  2. step by step through those ranges, each lane evaluates one candidate
//     column with the very same FP32 expressions as the backprojector (so the
//     discrete decisions u0, v0 and the masks agree bit for bit);
//  3. the columns that reach c are broadcast one at a time (ballot + shuffles);
//     the lanes then walk that column's slices whose rows reach the warp's 256
//     rows, one slice each, and add each slice's two row weights into the
//     warp's row accumulators in shared memory. Lanes that write in the same
//     instruction hold slices far enough apart that their rows differ, and the
//     order of the additions is fixed, so the result is deterministic.
// The volume is read in a z-fastest copy so that a warp's lanes (consecutive
// rows -> consecutive z) read contiguous memory.

#include "../ctb_internal.h"
#include "geom.cuh"

namespace ctb {

namespace {

// a CTA: kFC detector columns (one warp each) x kFR * kRPL rows (kRPL per lane)
constexpr int kFR = 32, kFC = 8, kRPL = 8;
constexpr unsigned kAll = 0xffffffffu;

__global__ void __launch_bounds__(kFR * kFC) fp_kernel(const float* __restrict__ volz,
                                                       const float4* __restrict__ views, ProjGeom g,
                                                       float* __restrict__ proj, int accumulate) {
    __shared__ float s_rows[kFC][kFR * kRPL];  // per warp: rows R .. R + 255
    const int lane = threadIdx.x;
    const int R = blockIdx.x * (kFR * kRPL);  // first row of the warp
    const int c = blockIdx.y * kFC + threadIdx.y;
    float* srow = s_rows[threadIdx.y];
    const int iv = blockIdx.z;
    if (c >= g.W) return;  // whole warps leave together
    const float4 q = __ldg(&views[iv]);
    const float sn = q.x, cs = q.y, h = q.z;
    const float D = g.D;
    const double Tlo = double(c - 1) - double(g.uPre), Thi = double(c + 1) - double(g.uPre);
    const bool x_major = fabsf(cs) >= fabsf(sn);
    const int np = x_major ? g.X : g.Y;
    const int ns = x_major ? g.Y : g.X;
    const float ppre = x_major ? g.xPre : g.yPre;
    const float spre = x_major ? g.yPre : g.xPre;
#pragma unroll
    for (int k = 0; k < kRPL; ++k) srow[lane + k * kFR] = 0.0f;
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
            float wb = 0.0f, mdv = 0.0f, c0 = 0.0f, inv = 0.0f, Uc = 0.0f;
            int colidx = 0;
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
                        if (u0 == c || u0 + 1 == c) {
                            hit = true;
                            const float bu = u0 == c ? 1.0f - fu : fu;
                            const float w = __fmul_rn(__fmul_rn(U, U), g.load_scale);
                            wb = w * bu;
                            const RowLine rl = row_line(U, h, g.zpv, g.vs, g.vPre);
                            mdv = rl.mdv;
                            c0 = rl.c0;
                            inv = 1.0f / -rl.mdv;
                            Uc = U;
                            colidx = x * g.Y + y;
                        }
                    }
                }
            }
            // (3) every lane adds the voxels of each hit column that reach its row
            unsigned mask = __ballot_sync(kAll, hit);
            while (mask) {
                const int j = __ffs(mask) - 1;
                mask &= mask - 1;
                const float jwb = __shfl_sync(kAll, wb, j);
                const RowLine rl{__shfl_sync(kAll, mdv, j), __shfl_sync(kAll, c0, j)};
                const float jinv = __shfl_sync(kAll, inv, j);
                const int jcol = __shfl_sync(kAll, colidx, j);
                const float jU = __shfl_sync(kAll, Uc, j);
                // slices whose rows can reach R-1 .. R+255: box z in
                // ((c0-R-257)/dv, (c0-R+1)/dv], dv = -mdv > 0, widened by m for the
                // rounding of vi, of the quotients and of 1/dv (together below inv/16
                // for rows under 2^17); the exact row test below decides
                const float m = 0.08f * jinv + 0.01f;
                const float zbig = float(g.z_begin + g.Zs) + 2.0f;
                const float zlo = (rl.c0 - float(R + kFR * kRPL) - 1.0f) * jinv - m;
                const float zhi = (rl.c0 - float(R) + 1.0f) * jinv + m;
                const int z0 = max(0, int(floorf(fminf(fmaxf(zlo, -2.0f), zbig))) + 1 - g.z_begin);
                const int z1 = min(g.Zs - 1, int(floorf(fmaxf(fminf(zhi, zbig), -2.0f))) - g.z_begin);
                // lanes st slices apart: their rows differ by st * dv > 1.02, more than
                // the rounding of two row coordinates (2^-6 for rows under 2^17), so
                // the lanes of one instruction never share a row (at st >= Zs only
                // lane 0 has a slice, so the cap keeps that true)
                const int st = min(int(fminf(jinv, 1.0e7f) * 1.02f) + 1, max(1, g.Zs));
                const float* col = volz + (long long)jcol * g.Zs;
                for (int zb = z0; zb <= z1; zb += kFR * st) {
                    for (int q = 0; q < st; ++q) {
                        const int z = zb + q + lane * st;
                        int lr = -2;
                        float ca = 0.0f, cb = 0.0f;
                        if (z <= z1) {
                            const float vi = row_at(rl, float(g.z_begin + z));
                            const float zw = __fmul_rn(__fsub_rn(float(z), g.zPre), g.vs);
                            if (v_inside(zw, h, jU, g.lbV, g.ubV)) {
                                const int v0 = int(vi);
                                const float fv = __fsub_rn(vi, float(v0));
                                const float val = jwb * __ldg(&col[z]);
                                lr = v0 - R;
                                ca = (1.0f - fv) * val;  // to row v0
                                cb = fv * val;           // to row v0 + 1
                            }
                        }
                        if (lr >= 0 && lr < kFR * kRPL) srow[lr] += ca;
                        __syncwarp();
                        if (lr + 1 >= 0 && lr + 1 < kFR * kRPL) srow[lr + 1] += cb;
                        __syncwarp();
                    }
                }
            }
        }
    }
    __syncwarp();
#pragma unroll
    for (int k = 0; k < kRPL; ++k) {
        const int rk = R + lane + k * kFR;
        if (rk >= g.H) break;
        float* out = proj + (long long)iv * g.view_stride + (long long)rk * g.W + c;
        const float acc = srow[lane + k * kFR];
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
        dim3 grid((g.H + kFR * kRPL - 1) / (kFR * kRPL), (g.W + kFC - 1) / kFC, n_views);
        fp_kernel<<<grid, block, 0, s>>>(volz, views, g, proj, accumulate);
        st = cuda_status(cudaGetLastError(), "fp_kernel launch");
    }
    cudaFreeAsync(volz, s);
    return st;
}

}  // namespace ctb
