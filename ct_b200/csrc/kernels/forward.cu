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
// Ray-driven gather (deterministic, no atomics): one thread per detector pixel,
// lanes of a warp along detector rows of one column so that the column search
// is uniform across the warp. The thread walks the in-plane axis that is most
// perpendicular to the ray; for each position it solves u(x, y) = c-1-W/2 and
// c+1-W/2 for the other axis (u is a ratio of linear functions), visits the
// few candidate columns in between, re-evaluates every quantity with the very
// same FP32 expressions as the backprojector (so the discrete decisions u0, v0
// and the masks agree bit for bit) and adds the voxels whose rows fall on r.
// The volume is read in a z-fastest copy so that a warp's lanes (consecutive
// rows -> consecutive z) read contiguous memory.

#include "../ctb_internal.h"
#include "geom.cuh"

namespace ctb {

namespace {

constexpr int kFR = 32, kFC = 8;

__global__ void __launch_bounds__(kFR * kFC) fp_kernel(const float* __restrict__ volz,
                                                       const float4* __restrict__ views, ProjGeom g,
                                                       float* __restrict__ proj, int accumulate) {
    const int r = blockIdx.x * kFR + threadIdx.x;
    const int c = blockIdx.y * kFC + threadIdx.y;
    const int iv = blockIdx.z;
    if (c >= g.W) return;
    const float4 q = __ldg(&views[iv]);
    const float sn = q.x, cs = q.y, h = q.z;
    const float D = g.D;
    const double Tlo = double(c - 1) - double(g.uPre), Thi = double(c + 1) - double(g.uPre);
    const bool x_major = fabsf(cs) >= fabsf(sn);
    const int np = x_major ? g.X : g.Y;
    const int ns = x_major ? g.Y : g.X;
    const float ppre = x_major ? g.xPre : g.yPre;
    const float spre = x_major ? g.yPre : g.xPre;
    float acc = 0.0f;
    for (int ip = 0; ip < np; ++ip) {
        const float pw = (float(ip) - ppre) * g.vs;
        // secondary world coordinate where u takes the values Tlo / Thi
        double s_a, s_b;
        if (x_major) {  // y = [T (D - x cs) + D (x sn - uOff)] / (D cs + T sn)
            s_a = (Tlo * (D - pw * cs) + D * (pw * sn - g.uOff)) / (D * cs + Tlo * sn);
            s_b = (Thi * (D - pw * cs) + D * (pw * sn - g.uOff)) / (D * cs + Thi * sn);
        } else {        // x = [T (D - y sn) - D (y cs + uOff)] / (T cs - D sn)
            s_a = (Tlo * (D - pw * sn) - D * (pw * cs + g.uOff)) / (Tlo * cs - D * sn);
            s_b = (Thi * (D - pw * sn) - D * (pw * cs + g.uOff)) / (Thi * cs - D * sn);
        }
        const double lo = fmin(s_a, s_b) / g.vs + spre, hi = fmax(s_a, s_b) / g.vs + spre;
        const int i0 = max(0, int(floor(lo)) - 1);
        const int i1 = min(ns - 1, int(ceil(hi)) + 1);
        for (int is = i0; is <= i1; ++is) {
            const int x = x_major ? ip : is, y = x_major ? is : ip;
            const float xw = world_coord(x, g.xPre, g.vs);
            const float yw = world_coord(y, g.yPre, g.vs);
            if (!in_cylinder(xw, yw, g.r2)) continue;
            float U, u;
            column_geom(xw, yw, sn, cs, D, g.uOff, &U, &u);
            if (!(u >= g.lbU && u <= g.ubU)) continue;
            const float ui = __fadd_rn(u, g.uPre);
            const int u0 = int(ui);
            const float fu = __fsub_rn(ui, float(u0));
            float bu;
            if (u0 == c) bu = 1.0f - fu;
            else if (u0 + 1 == c) bu = fu;
            else continue;
            const float w = __fmul_rn(__fmul_rn(U, U), g.load_scale);
            // rows: vi(z) = c0 + z mdv in [r-1, r+1)  ->  z range (mdv < 0)
            const float* col = volz + ((long long)x * g.Y + y) * g.Zs;
            const RowLine rl = row_line(U, h, g.zpv, g.vs, g.vPre);
            const double dv = -double(rl.mdv);
            // (box z index = slab-local z + z_begin)
            const double zlo = (double(rl.c0) - (r + 1)) / dv - g.z_begin;
            const double zhi = (double(rl.c0) - (r - 1)) / dv - g.z_begin;
            const int z0 = max(0, int(floor(zlo)) - 1);
            const int z1 = min(g.Zs - 1, int(ceil(zhi)) + 1);
            for (int z = z0; z <= z1; ++z) {
                const float vi = row_at(rl, float(g.z_begin + z));
                if (!row_ok(vi, g.vi_hi)) continue;
                const int v0 = int(vi);
                const float fv = __fsub_rn(vi, float(v0));
                float bv;
                if (v0 == r) bv = 1.0f - fv;
                else if (v0 + 1 == r) bv = fv;
                else continue;
                acc += w * bu * bv * __ldg(&col[z]);
            }
        }
    }
    if (r >= g.H) return;
    float* out = proj + (long long)iv * g.view_stride + (long long)r * g.W + c;
    *out = accumulate ? (*out + acc) : acc;
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
        dim3 grid((g.H + kFR - 1) / kFR, (g.W + kFC - 1) / kFC, n_views);
        fp_kernel<<<grid, block, 0, s>>>(volz, views, g, proj, accumulate);
        st = cuda_status(cudaGetLastError(), "fp_kernel launch");
    }
    cudaFreeAsync(volz, s);
    return st;
}

}  // namespace ctb
