// Synthetic data: analytic line integrals of a sum of ellipsoids through the
// reference's cone-beam model, in FP64, one thread per detector pixel.
//
// Model (consistent with the backprojection of Ct/CtVolume.cpp:989-1008): a
// point (x, y, z) maps to u = (t + uOffset) D/(D - s), v = (z + h) D/(D - s),
// with s = x cos + y sin, t = -x sin + y cos. Hence the ray through detector
// pixel (r, c), u = c - W/2, v = H/2 - r (matToImageU/V, :1459-1466), runs from
// the source S = D e_s - uOffset e_t - h e_z to Q = (u - uOffset) e_t + (v - h) e_z.
// Everything here is in millimetres; the result is the density line integral.

#include "../ctb_internal.h"

namespace ctb {

namespace {

__global__ void phantom_kernel(const double* __restrict__ ell, int ne, const double* __restrict__ ang,
                               const double* __restrict__ hmm, int nv, int W, int H, double pix, double D,
                               double uoff, double* __restrict__ out) {
    const long long n = (long long)nv * W * H;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const int c = int(i % W);
        const int r = int((i / W) % H);
        const int v = int(i / ((long long)W * H));
        double sn, cs;
        sincospi(ang[v] / 180.0, &sn, &cs);
        const double h = hmm[v];
        const double u = (double(c) - W / 2.0) * pix, vv = (H / 2.0 - double(r)) * pix;
        // e_s = (cs, sn, 0), e_t = (-sn, cs, 0)
        const double Sx = D * cs + uoff * sn, Sy = D * sn - uoff * cs, Sz = -h;
        const double tq = u - uoff;
        const double Qx = -tq * sn, Qy = tq * cs, Qz = vv - h;
        double dx = Qx - Sx, dy = Qy - Sy, dz = Qz - Sz;
        const double L = sqrt(dx * dx + dy * dy + dz * dz);
        dx /= L; dy /= L; dz /= L;
        double sum = 0.0;
        for (int e = 0; e < ne; ++e) {
            const double* E = ell + 16 * e;
            const double px = Sx - E[0], py = Sy - E[1], pz = Sz - E[2];
            // body coordinates: R^T p, scaled by the semi-axes
            const double pbx = (E[6] * px + E[9] * py + E[12] * pz) / E[3];
            const double pby = (E[7] * px + E[10] * py + E[13] * pz) / E[4];
            const double pbz = (E[8] * px + E[11] * py + E[14] * pz) / E[5];
            const double dbx = (E[6] * dx + E[9] * dy + E[12] * dz) / E[3];
            const double dby = (E[7] * dx + E[10] * dy + E[13] * dz) / E[4];
            const double dbz = (E[8] * dx + E[11] * dy + E[14] * dz) / E[5];
            const double a = dbx * dbx + dby * dby + dbz * dbz;
            const double b = pbx * dbx + pby * dby + pbz * dbz;
            const double g = pbx * pbx + pby * pby + pbz * pbz - 1.0;
            const double disc = b * b - a * g;
            if (disc > 0.0) sum += E[15] * 2.0 * sqrt(disc) / a;
        }
        out[i] = sum;
    }
}

}  // namespace

int phantom_launch(const double* ell, int n_ell, const double* angles_deg_dev, const double* heights_mm_dev,
                   int n_views, int W, int H, double pix, double D, double uoff, double* out, cudaStream_t s) {
    if (n_views <= 0 || W <= 0 || H <= 0) return CTB_OK;
    phantom_kernel<<<148 * 16, 256, 0, s>>>(ell, n_ell, angles_deg_dev, heights_mm_dev, n_views, W, H, pix, D,
                                             uoff, out);
    return cuda_status(cudaGetLastError(), "phantom_kernel launch");
}

}  // namespace ctb
