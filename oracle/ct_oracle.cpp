// ct_oracle.cpp -- TEST INFRASTRUCTURE ONLY.
//
// CPU restatement of the reference (bastian-weber/Ct) FDK reconstruction path,
// used as the parity checker for the CUDA engine and as the timed CPU baseline.
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load
// this library; the product path never calls it.
//
// Three groups of functions:
//   orc_ref_*  : reference-exact FP32 CPU path. Statement by statement the
//                float/double choices of Ct/CtVolume.cpp (convertTo32bit :802,
//                applyLogScaling :860, applyFeldkampWeight :814 + W :828,
//                applyFourierFilter :832, window functions :868-885,
//                reconstructionCore :923-1046, bilinearInterpolation :1048),
//                including the OpenMP x-loop with schedule(dynamic) (:975) and
//                the std::async prefetch of the next projection (:963-965).
//   orc_f64_*  : the same mathematics in double precision (exact-length DFT,
//                optional zero padding, voxel pitch != detector pitch). This is
//                the "FP64 oracle" that mixed-precision runs are scored against.
//   orc_geom_* : the reference's grid rule, cylinder radius and ROI rounding
//                (Ct/CtVolume.cpp:311-316, :370-373, :487-500, :1399-1424).
//
// Third-party arithmetic in the reference path and how it is restated here:
//   * OpenCV cv::dft / cv::idft(DFT_ROWS | DFT_REAL_OUTPUT), float: restated as
//     a double-precision FFT whose result is rounded to float; the inverse is
//     W * irfft(bins 0..W/2) (bins above W/2 are ignored, no 1/W scaling).
//     Pinned against cv2 4.13 fixtures in tests/golden (max rel diff ~2e-7).
//   * OpenCV cv::log (float): restated as logf; cv::log differs from the
//     correctly rounded log by <= 2 ulp (pinned in tests/golden).
//   * OpenCV Mat::convertTo(CV_32F, alpha, beta) for 8U/16U: float working type,
//     dst = float(src) * float(alpha) + float(beta), no fused multiply-add.
// Build with -ffp-contract=off so no FMA is formed where the reference has none.

#include <algorithm>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <future>
#include <memory>
#include <vector>
#include <omp.h>

extern "C" {

// Geometry of one reconstruction, in the reference's units (detector pixels of
// the "virtual" detector at the rotation axis).
typedef struct {
    int W, H;            // detector columns / rows
    float FCD;           // focus-to-centre distance in pixels (CSV FCD / pixelSize)
    float uOffset;       // rotation-axis offset in pixels (CSV uOffset / pixelSize)
    float radius;        // reconstruction cylinder radius in pixels (truncated)
    int xSize, ySize, zSize;                 // full grid
    int xFrom, xTo, yFrom, yTo, zFrom, zTo;  // reconstructed box, [from, to)
    float vs;            // voxel pitch in detector pixels (1 = reference grid)
} orc_geom;

enum { ORC_RAMLAK = 0, ORC_SHEPPLOGAN = 1, ORC_HANN = 2 };

}  // extern "C"

namespace {

// ---------------------------------------------------------------- FFT (double)
// Iterative radix-2 FFT for powers of two, Bluestein chirp-z for other lengths.
using cd = std::complex<double>;

bool is_pow2(size_t n) { return n && !(n & (n - 1)); }

// Radix-2 decimation-in-time plan with a precomputed twiddle table.
struct Pow2Fft {
    size_t n = 0;
    std::vector<cd> tw;        // exp(-2 pi i k / n), k < n/2
    std::vector<uint32_t> rev; // bit reversal permutation
    explicit Pow2Fft(size_t n_ = 0) : n(n_) {
        if (!n) return;
        tw.resize(n / 2);
        for (size_t k = 0; k < n / 2; ++k) {
            const double a = -2.0 * M_PI * double(k) / double(n);
            tw[k] = cd(std::cos(a), std::sin(a));
        }
        rev.resize(n);
        for (size_t i = 1, j = 0; i < n; ++i) {
            size_t bit = n >> 1;
            for (; j & bit; bit >>= 1) j ^= bit;
            j ^= bit;
            rev[i] = uint32_t(j);
        }
    }
    void run(cd* a, bool inverse) const {
        for (size_t i = 1; i < n; ++i)
            if (i < rev[i]) std::swap(a[i], a[rev[i]]);
        for (size_t len = 2; len <= n; len <<= 1) {
            const size_t half = len / 2, stride = n / len;
            for (size_t i = 0; i < n; i += len) {
                for (size_t k = 0; k < half; ++k) {
                    const cd w = inverse ? std::conj(tw[k * stride]) : tw[k * stride];
                    const cd u = a[i + k], v = a[i + k + half] * w;
                    a[i + k] = u + v;
                    a[i + k + half] = u - v;
                }
            }
        }
    }
};

// Unnormalised DFT of arbitrary length: X[k] = sum_n x[n] exp(-+2 pi i n k / N).
struct Dft {
    size_t n = 0, m = 0;
    Pow2Fft p2;
    std::vector<cd> chirp, bfft;  // Bluestein tables
    explicit Dft(size_t n_) : n(n_) {
        if (is_pow2(n)) { p2 = Pow2Fft(n); return; }
        m = 1;
        while (m < 2 * n - 1) m <<= 1;
        p2 = Pow2Fft(m);
        chirp.resize(n);
        for (size_t k = 0; k < n; ++k) {
            // exp(-i pi k^2 / n), k^2 reduced mod 2n for accuracy
            const unsigned long long k2 = (unsigned long long)k * k % (2ull * n);
            const double ang = M_PI * double(k2) / double(n);
            chirp[k] = cd(std::cos(ang), -std::sin(ang));
        }
        bfft.assign(m, cd(0, 0));
        bfft[0] = std::conj(chirp[0]);
        for (size_t k = 1; k < n; ++k) bfft[k] = bfft[m - k] = std::conj(chirp[k]);
        p2.run(bfft.data(), false);
    }
    void run(std::vector<cd>& x, bool inverse) const {
        if (is_pow2(n)) { p2.run(x.data(), inverse); return; }
        if (inverse) for (auto& v : x) v = std::conj(v);
        std::vector<cd> a(m, cd(0, 0));
        for (size_t k = 0; k < n; ++k) a[k] = x[k] * chirp[k];
        p2.run(a.data(), false);
        for (size_t k = 0; k < m; ++k) a[k] *= bfft[k];
        p2.run(a.data(), true);
        for (size_t k = 0; k < n; ++k) x[k] = a[k] * chirp[k] / double(m);
        if (inverse) for (auto& v : x) v = std::conj(v);
    }
};

// ------------------------------------------------------------ window functions
// Ct/CtVolume.cpp:868-885 (float n, float N; double sin/cos of a float product).
float ramLak(float n, float N) { return n / N; }
float sheppLogan(float n, float N) {
    if (n == 0) return 0.0f;
    float rl = ramLak(n, N);
    return float(double(rl) * std::sin(double(rl * 0.5f) * M_PI) / (double(rl * 0.5f) * M_PI));
}
float hann(float n, float N) {
    float rl = ramLak(n, N);
    return float(double(rl * 0.5f) * (1.0 + std::cos(M_PI * double(rl))));
}
float window_ref(int filter, unsigned k, unsigned nyq) {
    switch (filter) {
        case ORC_SHEPPLOGAN: return sheppLogan(float(k), float(nyq));
        case ORC_HANN: return hann(float(k), float(nyq));
        default: return ramLak(float(k), float(nyq));
    }
}
// Same windows in double, sampled at k of a length-N transform (N may be padded).
double window_f64(int filter, size_t k, size_t nyq) {
    const double rl = double(k) / double(nyq);
    switch (filter) {
        case ORC_SHEPPLOGAN: return k == 0 ? 0.0 : rl * std::sin(rl * 0.5 * M_PI) / (rl * 0.5 * M_PI);
        case ORC_HANN: return rl * 0.5 * (1.0 + std::cos(M_PI * rl));
        default: return rl;
    }
}

// ------------------------------------------------------- reference row filter
// applyFourierFilter (Ct/CtVolume.cpp:832-858): forward DFT of each row, bins
// 0..W/2 multiplied by window(k, W/2+1), inverse = W * irfft, no padding.
void filter_rows_ref(float* img, int W, int H, int filter, bool multithreading) {
    const unsigned nyq = unsigned(W) / 2 + 1;
    std::vector<float> win(nyq);
    for (unsigned k = 0; k < nyq; ++k) win[k] = window_ref(filter, k, nyq);
    const Dft dft{size_t(W)};
#pragma omp parallel for if (multithreading)
    for (int r = 0; r < H; ++r) {
        std::vector<cd> x(W);
        float* row = img + size_t(r) * W;
        for (int c = 0; c < W; ++c) x[c] = cd(row[c], 0.0);
        dft.run(x, false);
        // the reference keeps the spectrum in float
        for (int k = 0; k < W; ++k) x[k] = cd(float(x[k].real()), float(x[k].imag()));
        for (unsigned k = 0; k < nyq; ++k)
            x[k] = cd(float(x[k].real()) * win[k], float(x[k].imag()) * win[k]);
        // C2R: Hermitian extension of bins 0..W/2
        x[0] = cd(x[0].real(), 0.0);
        if (W % 2 == 0) x[W / 2] = cd(x[W / 2].real(), 0.0);
        for (int k = 1; k < (W + 1) / 2; ++k) x[W - k] = std::conj(x[k]);
        dft.run(x, true);
        for (int c = 0; c < W; ++c) row[c] = float(x[c].real());
    }
}

// ------------------------------------------------- reference preprocessing
// convertTo32bit (:802-812) + applyLogScaling (:860-866) + applyFeldkampWeight
// (:814-830). depth: 8 (uint8), 16 (uint16) or 32 (float).
void preprocess_ref(const void* img, int depth, int W, int H, float base, float FCD,
                    int filter, float* out, bool multithreading) {
    const size_t n = size_t(W) * H;
    if (depth == 8 || depth == 16) {
        const float alpha = float(depth == 8 ? 1.0 / 255.0 : 1.0 / 65535.0);
        const float beta = float(0.000001 * base);
        for (size_t i = 0; i < n; ++i) {
            const float s = depth == 8 ? float(((const uint8_t*)img)[i]) : float(((const uint16_t*)img)[i]);
            out[i] = s * alpha + beta;
        }
    } else {
        std::memcpy(out, img, n * sizeof(float));
    }
    // image *= 1/(base + 1e-6*base); cv::log; image *= -1
    const float scale = float(1.0 / (double(base) + 0.000001 * double(base)));
    for (size_t i = 0; i < n; ++i) out[i] = -std::log(out[i] * scale);
    // Feldkamp weight, u = c - W/2, v = -r + H/2 (matToImageU/V, :1459-1466)
    const float uPre = float(double(W) / 2.0), vPre = float(double(H) / 2.0);
#pragma omp parallel for if (multithreading)
    for (int r = 0; r < H; ++r) {
        float* row = out + size_t(r) * W;
        for (int c = 0; c < W; ++c) {
            const float u = float(c) - uPre;
            const float v = (-1) * float(r) + vPre;
            const float w = FCD / std::sqrt(FCD * FCD + u * u + v * v);
            row[c] = row[c] * w;
        }
    }
    filter_rows_ref(out, W, H, filter, multithreading);
}

// bilinearInterpolation (:1048-1054): float lerps along u stored as double,
// final lerp along v in double, returned as float.
inline float bilerp_ref(float u, float v, float u0v0, float u1v0, float u0v1, float u1v1) {
    double a = (1.0f - u) * u0v0 + u * u1v0;
    double b = (1.0f - u) * u0v1 + u * u1v1;
    return float((1.0f - v) * a + v * b);
}

struct RefBounds {
    float lbU, ubU, lbV, ubV, uPre, vPre, xPre, yPre, zPre;
    float lbY, ubY, lbZ, ubZ, radiusSquared;
    int xMax, yMax, zMax;
};

RefBounds ref_bounds(const orc_geom& g) {
    RefBounds b;
    b.uPre = float(double(g.W) / 2.0);
    b.vPre = float(double(g.H) / 2.0);
    b.xPre = float(float(g.xSize) / 2.0 - float(g.xFrom));
    b.yPre = float(float(g.ySize) / 2.0 - float(g.yFrom));
    b.zPre = float(float(g.zSize) / 2.0 - float(g.zFrom));
    b.xMax = g.xTo - g.xFrom;
    b.yMax = g.yTo - g.yFrom;
    b.zMax = g.zTo - g.zFrom;
    // reconstructionCore :924-933
    b.lbU = 0.0f - b.uPre;
    b.ubU = float(double(g.W) - 1 - 0.1) - b.uPre;
    b.lbV = (-1) * float(double(g.H) - 1 - 0.1) + b.vPre;
    b.ubV = (-1) * 0.0f + b.vPre;
    b.lbY = 0.0f - b.yPre;
    b.ubY = float(b.yMax) - b.yPre;
    b.lbZ = 0.0f - b.zPre;
    b.ubZ = float(b.zMax) - b.zPre;
    b.radiusSquared = g.radius * g.radius;
    return b;
}

// One view of reconstructionCore (:945-1043) into a Z_FASTEST volume
// (idx = x*yMax*zMax + y*zMax + z, Common/Volume.h:260). With vs != 1 the world
// coordinates are scaled by the voxel pitch (engine extension; vs == 1 is exact).
void backproject_view_ref(const float* image, const orc_geom& g, const RefBounds& b,
                          double angleDeg, double heightOffsetD, float* vol) {
    const float FCD = g.FCD, uOffset = g.uOffset, vs = g.vs;
    const float angle_rad = float((angleDeg / 180.0) * M_PI);
    const float sine = float(std::sin(double(angle_rad)));
    const float cosine = float(std::cos(double(angle_rad)));
    const float heightOffset = float(heightOffsetD);
    const int W = g.W;
    const long yz = long(b.yMax) * b.zMax;
#pragma omp parallel for schedule(dynamic)
    for (long xIndex = 0; xIndex < b.xMax; ++xIndex) {
        const float x = (float(xIndex) - b.xPre) * vs;
        float* volumePtr = vol + xIndex * yz;
        for (float yi = b.lbY; yi < b.ubY; ++yi) {
            const float y = yi * vs;
            if ((x * x + y * y) >= b.radiusSquared) { volumePtr += b.zMax; continue; }
            float U, u;
            {
                float t = (-1) * x * sine + y * cosine;
                t += uOffset;
                float s = x * cosine + y * sine;
                U = FCD / (FCD - s);
                u = t * U;
            }
            if (u < b.lbU || u > b.ubU) { volumePtr += b.zMax; continue; }
            const float w = U * U;
            for (float zi = b.lbZ; zi < b.ubZ; ++zi, ++volumePtr) {
                const float z = zi * vs;
                const float v = (z + heightOffset) * U;
                if (v >= b.lbV && v <= b.ubV) {
                    const float uIndex = u + b.uPre;
                    const float vIndex = (-1) * v + b.vPre;
                    const int u0 = int(uIndex), u1 = u0 + 1;
                    const int v0 = int(vIndex), v1 = v0 + 1;
                    const float* row0 = image + size_t(v0) * W;
                    const float* row1 = image + size_t(v1) * W;
                    const float value = w * bilerp_ref(uIndex - float(u0), vIndex - float(v0),
                                                       row0[u0], row0[u1], row1[u0], row1[u1]);
                    (*volumePtr) += value;
                }
            }
        }
    }
}

// ------------------------------------------------------------- FP64 oracle
// Rows [r0, r0 + nrows) of a projection of height H; img points at row r0.
void preprocess_f64(const void* img, int depth, int W, int H, int r0, int nrows, double base, double FCD,
                    int filter, int pad, double* out) {
    const size_t n = size_t(W) * nrows;
    std::vector<double> p(n);
    for (size_t i = 0; i < n; ++i) {
        double s;
        if (depth == 8) s = ((const uint8_t*)img)[i] / 255.0;
        else if (depth == 16) s = ((const uint16_t*)img)[i] / 65535.0;
        else s = ((const float*)img)[i];
        s += 0.000001 * base;
        p[i] = -std::log(s / (base + 0.000001 * base));
    }
    const double uPre = W / 2.0, vPre = H / 2.0;
    for (int r = 0; r < nrows; ++r)
        for (int c = 0; c < W; ++c) {
            const double u = c - uPre, v = -(r + r0) + vPre;
            p[size_t(r) * W + c] *= FCD / std::sqrt(FCD * FCD + u * u + v * v);
        }
    // pad 1: the reference's length-W circular filter; pad >= 2: zero padding
    // to the next power of two >= 2W with the window sampled on that grid
    size_t N = size_t(W);
    if (pad >= 2) { N = 1; while (N < 2 * size_t(W)) N <<= 1; }
    const size_t nyq = N / 2 + 1;
    const Dft dft(N);
    std::vector<double> win(N);
    for (size_t k = 0; k < N; ++k) win[k] = window_f64(filter, std::min(k, N - k), nyq);
    // output scale follows the reference's x W convention for every padding
    const double scale = double(W) / double(N);
#pragma omp parallel for
    for (int r = 0; r < nrows; ++r) {
        std::vector<cd> x(N, cd(0, 0));
        for (int c = 0; c < W; ++c) x[c] = cd(p[size_t(r) * W + c], 0.0);
        dft.run(x, false);
        for (size_t k = 0; k < N; ++k) x[k] *= win[k];
        dft.run(x, true);
        for (int c = 0; c < W; ++c) out[size_t(r) * W + c] = x[c].real() * scale;
    }
}

}  // namespace

extern "C" {

// Grid rule (Ct/CtVolume.cpp:311-316) and cylinder radius (:370-373).
unsigned orc_ref_cylinder_radius(int W, float FCD) {
    double radius = unsigned(W) / 2;
    return unsigned(std::sqrt((double(FCD) * FCD * radius * radius) / (double(FCD) * FCD + radius * radius)));
}

// setVolumeBounds clamps (:487-500, including the yTo/zTo lower clamp against
// xFrom) followed by updateBoundaries rounding (:1399-1409). Returns 0 when the
// call is ignored because a lower and upper bound are identical.
int orc_ref_clamp_bounds(float xF, float xT, float yF, float yT, float zF, float zT, float* out6) {
    if (xF == xT || yF == yT || zF == zT) return 0;
    const float xf = std::max(0.0f, std::min(1.0f, xF));
    const float xt = std::max(xf, std::min(1.0f, xT));
    const float yf = std::max(0.0f, std::min(1.0f, yF));
    const float yt = std::max(xf, std::min(1.0f, yT));
    const float zf = std::max(0.0f, std::min(1.0f, zF));
    const float zt = std::max(xf, std::min(1.0f, zT));
    out6[0] = xf; out6[1] = xt; out6[2] = yf; out6[3] = yt; out6[4] = zf; out6[5] = zt;
    return 1;
}

void orc_ref_geom(int W, int H, float FCD, float uOffset, const float* rel6, orc_geom* g) {
    g->W = W; g->H = H; g->FCD = FCD; g->uOffset = uOffset;
    const unsigned radius = orc_ref_cylinder_radius(W, FCD);
    g->radius = float(radius);
    g->xSize = int(radius * 2); g->ySize = int(radius * 2); g->zSize = H;
    g->xFrom = unsigned(rel6[0] * g->xSize + 0.5); g->xTo = unsigned(rel6[1] * g->xSize + 0.5);
    g->yFrom = unsigned(rel6[2] * g->ySize + 0.5); g->yTo = unsigned(rel6[3] * g->ySize + 0.5);
    g->zFrom = unsigned(rel6[4] * g->zSize + 0.5); g->zTo = unsigned(rel6[5] * g->zSize + 0.5);
    g->vs = 1.0f;
}

// Angle direction correction (:755-767) and relative height offsets (:742-753).
void orc_ref_fix_sinogram(double* angles, double* heights, int n, int ccw, double pixelSize) {
    if (n > 1) {
        const double diff = angles[1] - angles[0];
        if ((!ccw && diff > 0) || (ccw && diff < 0))
            for (int i = 0; i < n; ++i) angles[i] *= -1;
    }
    double sum = 0;
    for (int i = 0; i < n; ++i) sum += heights[i];
    sum /= double(n);
    // pixelSize is a float member of the reference's CtVolume (Ct/CtVolume.h:224)
    const double pix = double(float(pixelSize));
    for (int i = 0; i < n; ++i) { heights[i] -= sum; heights[i] /= pix; }
}

// The reference's window value for bin k of nyq bins.
float orc_ref_window(int filter, unsigned k, unsigned nyq) { return window_ref(filter, k, nyq); }

// One projection through the reference CPU preprocessing chain.
void orc_ref_preprocess(const void* img, int depth, int W, int H, float base, float FCD,
                        int filter, float* out) {
    preprocess_ref(img, depth, W, H, base, FCD, filter, out, false);
}

// Row filter only (input already log-scaled and weighted).
void orc_ref_filter_rows(float* img, int W, int H, int filter) {
    filter_rows_ref(img, W, H, filter, false);
}

// Backprojection of already filtered projections (nviews x H x W floats) into a
// Z_FASTEST volume that the caller zero-initialises; views stepped by `step`.
void orc_ref_backproject(const float* proj, int nviews, int step, const double* anglesDeg,
                         const double* heightsPx, const orc_geom* g, int nthreads, float* vol) {
    if (nthreads > 0) omp_set_num_threads(nthreads);
    const RefBounds b = ref_bounds(*g);
    for (int p = 0; p < nviews; p += (step < 1 ? 1 : step))
        backproject_view_ref(proj + size_t(p) * g->W * g->H, *g, b, anglesDeg[p], heightsPx[p], vol);
}

// The whole CPU reconstruction (reconstructionCore :923-1046) from raw images
// held in memory: per-view preprocessing runs on a std::async thread one view
// ahead of the OpenMP backprojection, as in the reference. Returns wall seconds
// (steady clock) in *seconds.
int orc_ref_reconstruct(const void* imgs, int depth, int nviews, int step, const double* anglesDeg,
                        const double* heightsPx, float base, int filter, const orc_geom* g,
                        int nthreads, float* vol, double* seconds) {
    if (nthreads > 0) omp_set_num_threads(nthreads);
    const auto t0 = std::chrono::steady_clock::now();
    const size_t pix = size_t(g->W) * g->H;
    const size_t bytes = depth == 8 ? 1 : depth == 16 ? 2 : 4;
    const RefBounds b = ref_bounds(*g);
    auto prepare = [&](int p) {
        std::vector<float> out(pix);
        preprocess_ref((const char*)imgs + size_t(p) * pix * bytes, depth, g->W, g->H, base, g->FCD,
                       filter, out.data(), false);
        return out;
    };
    if (step < 1) step = 1;
    std::future<std::vector<float>> future;
    for (int p = 0; p < nviews; p += step) {
        std::vector<float> image = (p == 0) ? prepare(p) : future.get();
        if (p + step < nviews) future = std::async(std::launch::async, prepare, p + step);
        backproject_view_ref(image.data(), *g, b, anglesDeg[p], heightsPx[p], vol);
    }
    *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return 0;
}

// ------------------------------------------------------------- FP64 oracle
// Preprocess one projection in double: log, Feldkamp weight, ramp filter with
// the transform length N = W (pad 1) or the next power of two >= 2W (pad 2,
// zero padded), window sampled on that grid, output scaled by W/N so every
// padding keeps the reference's x W convention.
void orc_f64_preprocess(const void* img, int depth, int W, int H, double base, double FCD,
                        int filter, int pad, double* out) {
    preprocess_f64(img, depth, W, H, 0, H, base, FCD, filter, pad, out);
}

// The same for the detector rows [r0, r0 + nrows) only; img points at row r0.
void orc_f64_preprocess_rows(const void* img, int depth, int W, int H, int r0, int nrows, double base,
                             double FCD, int filter, int pad, double* out) {
    preprocess_f64(img, depth, W, H, r0, nrows, base, FCD, filter, pad, out);
}

// Double-precision voxel-driven backprojection of filtered projections into a
// Z_FASTEST volume, restricted to z indices [z0, z1) of the box when z1 > z0.
// Projections hold detector rows [row0, row0 + nrows) of every view; samples
// outside that window are counted in *missed (the caller sizes the window).
int orc_f64_backproject_rows(const double* proj, int nviews, const double* anglesDeg,
                             const double* heightsPx, const orc_geom* g, int row0, int nrows, int z0, int z1,
                             double* vol, long long* missed);

void orc_f64_backproject(const double* proj, int nviews, const double* anglesDeg,
                         const double* heightsPx, const orc_geom* g, int z0, int z1, double* vol) {
    long long missed = 0;
    orc_f64_backproject_rows(proj, nviews, anglesDeg, heightsPx, g, 0, g->H, z0, z1, vol, &missed);
}

int orc_f64_backproject_rows(const double* proj, int nviews, const double* anglesDeg,
                             const double* heightsPx, const orc_geom* g, int row0, int nrows, int z0, int z1,
                             double* vol, long long* missed) {
    const int W = g->W, H = g->H;
    const double uPre = W / 2.0, vPre = H / 2.0;
    const double xPre = g->xSize / 2.0 - g->xFrom, yPre = g->ySize / 2.0 - g->yFrom,
                 zPre = g->zSize / 2.0 - g->zFrom;
    const int xMax = g->xTo - g->xFrom, yMax = g->yTo - g->yFrom, zMax = g->zTo - g->zFrom;
    if (z1 <= z0) { z0 = 0; z1 = zMax; }
    const int zn = z1 - z0;
    const double lbU = -uPre, ubU = (W - 1.1) - uPre, lbV = -(H - 1.1) + vPre, ubV = vPre;
    const double D = g->FCD, vs = g->vs, r2 = double(g->radius) * g->radius;
    long long miss = 0;
    for (int p = 0; p < nviews; ++p) {
        const double th = anglesDeg[p] / 180.0 * M_PI, sn = std::sin(th), cs = std::cos(th);
        const double h = heightsPx[p];
        const double* img = proj + size_t(p) * W * nrows;
#pragma omp parallel for schedule(dynamic) reduction(+ : miss)
        for (int xi = 0; xi < xMax; ++xi) {
            const double x = (xi - xPre) * vs;
            for (int yi = 0; yi < yMax; ++yi) {
                const double y = (yi - yPre) * vs;
                if (x * x + y * y >= r2) continue;
                const double t = -x * sn + y * cs + g->uOffset, s = x * cs + y * sn;
                const double U = D / (D - s), u = t * U;
                if (u < lbU || u > ubU) continue;
                const double w = U * U, ui = u + uPre;
                const int u0 = int(ui);
                const double fu = ui - u0;
                double* col = vol + (size_t(xi) * yMax + yi) * zn;
                for (int zi = z0; zi < z1; ++zi) {
                    const double v = ((zi - zPre) * vs + h) * U;
                    if (v < lbV || v > ubV) continue;
                    const double vi = -v + vPre;
                    const int v0 = int(vi);
                    const double fv = vi - v0;
                    if (v0 < row0 || v0 + 1 >= row0 + nrows) { ++miss; continue; }
                    const double* r0 = img + size_t(v0 - row0) * W;
                    const double* r1 = r0 + W;
                    const double a = (1 - fu) * r0[u0] + fu * r0[u0 + 1];
                    const double c = (1 - fu) * r1[u0] + fu * r1[u0 + 1];
                    col[zi - z0] += w * ((1 - fv) * a + fv * c);
                }
            }
        }
    }
    *missed = miss;
    return miss == 0 ? 0 : 1;
}

int orc_num_threads(void) { return omp_get_max_threads(); }

}  // extern "C"
