// Kernels (a)+(b): projection preprocessing fused into a shared-memory FFT ramp
// filter, plus the FP64 kernels that build the filter tables.
//
// Reference semantics (bastian-weber/Ct, CPU path, which is the parity target):
//   convertTo32bit      Ct/CtVolume.cpp:802-812  s = float(I)*alpha + beta
//   applyLogScaling     Ct/CtVolume.cpp:860-866  p = -ln(s * 1/(I0 + 1e-6*I0))
//   applyFeldkampWeight Ct/CtVolume.cpp:814-830  p *= D / sqrt(D^2 + u^2 + v^2)
//   applyFourierFilter  Ct/CtVolume.cpp:832-858  row DFT, bins 0..W/2 times
//                        window(k, W/2+1), unnormalised C2R (x W), no padding
//   windows             Ct/CtVolume.cpp:868-885
//
// Design. A row filter is a circular convolution of length W with a real, even
// kernel (the window is real and applied symmetrically by the C2R transform).
// Every case is therefore computed as
//     out = IFFT_M( FFT_M(x zero-padded to M) * K ),   K real,
// with a power-of-two M: M = W when W is a power of two (reference-exact
// circular filter), M = nextpow2(2W-1) with K = FFT of the periodically
// extended kernel otherwise (still exactly the length-W circular filter), and
// M = nextpow2(2W) with the window sampled on the padded grid for pad = 2.
// Because K is real and even, two detector rows are filtered at once as the
// real and imaginary parts of one complex signal.
//
// Each group of M/8 threads owns one row pair in shared memory (M complex
// floats); the FFT is a Stockham radix-4 (+ one radix-2) autosort transform
// with two barriers per stage. Raw pixels are read once, filtered values are
// written once: HBM traffic is the algorithmic minimum.

#include <type_traits>
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "../ctb_internal.h"

namespace ctb {

namespace {

// ------------------------------------------------------------- FP64 tables
__global__ void twiddle_kernel(float2* tw, int M) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= M) return;
    double s, c;
    sincospi(-2.0 * double(k) / double(M), &s, &c);
    tw[k] = make_float2(float(c), float(s));
}

// Reference window, Ct/CtVolume.cpp:868-885: rl = float(n)/float(N) in float,
// sin/cos evaluated in double on a float product, result rounded to float.
__device__ float window_ref(int filter, int k, int nyq) {
    const float rl = float(k) / float(nyq);
    if (filter == CTB_SHEPPLOGAN) {
        if (k == 0) return 0.0f;
        const double a = double(rl * 0.5f) * 3.14159265358979323846;
        return float(double(rl) * sin(a) / a);
    }
    if (filter == CTB_HANN) {
        return float(double(rl * 0.5f) * (1.0 + cos(3.14159265358979323846 * double(rl))));
    }
    return rl;
}

// Window in double on an arbitrary transform grid (padded mode).
__device__ double window_f64(int filter, int k, int nyq) {
    const double rl = double(k) / double(nyq);
    if (filter == CTB_SHEPPLOGAN) {
        if (k == 0) return 0.0;
        const double a = rl * 0.5 * 3.14159265358979323846;
        return rl * sin(a) / a;
    }
    if (filter == CTB_HANN) return rl * 0.5 * (1.0 + cos(3.14159265358979323846 * rl));
    return rl;
}

// K[k] for M == W (power of two, pad 1): the symmetric reference window.
__global__ void kernel_direct(float* K, int M, int filter) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= M) return;
    const int kk = min(k, M - k);
    K[k] = window_ref(filter, kk, M / 2 + 1);
}

// K[k] for pad 2: (W/M) * window on the padded grid.
__global__ void kernel_padded(float* K, int M, int W, int filter) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= M) return;
    const int kk = min(k, M - k);
    K[k] = float(double(W) / double(M) * window_f64(filter, kk, M / 2 + 1));
}

// Spatial kernel of the length-W circular filter:
//   g[j] = sum_k Hsym[k] cos(2 pi j k / W)   (unnormalised, real, even).
__global__ void spatial_kernel(double* g, int W, int filter) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= W) return;
    const int nyq = W / 2 + 1;
    double acc = 0.0;
    for (int k = 0; k < W; ++k) {
        const int kk = min(k, W - k);
        const long long jk = (long long)j * k % W;
        acc += double(window_ref(filter, kk, nyq)) * cospi(2.0 * double(jk) / double(W));
    }
    g[j] = acc;
}

// K[k] = (1/M) sum_j G_M[j] cos(2 pi j k / M) with G_M the periodic extension
// of g placed at indices [0, W) and [M-W+1, M).
__global__ void embedded_kernel(float* K, const double* g, int W, int M) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= M) return;
    double acc = g[0];
    for (int j = 1; j < W; ++j) {
        const long long jk = (long long)j * k % M;
        acc += 2.0 * g[j] * cospi(2.0 * double(jk) / double(M));
    }
    K[k] = float(acc / double(M));
}

// ----------------------------------------------------------- storage types
template <typename T> __device__ __forceinline__ T to_store(float v);
template <> __device__ __forceinline__ float to_store<float>(float v) { return v; }
template <> __device__ __forceinline__ __half to_store<__half>(float v) { return __float2half_rn(v); }
template <> __device__ __forceinline__ __nv_bfloat16 to_store<__nv_bfloat16>(float v) {
    return __float2bfloat16_rn(v);
}

template <typename T> __device__ __forceinline__ float raw_value(const T* p, const FilterArgs& a);
template <> __device__ __forceinline__ float raw_value<uint8_t>(const uint8_t* p, const FilterArgs& a) {
    return __fadd_rn(__fmul_rn(float(*p), a.alpha), a.beta);
}
template <> __device__ __forceinline__ float raw_value<uint16_t>(const uint16_t* p, const FilterArgs& a) {
    return __fadd_rn(__fmul_rn(float(*p), a.alpha), a.beta);
}
template <> __device__ __forceinline__ float raw_value<float>(const float* p, const FilterArgs& a) {
    return *p;
}

// -ln(s * scale) * D / sqrt(D^2 + u^2 + v^2), no contraction (reference order).
__device__ __forceinline__ float log_part(float s, const FilterArgs& a) { return -logf(__fmul_rn(s, a.log_scale)); }
__device__ __forceinline__ float weight_part(int r, int c, const FilterArgs& a) {
    const float u = __fsub_rn(float(c), a.uPre);
    const float v = __fadd_rn(-float(r), a.vPre);
    const float d2 = __fadd_rn(__fadd_rn(__fmul_rn(a.D, a.D), __fmul_rn(u, u)), __fmul_rn(v, v));
    return __fdiv_rn(a.D, __fsqrt_rn(d2));
}
__device__ __forceinline__ float preprocess(float s, int r, int c, const FilterArgs& a) {
    return __fmul_rn(log_part(s, a), weight_part(r, c, a));
}

// TAB: the Feldkamp weight of every pixel comes from a table (exactly
// weight_part's values), loaded together with the raw samples, instead of a
// square root and a divide per pixel.

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// ------------------------------------------------------ shared-memory FFT
// Stockham autosort FFT of length M (power of two) by a group of TG = M/8
// threads: one radix-2 or radix-4 stage (when log2 M is not a multiple of 3)
// followed by radix-8 stages; every thread owns 8 elements per stage. The
// last forward stage multiplies by the kernel spectrum on its way to shared
// memory and the last inverse stage writes the filtered row pair straight to
// global memory, so each transform costs one shared-memory round trip per
// stage and no separate passes.
constexpr float kSqrtHalf = 0.70710678118654752440f;

template <bool INV>
__device__ __forceinline__ void dft2(float2* v) {
    const float2 a = v[0], b = v[1];
    v[0] = make_float2(a.x + b.x, a.y + b.y);
    v[1] = make_float2(a.x - b.x, a.y - b.y);
}

// forward: multiply by -i; inverse: by +i
template <bool INV>
__device__ __forceinline__ float2 rot90(float2 d) {
    return INV ? make_float2(-d.y, d.x) : make_float2(d.y, -d.x);
}

template <bool INV>
__device__ __forceinline__ void dft4(float2& v0, float2& v1, float2& v2, float2& v3) {
    const float2 a0 = make_float2(v0.x + v2.x, v0.y + v2.y);
    const float2 a1 = make_float2(v0.x - v2.x, v0.y - v2.y);
    const float2 a2 = make_float2(v1.x + v3.x, v1.y + v3.y);
    const float2 a3 = rot90<INV>(make_float2(v1.x - v3.x, v1.y - v3.y));
    v0 = make_float2(a0.x + a2.x, a0.y + a2.y);
    v1 = make_float2(a1.x + a3.x, a1.y + a3.y);
    v2 = make_float2(a0.x - a2.x, a0.y - a2.y);
    v3 = make_float2(a1.x - a3.x, a1.y - a3.y);
}

// 8-point DFT in registers: two 4-point DFTs of the even and odd samples joined
// by the eighth roots of unity.
template <bool INV>
__device__ __forceinline__ void dft8(float2* v) {
    float2 e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
    float2 o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
    dft4<INV>(e0, e1, e2, e3);
    dft4<INV>(o0, o1, o2, o3);
    // w^1 = (1 -+ i)/sqrt2, w^2 = -+i, w^3 = (-1 -+ i)/sqrt2 (upper sign: forward)
    const float2 t1 = INV ? make_float2(kSqrtHalf * (o1.x - o1.y), kSqrtHalf * (o1.x + o1.y))
                          : make_float2(kSqrtHalf * (o1.x + o1.y), kSqrtHalf * (o1.y - o1.x));
    const float2 t2 = rot90<INV>(o2);
    const float2 t3 = INV ? make_float2(-kSqrtHalf * (o3.x + o3.y), kSqrtHalf * (o3.x - o3.y))
                          : make_float2(kSqrtHalf * (o3.y - o3.x), -kSqrtHalf * (o3.x + o3.y));
    v[0] = make_float2(e0.x + o0.x, e0.y + o0.y);
    v[4] = make_float2(e0.x - o0.x, e0.y - o0.y);
    v[1] = make_float2(e1.x + t1.x, e1.y + t1.y);
    v[5] = make_float2(e1.x - t1.x, e1.y - t1.y);
    v[2] = make_float2(e2.x + t2.x, e2.y + t2.y);
    v[6] = make_float2(e2.x - t2.x, e2.y - t2.y);
    v[3] = make_float2(e3.x + t3.x, e3.y + t3.y);
    v[7] = make_float2(e3.x - t3.x, e3.y - t3.y);
}

template <int R, bool INV>
__device__ __forceinline__ void butterfly(float2* v) {
    if (R == 2) dft2<INV>(v);
    else if (R == 4) dft4<INV>(v[0], v[1], v[2], v[3]);
    else dft8<INV>(v);
}

enum { kFromSmem = 0, kFromInput = 1 };
enum { kToSmem = 0, kToSmemTimesK = 1, kToOutput = 2 };

// One radix-R stage; each of the TG threads does 8/R butterflies.
template <int R, bool INV, int SRC, int DST, typename In, typename Out>
__device__ __forceinline__ void fft_stage(float2* s, int M, int Ns, const float2* __restrict__ tw,
                                          const float* __restrict__ K, int lt, int TG, const In& in, const Out& out) {
    constexpr int PER = 8 / R;
    const int nb = M / R;
    const int step = M / (Ns * R);
    float2 y[PER][R];
#pragma unroll
    for (int i = 0; i < PER; ++i) {
        const int b = lt + i * TG;
        const int jm = b & (Ns - 1);
#pragma unroll
        for (int r = 0; r < R; ++r) y[i][r] = SRC == kFromInput ? in(b + r * nb) : s[b + r * nb];
        if (Ns > 1) {
#pragma unroll
            for (int r = 1; r < R; ++r) {
                float2 w = __ldg(&tw[(jm * r * step) & (M - 1)]);
                if (INV) w.y = -w.y;
                y[i][r] = cmul(y[i][r], w);
            }
        }
        butterfly<R, INV>(y[i]);
    }
    if (SRC == kFromSmem && DST != kToOutput) __syncthreads();  // in place: all reads before any write
#pragma unroll
    for (int i = 0; i < PER; ++i) {
        const int b = lt + i * TG;
        const int jm = b & (Ns - 1);
        const int d0 = (b - jm) * R + jm;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int idx = d0 + r * Ns;
            if (DST == kToOutput) {
                out(idx, y[i][r]);
            } else if (DST == kToSmemTimesK) {
                const float k = __ldg(&K[idx]);
                s[idx] = make_float2(y[i][r].x * k, y[i][r].y * k);
            } else {
                s[idx] = y[i][r];
            }
        }
    }
    if (DST != kToOutput) __syncthreads();
}

// Whole transform: first stage from SRC0, last stage to DSTL. All threads of
// the CTA must call it (barriers).
template <bool INV, int SRC0, int DSTL, typename In, typename Out>
__device__ void fft_run(float2* s, int M, int logM, const float2* __restrict__ tw, const float* __restrict__ K,
                        int lt, int TG, const In& in, const Out& out) {
    const int rem = logM % 3;
    const int first = rem == 1 ? 2 : rem == 2 ? 4 : 8;
    const int nst = logM / 3 + (rem ? 1 : 0);
    int Ns = 1;
    for (int st = 0; st < nst; ++st) {
        if (st == 0) {
            if (nst == 1) fft_stage<8, INV, SRC0, DSTL>(s, M, Ns, tw, K, lt, TG, in, out);
            else if (first == 2) fft_stage<2, INV, SRC0, kToSmem>(s, M, Ns, tw, K, lt, TG, in, out);
            else if (first == 4) fft_stage<4, INV, SRC0, kToSmem>(s, M, Ns, tw, K, lt, TG, in, out);
            else fft_stage<8, INV, SRC0, kToSmem>(s, M, Ns, tw, K, lt, TG, in, out);
            Ns *= first;
        } else if (st == nst - 1) {
            fft_stage<8, INV, kFromSmem, DSTL>(s, M, Ns, tw, K, lt, TG, in, out);
            Ns *= 8;
        } else {
            fft_stage<8, INV, kFromSmem, kToSmem>(s, M, Ns, tw, K, lt, TG, in, out);
            Ns *= 8;
        }
    }
}

// One group of TG = M/8 threads per detector row pair; groups = blockDim/TG.
template <typename InT, typename OutT, bool TAB>
__global__ void __launch_bounds__(1024) filter_kernel(const InT* __restrict__ raw, OutT* __restrict__ out,
                                                      FilterArgs a, const float2* __restrict__ tw,
                                                      const float* __restrict__ K) {
    extern __shared__ float2 smem[];
    const int M = a.M, TG = M >> 3;
    const int g = threadIdx.x / TG, lt = threadIdx.x - g * TG;
    const int groups = blockDim.x / TG;
    float2* s = smem + (size_t)g * M;

    const int W = a.W, H = a.H;
    const int pairs = (H + 1) >> 1;
    const long long q = (long long)blockIdx.x * groups + g;
    const bool active = q < a.n_views * pairs;
    const long long view = active ? q / pairs : 0;
    const int r0 = active ? int(q - view * pairs) * 2 : 0;
    const bool has1 = r0 + 1 < H;
    const size_t base0 = (size_t)view * H * W + (size_t)r0 * W;              // raw rows (dense)
    const size_t obase = (size_t)view * H * a.out_pitch + (size_t)r0 * a.out_pitch;  // filtered rows

    // rows r0 and r0+1 as the real and imaginary parts, zero beyond W
    auto load = [&](int c) {
        float2 z = make_float2(0.f, 0.f);
        if (active && c < W) {
            z.x = preprocess(raw_value(raw + base0 + c, a), r0, c, a);
            if (has1) z.y = preprocess(raw_value(raw + base0 + W + c, a), r0 + 1, c, a);
        }
        return z;
    };
    auto store = [&](int c, float2 z) {
        if (active && c < W) {
            out[obase + c] = to_store<OutT>(z.x * a.store_scale);
            if (has1) out[obase + a.out_pitch + c] = to_store<OutT>(z.y * a.store_scale);
        }
    };
    // Preprocessing is kept out of the first FFT stage (done there it raises the
    // register footprint: it involves log, sqrt and divide). All 16 raw loads of
    // a thread (8 columns x 2 rows; TG = M/8) are issued before any arithmetic,
    // so their latencies overlap instead of adding up.
    InT v0[8], v1[8];
    float w0[8], w1[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const int c = lt + k * TG;
        const bool in = active && c < W;
        v0[k] = in ? raw[base0 + c] : InT(0);
        v1[k] = in && has1 ? raw[base0 + W + c] : InT(0);
        if constexpr (TAB) {
            w0[k] = in ? __ldg(&a.wt[(size_t)r0 * W + c]) : 0.0f;
            w1[k] = in && has1 ? __ldg(&a.wt[(size_t)(r0 + 1) * W + c]) : 0.0f;
        }
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const int c = lt + k * TG;
        float2 z = make_float2(0.f, 0.f);
        if (active && c < W) {
            const float wa = TAB ? w0[k] : weight_part(r0, c, a);
            z.x = __fmul_rn(log_part(raw_value(&v0[k], a), a), wa);
            if (has1) {
                const float wb = TAB ? w1[k] : weight_part(r0 + 1, c, a);
                z.y = __fmul_rn(log_part(raw_value(&v1[k], a), a), wb);
            }
        }
        s[c] = z;
    }
    __syncthreads();
    fft_run<false, kFromSmem, kToSmemTimesK>(s, M, a.logM, tw, K, lt, TG, load, store);
    fft_run<true, kFromSmem, kToOutput>(s, M, a.logM, tw, K, lt, TG, load, store);
}

// --------------------------------------- register four-step transform
// For M = 16 L with L = 16 L2 (M = 512 ... 4096) a group of L threads owns one
// row pair. Every thread keeps 16 complex values in registers and the
// transform is three register passes joined by two shared-memory transposes:
//   1. thread t:       16-point DFT over r of x[t + L r], times w_M^(t s)
//   2. thread (s, t2): 16-point DFT over r of pass 1's values (t2 + L2 r, s),
//                      times w_L^(t2 s2)
//   3. thread (s, j):  for s2 = j + L2 q (q < 16 / L2) the L2-point DFT over t2,
// which leaves X[s + 16 s2 + 256 k3] in registers (k3 < L2). The kernel
// spectrum multiplies it there; the inverse runs the passes backwards with
// conjugate factors and ends with thread t holding x[t + L r] again, so raw
// rows are read and filtered rows written with the same coalesced pattern.
// The exchange between passes 2 and 3 stays inside a warp. The paddings (L2
// per 16-value row of the first transpose, 1 per s2 row and L2 per s block of
// the second) keep every shared-memory access at two wavefronts per warp (one
// per half-warp, the minimum for 8-byte elements). Three block barriers per
// row pair; four where the second transpose reuses the first one's space so
// that three CTAs fit an SM.
template <int M> struct RF {
    static constexpr int L = M / 16, L2 = L / 16, Q = 16 / L2;
    static constexpr int SA = 16 * (L + L2);       // first transpose, float2 per group
    static constexpr int SB = 16 * (L2 + 1) + L2;  // second transpose, float2 per s block
    static constexpr int G = 256 / L;              // row pairs per CTA of 256 threads
    static constexpr bool ALIAS = 3 * (size_t(G) * (SA + 16 * SB) * 8 + 1024) > 227 * 1024;
    static constexpr int SG = ALIAS ? (SA > 16 * SB ? SA : 16 * SB) : SA + 16 * SB;  // float2 per group
    static_assert(M >= 512 && M <= 4096 && (M & (M - 1)) == 0, "register transform lengths");
};

__device__ __forceinline__ float2 cmul_conj(float2 a, float2 b) {
    return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}

// x times w16^m (forward: exp(-2 pi i m / 16); inverse: the conjugate)
template <bool INV, int m>
__device__ __forceinline__ float2 tw16(float2 x) {
    constexpr float c1 = 0.92387953251128675613f, s1 = 0.38268343236508977173f;
    // cos and sin of 2 pi m / 16 for m = 0 ... 9 (m = n1 k2 <= 9)
    constexpr float cs[10] = {1.0f, c1, kSqrtHalf, s1, 0.0f, -s1, -kSqrtHalf, -c1, -1.0f, -c1};
    constexpr float sn[10] = {0.0f, s1, kSqrtHalf, c1, 1.0f, c1, kSqrtHalf, s1, 0.0f, -s1};
    static_assert(m >= 0 && m <= 9, "twiddle index");
    if constexpr (m == 0) return x;
    else if constexpr (m == 4) return rot90<INV>(x);
    else {
        const float c = cs[m], sv = sn[m];
        return INV ? make_float2(x.x * c - x.y * sv, x.y * c + x.x * sv)
                   : make_float2(x.x * c + x.y * sv, x.y * c - x.x * sv);
    }
}

template <bool INV, int n1>
__device__ __forceinline__ void tw16_row(float2* a) {
    a[1] = tw16<INV, n1 * 1>(a[1]);
    a[2] = tw16<INV, n1 * 2>(a[2]);
    a[3] = tw16<INV, n1 * 3>(a[3]);
}

// 16-point DFT in registers, natural order in and out: n = n1 + 4 n2,
// k = 4 k1 + k2; 4-point DFTs over n2, twiddles w16^(n1 k2), 4-point DFTs over n1.
template <bool INV>
__device__ __forceinline__ void dft16(float2* v) {
    float2 a[4][4];
#pragma unroll
    for (int n1 = 0; n1 < 4; ++n1) {
        a[n1][0] = v[n1]; a[n1][1] = v[n1 + 4]; a[n1][2] = v[n1 + 8]; a[n1][3] = v[n1 + 12];
        dft4<INV>(a[n1][0], a[n1][1], a[n1][2], a[n1][3]);
    }
    tw16_row<INV, 1>(a[1]);
    tw16_row<INV, 2>(a[2]);
    tw16_row<INV, 3>(a[3]);
#pragma unroll
    for (int k2 = 0; k2 < 4; ++k2) {
        dft4<INV>(a[0][k2], a[1][k2], a[2][k2], a[3][k2]);
#pragma unroll
        for (int k1 = 0; k1 < 4; ++k1) v[4 * k1 + k2] = a[k1][k2];
    }
}

template <int N, bool INV>
__device__ __forceinline__ void dft_n(float2* v) {
    if constexpr (N == 2) dft2<INV>(v);
    else if constexpr (N == 4) dft4<INV>(v[0], v[1], v[2], v[3]);
    else if constexpr (N == 8) dft8<INV>(v);
    else dft16<INV>(v);
}

template <int M, typename InT, typename OutT>
__global__ void __launch_bounds__(256, 3) filter_rf_kernel(const InT* __restrict__ raw, OutT* __restrict__ out,
                                                           FilterArgs a, const float2* __restrict__ tw,
                                                           const float* __restrict__ K) {
    using C = RF<M>;
    constexpr int L = C::L, L2 = C::L2, Q = C::Q;
    extern __shared__ float2 smem[];
    const int g = threadIdx.x / L, lt = threadIdx.x % L;
    float2* sa = smem + g * C::SG;
    const int W = a.W, H = a.H;
    const int pairs = (H + 1) >> 1;
    const long long q = (long long)blockIdx.x * C::G + g;
    const bool active = q < a.n_views * pairs;
    const long long view = active ? q / pairs : 0;
    const int r0 = active ? int(q - view * pairs) * 2 : 0;
    const bool has1 = active && r0 + 1 < H;
    const InT* src = raw + (size_t)view * H * W + (size_t)r0 * W;
    const float* wrow = a.wt + (size_t)r0 * W;

    float2 v[16];
    if (has1 && W == M) {
        // whole row pair inside the detector: no per-column tests; the weights
        // of the second row are loaded after the first row is done
        InT x0[16], x1[16];
        float wv[16];
#pragma unroll
        for (int r = 0; r < 16; ++r) {
            x0[r] = src[lt + L * r];
            x1[r] = src[W + lt + L * r];
            wv[r] = __ldg(wrow + lt + L * r);
        }
#pragma unroll
        for (int r = 0; r < 16; ++r) v[r].x = __fmul_rn(log_part(raw_value(&x0[r], a), a), wv[r]);
#pragma unroll
        for (int r = 0; r < 16; ++r) wv[r] = __ldg(wrow + W + lt + L * r);
#pragma unroll
        for (int r = 0; r < 16; ++r) v[r].y = __fmul_rn(log_part(raw_value(&x1[r], a), a), wv[r]);
    } else {
        // all 64 loads of the thread (16 columns x 2 rows, samples and weights)
        // are issued before any arithmetic
        InT x0[16], x1[16];
        float w0[16], w1[16];
#pragma unroll
        for (int r = 0; r < 16; ++r) {
            const int c = lt + L * r;
            const bool in = active && c < W;
            x0[r] = in ? src[c] : InT(0);
            x1[r] = in && has1 ? src[W + c] : InT(0);
            w0[r] = in ? __ldg(wrow + c) : 0.0f;
            w1[r] = in && has1 ? __ldg(wrow + W + c) : 0.0f;
        }
#pragma unroll
        for (int r = 0; r < 16; ++r) {
            const int c = lt + L * r;
            float2 z = make_float2(0.f, 0.f);
            if (active && c < W) {
                z.x = __fmul_rn(log_part(raw_value(&x0[r], a), a), w0[r]);
                if (has1) z.y = __fmul_rn(log_part(raw_value(&x1[r], a), a), w1[r]);
            }
            v[r] = z;
        }
    }
    // pass 1
    dft16<false>(v);
#pragma unroll
    for (int s = 1; s < 16; ++s) v[s] = cmul(v[s], __ldg(&tw[lt * s]));
#pragma unroll
    for (int s = 0; s < 16; ++s) sa[s * (L + L2) + lt] = v[s];
    __syncthreads();
    // pass 2
    const int ps = lt / L2, t2 = lt % L2;
    float2* bs = sa + (C::ALIAS ? 0 : C::SA) + ps * C::SB;
#pragma unroll
    for (int r = 0; r < 16; ++r) v[r] = sa[ps * (L + L2) + t2 + L2 * r];
    dft16<false>(v);
#pragma unroll
    for (int s2 = 1; s2 < 16; ++s2) v[s2] = cmul(v[s2], __ldg(&tw[16 * t2 * s2]));
    if (C::ALIAS) __syncthreads();  // the second transpose overwrites the first
#pragma unroll
    for (int s2 = 0; s2 < 16; ++s2) bs[s2 * (L2 + 1) + t2] = v[s2];
    __syncwarp();
    // pass 3, the kernel spectrum, inverse pass 3
    {
        float2 u[Q][L2];
#pragma unroll
        for (int qq = 0; qq < Q; ++qq)
#pragma unroll
            for (int k = 0; k < L2; ++k) u[qq][k] = bs[(t2 + L2 * qq) * (L2 + 1) + k];
#pragma unroll
        for (int qq = 0; qq < Q; ++qq) {
            dft_n<L2, false>(u[qq]);
#pragma unroll
            for (int k3 = 0; k3 < L2; ++k3) {
                const float kf = __ldg(&K[ps + 16 * (t2 + L2 * qq) + 256 * k3]);
                u[qq][k3] = make_float2(u[qq][k3].x * kf, u[qq][k3].y * kf);
            }
            dft_n<L2, true>(u[qq]);
        }
        __syncwarp();
#pragma unroll
        for (int qq = 0; qq < Q; ++qq)
#pragma unroll
            for (int k = 0; k < L2; ++k) bs[(t2 + L2 * qq) * (L2 + 1) + k] = u[qq][k];
        __syncwarp();
    }
    // inverse pass 2
#pragma unroll
    for (int s2 = 0; s2 < 16; ++s2) v[s2] = bs[s2 * (L2 + 1) + t2];
#pragma unroll
    for (int s2 = 1; s2 < 16; ++s2) v[s2] = cmul_conj(v[s2], __ldg(&tw[16 * t2 * s2]));
    dft16<true>(v);
    __syncthreads();  // every warp has read its pass-2 values from sa
#pragma unroll
    for (int r = 0; r < 16; ++r) sa[ps * (L + L2) + t2 + L2 * r] = v[r];
    __syncthreads();
    // inverse pass 1 and the filtered rows
#pragma unroll
    for (int s = 0; s < 16; ++s) v[s] = sa[s * (L + L2) + lt];
#pragma unroll
    for (int s = 1; s < 16; ++s) v[s] = cmul_conj(v[s], __ldg(&tw[lt * s]));
    dft16<true>(v);
    const size_t obase = (size_t)view * H * a.out_pitch + (size_t)r0 * a.out_pitch;
#pragma unroll
    for (int r = 0; r < 16; ++r) {
        const int c = lt + L * r;
        if (active && c < W) {
            out[obase + c] = to_store<OutT>(v[r].x * a.store_scale);
            if (has1) out[obase + a.out_pitch + c] = to_store<OutT>(v[r].y * a.store_scale);
        }
    }
}

template <int M, typename InT, typename OutT>
int launch_rf(const InT* raw, OutT* out, const FilterArgs& a, const float2* tw, const float* K, cudaStream_t s) {
    using C = RF<M>;
    const long long pairs = a.n_views * ((a.H + 1) / 2);
    const long long blocks = (pairs + C::G - 1) / C::G;
    if (blocks <= 0) return CTB_OK;
    if (blocks > 0x7fffffffLL) {
        set_global_error("filter: too many rows for one launch");
        return CTB_ERR_UNSUPPORTED;
    }
    const size_t smem = size_t(C::G) * C::SG * sizeof(float2);
    auto kern = filter_rf_kernel<M, InT, OutT>;
    if (const int st = ensure_dynamic_smem(reinterpret_cast<const void*>(kern), smem)) return st;
    kern<<<unsigned(blocks), 256, smem, s>>>(raw, out, a, tw, K);
    return cuda_status(cudaGetLastError(), "filter_rf_kernel launch");
}

template <typename InT, typename OutT>
int launch_typed(const InT* raw, OutT* out, const FilterArgs& a, const float2* tw, const float* K,
                 cudaStream_t s) {
    const int TG = a.M / 8;
    const int groups = TG >= 256 ? 1 : 256 / TG;
    const int threads = groups * TG;
    const long long pairs = a.n_views * ((a.H + 1) / 2);
    const long long blocks = (pairs + groups - 1) / groups;
    const size_t smem = (size_t)groups * a.M * sizeof(float2);
    if (blocks <= 0) return CTB_OK;
    if (blocks > 0x7fffffffLL) {
        set_global_error("filter: too many rows for one launch");
        return CTB_ERR_UNSUPPORTED;
    }
    const bool tab = a.wt != nullptr;
    if (tab) {
        switch (a.M) {
            case 512: return launch_rf<512>(raw, out, a, tw, K, s);
            case 1024: return launch_rf<1024>(raw, out, a, tw, K, s);
            case 2048: return launch_rf<2048>(raw, out, a, tw, K, s);
            case 4096: return launch_rf<4096>(raw, out, a, tw, K, s);
        }
    }
    auto kern = tab ? filter_kernel<InT, OutT, true> : filter_kernel<InT, OutT, false>;
    if (smem > 48 * 1024)
        if (const int st = ensure_dynamic_smem(reinterpret_cast<const void*>(kern), smem)) return st;
    kern<<<unsigned(blocks), threads, smem, s>>>(raw, out, a, tw, K);
    return cuda_status(cudaGetLastError(), "filter_kernel launch");
}

template <typename InT>
int launch_out(const InT* raw, void* out, int store_type, const FilterArgs& a, const float2* tw,
               const float* K, cudaStream_t s) {
    switch (store_type) {
        case CTB_FP32: return launch_typed(raw, (float*)out, a, tw, K, s);
        case CTB_FP16: return launch_typed(raw, (__half*)out, a, tw, K, s);
        case CTB_BF16: return launch_typed(raw, (__nv_bfloat16*)out, a, tw, K, s);
    }
    set_global_error("filter: unknown storage type");
    return CTB_ERR_ARG;
}

}  // namespace

int filter_transform_length(int W, int pad) {
    if (W < 2) return 0;
    auto nextpow2 = [](long long n) { long long m = 1; while (m < n) m <<= 1; return m; };
    long long M;
    if (pad <= 1) M = ((W & (W - 1)) == 0) ? W : nextpow2(2LL * W - 1);
    else M = nextpow2(2LL * W);
    if (M < 8) M = 8;
    return M > kMaxFftLen ? 0 : int(M);
}

int filter_build_tables(int W, int pad, int filter, int M, float2* tw, float* K, cudaStream_t s) {
    const int T = 256;
    twiddle_kernel<<<(M + T - 1) / T, T, 0, s>>>(tw, M);
    CTB_CUDA_TRY(cudaGetLastError());
    if (pad >= 2) {
        kernel_padded<<<(M + T - 1) / T, T, 0, s>>>(K, M, W, filter);
    } else if (M == W) {
        kernel_direct<<<(M + T - 1) / T, T, 0, s>>>(K, M, filter);
    } else {
        double* g = nullptr;
        CTB_CUDA_TRY(cudaMallocAsync((void**)&g, sizeof(double) * W, s));
        spatial_kernel<<<(W + T - 1) / T, T, 0, s>>>(g, W, filter);
        embedded_kernel<<<(M + T - 1) / T, T, 0, s>>>(K, g, W, M);
        CTB_CUDA_TRY(cudaFreeAsync(g, s));
    }
    return cuda_status(cudaGetLastError(), "filter table kernels");
}

FilterArgs filter_args(const ctb_detector& det, int raw_type, int M, int logM, long long n_views,
                       float store_scale) {
    FilterArgs a;
    a.W = det.width;
    a.H = det.height;
    a.M = M;
    a.logM = logM;
    a.n_views = n_views;
    const double base = det.base_intensity;
    a.alpha = float(raw_type == CTB_U8 ? 1.0 / 255.0 : 1.0 / 65535.0);
    a.beta = float(0.000001 * base);
    a.log_scale = float(1.0 / (base + 0.000001 * base));
    a.D = det.fcd;
    a.uPre = float(double(det.width) / 2.0);
    a.vPre = float(double(det.height) / 2.0);
    a.store_scale = store_scale;
    a.out_pitch = det.width;
    return a;
}

namespace {
__global__ void weight_table_kernel(float* t, FilterArgs a) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int r = blockIdx.y;
    if (c >= a.W) return;
    t[(size_t)r * a.W + c] = weight_part(r, c, a);
}
}  // namespace

int build_weight_table(const FilterArgs& a, float* t, cudaStream_t s) {
    if (a.H > 65535) return CTB_ERR_UNSUPPORTED;
    weight_table_kernel<<<dim3((a.W + 255) / 256, a.H), 256, 0, s>>>(t, a);
    return cuda_status(cudaGetLastError(), "weight_table_kernel launch");
}

int filter_launch(const void* raw, int raw_type, void* out, int store_type, const FilterArgs& args,
                  const float2* tw, const float* K, cudaStream_t s) {
    FilterArgs a = args;
    if (!a.wt) {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        if (cudaStreamIsCapturing(s, &cs) != cudaSuccess) cudaGetLastError();
        const int st = pre_tables(&a, s, cs == cudaStreamCaptureStatusNone);
        if (st != CTB_OK) return st;
    }
    switch (raw_type) {
        case CTB_U8: return launch_out((const uint8_t*)raw, out, store_type, a, tw, K, s);
        case CTB_U16: return launch_out((const uint16_t*)raw, out, store_type, a, tw, K, s);
        case CTB_F32: return launch_out((const float*)raw, out, store_type, a, tw, K, s);
    }
    set_global_error("filter: unknown raw pixel type");
    return CTB_ERR_ARG;
}

}  // namespace ctb
