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
__device__ __forceinline__ float preprocess(float s, int r, int c, const FilterArgs& a) {
    const float p = -logf(__fmul_rn(s, a.log_scale));
    const float u = __fsub_rn(float(c), a.uPre);
    const float v = __fadd_rn(-float(r), a.vPre);
    const float d2 = __fadd_rn(__fadd_rn(__fmul_rn(a.D, a.D), __fmul_rn(u, u)), __fmul_rn(v, v));
    return __fmul_rn(p, __fdiv_rn(a.D, __fsqrt_rn(d2)));
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// In-place Stockham autosort FFT of length M (power of two) on s[0..M), by TG =
// M/8 threads (lt = 0..TG-1). Forward: exp(-2 pi i nk/M); inverse: conjugate
// twiddles, unnormalised. All threads of the CTA must call it (barriers).
template <bool INV>
__device__ void fft_smem(float2* s, int M, int logM, const float2* __restrict__ tw, int lt, int TG) {
    int Ns = 1;
    if (logM & 1) {
        // radix-2 first stage (Ns = 1: no twiddles), 4 butterflies per thread
        const int nb = M >> 1;
        float2 y[4][2];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int b = lt + i * TG;
            const float2 v0 = s[b], v1 = s[b + nb];
            y[i][0] = make_float2(v0.x + v1.x, v0.y + v1.y);
            y[i][1] = make_float2(v0.x - v1.x, v0.y - v1.y);
        }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int b = lt + i * TG;
            s[2 * b] = y[i][0];
            s[2 * b + 1] = y[i][1];
        }
        __syncthreads();
        Ns = 2;
    }
    const int nb = M >> 2;
    for (; Ns < M; Ns <<= 2) {
        float2 y[2][4];
        const int step = M / (Ns * 4);
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const int b = lt + i * TG;
            const int jm = b & (Ns - 1);
            float2 v[4];
#pragma unroll
            for (int r = 0; r < 4; ++r) v[r] = s[b + r * nb];
            if (Ns > 1) {
#pragma unroll
                for (int r = 1; r < 4; ++r) {
                    float2 w = __ldg(&tw[(jm * r * step) & (M - 1)]);
                    if (INV) w.y = -w.y;
                    v[r] = cmul(v[r], w);
                }
            }
            const float2 a0 = make_float2(v[0].x + v[2].x, v[0].y + v[2].y);
            const float2 a1 = make_float2(v[0].x - v[2].x, v[0].y - v[2].y);
            const float2 a2 = make_float2(v[1].x + v[3].x, v[1].y + v[3].y);
            const float2 d = make_float2(v[1].x - v[3].x, v[1].y - v[3].y);
            // forward: a3 = -i * d ; inverse: a3 = +i * d
            const float2 a3 = INV ? make_float2(-d.y, d.x) : make_float2(d.y, -d.x);
            y[i][0] = make_float2(a0.x + a2.x, a0.y + a2.y);
            y[i][1] = make_float2(a1.x + a3.x, a1.y + a3.y);
            y[i][2] = make_float2(a0.x - a2.x, a0.y - a2.y);
            y[i][3] = make_float2(a1.x - a3.x, a1.y - a3.y);
        }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const int b = lt + i * TG;
            const int jm = b & (Ns - 1);
            const int d0 = (b - jm) * 4 + jm;
#pragma unroll
            for (int r = 0; r < 4; ++r) s[d0 + r * Ns] = y[i][r];
        }
        __syncthreads();
    }
}

// One group of TG = M/8 threads per detector row pair; groups = blockDim/TG.
template <typename InT, typename OutT>
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
    const size_t base0 = (size_t)view * H * W + (size_t)r0 * W;

    for (int c = lt; c < M; c += TG) {
        float2 z = make_float2(0.f, 0.f);
        if (active && c < W) {
            z.x = preprocess(raw_value(raw + base0 + c, a), r0, c, a);
            if (has1) z.y = preprocess(raw_value(raw + base0 + W + c, a), r0 + 1, c, a);
        }
        s[c] = z;
    }
    __syncthreads();
    fft_smem<false>(s, M, a.logM, tw, lt, TG);
    for (int k = lt; k < M; k += TG) {
        const float kk = __ldg(&K[k]);
        float2 z = s[k];
        s[k] = make_float2(z.x * kk, z.y * kk);
    }
    __syncthreads();
    fft_smem<true>(s, M, a.logM, tw, lt, TG);
    if (active) {
        for (int c = lt; c < W; c += TG) {
            const float2 z = s[c];
            out[base0 + c] = to_store<OutT>(z.x * a.store_scale);
            if (has1) out[base0 + W + c] = to_store<OutT>(z.y * a.store_scale);
        }
    }
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
    auto kern = filter_kernel<InT, OutT>;
    if (smem > 48 * 1024)
        CTB_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
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
    return a;
}

int filter_launch(const void* raw, int raw_type, void* out, int store_type, const FilterArgs& a,
                  const float2* tw, const float* K, cudaStream_t s) {
    switch (raw_type) {
        case CTB_U8: return launch_out((const uint8_t*)raw, out, store_type, a, tw, K, s);
        case CTB_U16: return launch_out((const uint16_t*)raw, out, store_type, a, tw, K, s);
        case CTB_F32: return launch_out((const float*)raw, out, store_type, a, tw, K, s);
    }
    set_global_error("filter: unknown raw pixel type");
    return CTB_ERR_ARG;
}

}  // namespace ctb
