// Autotuner of the facade's backprojection: the block tile height (z voxels
// per thread), the views in flight (projection boxes staged per CTA) and the
// slab height, picked by timing the context's own scan on its first active
// device and remembered per scan/box shape for the rest of the process. No
// counterpart in the reference, which sizes its z-chunks by free memory only
// (getMaxChunkSize, Ct/CtVolume.cpp:1385-1397).
//
// The timing runs on an evenly spaced subset of the views (at most 180),
// filtered once; each candidate launch shape backprojects the central slab,
// then each candidate slab height the whole box, and the fastest device time
// (CUDA events) wins. Backprojection time is linear in the views, so the
// subset ranks the candidates as the whole scan would.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <sstream>

#include "../ctb_internal.h"
#include "reconstructor.h"

namespace ctb {

namespace {

struct Tuned {
    int zc = 0, nbuf = 0, slab = 0;
    double ms = 0;
};
std::mutex g_tuned_mtx;
std::map<std::string, Tuned> g_tuned;

struct Events {
    cudaEvent_t a = nullptr, b = nullptr;
    Events() {
        cudaEventCreate(&a);
        cudaEventCreate(&b);
    }
    ~Events() {
        cudaEventDestroy(a);
        cudaEventDestroy(b);
    }
};

}  // namespace

std::string Reconstructor::tune_key(int z_lo, int z_hi) const {
    std::ostringstream k;
    const int V = (int(angles_.size()) + std::max(1, step_) - 1) / std::max(1, step_);
    k << store_ << ':' << det_.width << 'x' << det_.height << ':' << V << ':' << det_.fcd << ':'
      << (grid_.x_to - grid_.x_from) << 'x' << (grid_.y_to - grid_.y_from) << 'x' << (z_hi - z_lo) << ':'
      << grid_.voxel_pitch;
    return k.str();
}

bool Reconstructor::tuned_for(int z_lo, int z_hi, BpConfig* cfg, int* slab) const {
    std::lock_guard<std::mutex> lk(g_tuned_mtx);
    auto it = g_tuned.find(tune_key(z_lo, z_hi));
    if (it == g_tuned.end()) return false;
    cfg->zc = it->second.zc;
    cfg->nbuf = it->second.nbuf;
    *slab = it->second.slab;
    return true;
}

int Reconstructor::autotune(ctb_tuning* out) {
    std::lock_guard<std::mutex> lk(mtx_);
    return autotune_locked(out);
}

int Reconstructor::autotune_locked(ctb_tuning* out) {
    if (!have_scan_) return fail(CTB_ERR_ARG, "No projections are loaded.");
    const int W = det_.width, H = det_.height;
    const int X = grid_.x_to - grid_.x_from, Y = grid_.y_to - grid_.y_from, Z = grid_.z_to - grid_.z_from;
    if (X <= 0 || Y <= 0 || Z <= 0) return fail(CTB_ERR_ARG, "The reconstructed box is empty.");
    const std::string key = tune_key(0, Z);
    {
        std::lock_guard<std::mutex> g(g_tuned_mtx);
        auto it = g_tuned.find(key);
        if (it != g_tuned.end()) {
            if (out) *out = ctb_tuning{it->second.slab, it->second.zc, it->second.nbuf, it->second.ms, 1};
            return CTB_OK;
        }
    }
    const int dev = devices_.empty() ? 0 : devices_[0];
    int prev = 0;
    CTB_CUDA_TRY(cudaGetDevice(&prev));
    CTB_CUDA_TRY(cudaSetDevice(dev));
    struct Restore {
        int d;
        ~Restore() { cudaSetDevice(d); }
    } restore{prev};

    // views used (skip setting), then an evenly spaced subset of them
    std::vector<int> used;
    for (int p = 0; p < int(angles_.size()); p += std::max(1, step_)) used.push_back(p);
    const int Vs = std::min<int>(int(used.size()), 180);
    std::vector<double> ang(Vs), hp(Vs);
    std::vector<int> pick(Vs);
    double hmax = 0;
    for (int i = 0; i < Vs; ++i) {
        pick[i] = used[size_t(i) * used.size() / Vs];
        ang[i] = angles_[pick[i]];
        hp[i] = heights_px_[pick[i]];
        hmax = std::max(hmax, std::fabs(hp[i]));
    }
    const int M = filter_transform_length(W, pad_);
    if (M == 0) return fail(CTB_ERR_UNSUPPORTED, "Detector width exceeds the largest supported FFT length.");
    int logM = 0;
    while ((1 << logM) < M) ++logM;
    const float store_scale = store_ == CTB_FP32 ? 1.0f : 1.0f / float(W);
    const float load_scale = store_ == CTB_FP32 ? 1.0f : float(W);
    const int pitch = (W + 7) / 8 * 8;
    const size_t view_raw = size_t(W) * H * raw_bytes(raw_type_);
    const size_t view_filt = size_t(pitch) * H * store_bytes(store_);
    const size_t plane = size_t(X) * Y;
    const int slab_max = std::min(Z, std::max(16, ((Z + 3) / 4 + 15) / 16 * 16));

    cudaStream_t s = nullptr;
    CTB_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() { cudaStreamDestroy(s); }
    } sg{s};
    DevBuf d_raw, d_filt, d_vol, d_views, d_ang, d_h, d_tw, d_K;
    int st;
    if ((st = d_raw.ensure(view_raw * Vs, "tuning projections")) ||
        (st = d_filt.ensure(view_filt * Vs, "tuning filtered projections")) ||
        (st = d_vol.ensure(sizeof(float) * plane * slab_max, "tuning slab")) ||
        (st = d_views.ensure(sizeof(float4) * Vs, "tuning view table")) ||
        (st = d_ang.ensure(sizeof(double) * Vs, "tuning angles")) ||
        (st = d_h.ensure(sizeof(double) * Vs, "tuning heights")) ||
        (st = d_tw.ensure(sizeof(float2) * M, "tuning twiddles")) ||
        (st = d_K.ensure(sizeof(float) * M, "tuning filter")))
        return fail(st, global_error());
    for (int i = 0; i < Vs; ++i)
        CTB_CUDA_TRY(cudaMemcpyAsync((char*)d_raw.p + view_raw * i, (const char*)images_ + view_raw * pick[i],
                                     view_raw, cudaMemcpyHostToDevice, s));
    CTB_CUDA_TRY(cudaMemcpyAsync(d_ang.p, ang.data(), sizeof(double) * Vs, cudaMemcpyHostToDevice, s));
    CTB_CUDA_TRY(cudaMemcpyAsync(d_h.p, hp.data(), sizeof(double) * Vs, cudaMemcpyHostToDevice, s));
    if ((st = view_table_build((double*)d_ang.p, (double*)d_h.p, Vs, (float4*)d_views.p, s)) ||
        (st = filter_build_tables(W, pad_, filter_, M, (float2*)d_tw.p, (float*)d_K.p, s)))
        return fail(st, global_error());
    FilterArgs fa = filter_args(det_, raw_type_, M, logM, Vs, store_scale);
    fa.out_pitch = pitch;
    if ((st = filter_launch(d_raw.p, raw_type_, d_filt.p, store_, fa, (const float2*)d_tw.p, (const float*)d_K.p, s)))
        return fail(st, global_error());

    Events ev;
    auto geom = [&](int zb, int ze) {
        ProjGeom g = proj_geom(det_, grid_, zb, ze, load_scale);
        g.pitch = pitch;
        g.view_stride = (long long)pitch * H;
        return g;
    };
    // device time of backprojecting slices [zb, ze) in slabs of `slab` with cfg; < 0 if a launch is refused
    auto time_bp = [&](int zb, int ze, int slab, BpConfig cfg) -> double {
        for (int rep = 0; rep < 2; ++rep) {   // the first pass warms up
            if (rep == 1) cudaEventRecord(ev.a, s);
            for (int z = zb; z < ze; z += slab) {
                const int z1 = std::min(ze, z + slab);
                if (backproject_launch(d_filt.p, store_, (const float4*)d_views.p, Vs, geom(z, z1), hmax,
                                       (float*)d_vol.p, 0, s, cfg) != CTB_OK) {
                    cudaStreamSynchronize(s);
                    cudaGetLastError();
                    return -1.0;
                }
            }
        }
        cudaEventRecord(ev.b, s);
        if (cudaStreamSynchronize(s) != cudaSuccess) return -1.0;
        float ms = 0;
        cudaEventElapsedTime(&ms, ev.a, ev.b);
        return ms;
    };

    // 1. launch shape on the central slab
    const int zc_mid = std::max(0, Z / 2 - slab_max / 2);
    const BpConfig shapes[] = {{0, 0}, {32, 2}, {32, 3}, {32, 4}, {16, 3}, {16, 4}};
    BpConfig best_cfg;
    double best = -1;
    for (const BpConfig& c : shapes) {
        const double ms = time_bp(zc_mid, std::min(Z, zc_mid + slab_max), slab_max, c);
        if (ms >= 0 && (best < 0 || ms < best)) {
            best = ms;
            best_cfg = c;
        }
    }
    if (best < 0) return fail(CTB_ERR_CUDA, "autotune: no backprojection launch shape could run");
    // 2. slab height over the whole box
    int best_slab = slab_max;
    double best_all = -1;
    for (int sl : {slab_max, std::max(16, (slab_max / 2 + 15) / 16 * 16)}) {
        sl = std::min(sl, slab_max);
        const double ms = time_bp(0, Z, sl, best_cfg);
        if (ms >= 0 && (best_all < 0 || ms < best_all)) {
            best_all = ms;
            best_slab = sl;
        }
    }
    unsigned gave_up = 0;
    if (device_wait_timeouts(&gave_up, 1) == CTB_OK && gave_up)
        return fail(CTB_ERR_TIMEOUT, "autotune: a device wait of the backprojection gave up");
    Tuned t;
    t.zc = best_cfg.zc;
    t.nbuf = best_cfg.nbuf;
    t.slab = best_slab;
    t.ms = best_all * double(used.size()) / double(Vs);   // scaled to every used view
    {
        std::lock_guard<std::mutex> g(g_tuned_mtx);
        g_tuned[key] = t;
    }
    if (out) *out = ctb_tuning{t.slab, t.zc, t.nbuf, t.ms, 1};
    return CTB_OK;
}

int Reconstructor::tuning(ctb_tuning* out) const {
    const int Z = grid_.z_to - grid_.z_from;
    BpConfig cfg;
    int slab = 0;
    if (have_scan_ && tuned_for(0, Z, &cfg, &slab)) {
        *out = ctb_tuning{slab, cfg.zc, cfg.nbuf, 0.0, 1};
        std::lock_guard<std::mutex> g(g_tuned_mtx);
        out->backproject_ms = g_tuned[tune_key(0, Z)].ms;
    } else {
        *out = ctb_tuning{0, 0, 0, 0.0, 0};
    }
    return CTB_OK;
}

}  // namespace ctb
