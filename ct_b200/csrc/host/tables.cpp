// Process-wide caches of the filter tables (twiddles + kernel spectrum) per
// (device, W, pad, filter) and of the Feldkamp weight tables per device and
// detector geometry, shared by the operator layer, the facade and batches.
#include <cstring>
#include <functional>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "../ctb_internal.h"

namespace ctb {

namespace {
struct Key {
    int dev, W, pad, filter;
    bool operator<(const Key& o) const { return std::tie(dev, W, pad, filter) < std::tie(o.dev, o.W, o.pad, o.filter); }
};
std::mutex g_mtx;
std::map<Key, FilterTables> g_tables;
}  // namespace

int filter_tables(int W, int pad, int filter, cudaStream_t s, FilterTables* out) {
    int dev = 0;
    CTB_CUDA_TRY(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(g_mtx);
    const Key key{dev, W, pad, filter};
    auto it = g_tables.find(key);
    if (it != g_tables.end()) {
        *out = it->second;
        return CTB_OK;
    }
    FilterTables t;
    t.M = filter_transform_length(W, pad);
    if (t.M == 0) {
        set_global_error("detector width exceeds the largest supported FFT length");
        return CTB_ERR_UNSUPPORTED;
    }
    while ((1 << t.logM) < t.M) ++t.logM;
    float2* tw = nullptr;
    float* K = nullptr;
    CTB_CUDA_TRY(cudaMalloc(&tw, sizeof(float2) * t.M));
    CTB_CUDA_TRY(cudaMalloc(&K, sizeof(float) * t.M));
    const int st = filter_build_tables(W, pad, filter, t.M, tw, K, s);
    if (st != CTB_OK) return st;
    CTB_CUDA_TRY(cudaStreamSynchronize(s));
    t.tw = tw;
    t.K = K;
    g_tables[key] = t;
    *out = t;
    return CTB_OK;
}

namespace {
uint32_t bits(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
}
// (device, W, H, D, uPre, vPre) -> weight table
using PreKey = std::tuple<int, int, int, uint32_t, uint32_t, uint32_t>;
std::map<PreKey, float*> g_pre;
size_t g_pre_bytes = 0;
constexpr size_t kPreBudget = size_t(512) << 20;  // above this the cache is emptied first

int pre_table(const PreKey& key, size_t n, bool build, const std::function<int(float*)>& make, const float** out) {
    auto it = g_pre.find(key);
    if (it != g_pre.end()) {
        *out = it->second;
        return CTB_OK;
    }
    *out = nullptr;
    if (!build) return CTB_OK;
    if (g_pre_bytes + n * sizeof(float) > kPreBudget) {
        // cudaFree waits for the work that may still read these tables
        for (auto& kv : g_pre) cudaFree(kv.second);
        g_pre.clear();
        g_pre_bytes = 0;
    }
    float* t = nullptr;
    if (cudaMalloc(&t, n * sizeof(float)) != cudaSuccess) {
        cudaGetLastError();
        return CTB_OK;  // no table: the filter evaluates per pixel
    }
    const int st = make(t);
    if (st != CTB_OK) {
        cudaFree(t);
        return st;
    }
    g_pre[key] = t;
    g_pre_bytes += n * sizeof(float);
    *out = t;
    return CTB_OK;
}
}  // namespace

int pre_tables(FilterArgs* a, cudaStream_t s, bool build) {
    int dev = 0;
    CTB_CUDA_TRY(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(g_mtx);
    const PreKey k{dev, a->W, a->H, bits(a->D), bits(a->uPre), bits(a->vPre)};
    return pre_table(k, size_t(a->W) * a->H, build, [&](float* t) {
        int r = build_weight_table(*a, t, s);
        if (r == CTB_OK) r = cuda_status(cudaStreamSynchronize(s), "weight table");
        return r;
    }, &a->wt);
}

}  // namespace ctb
