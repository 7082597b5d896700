// Process-wide cache of filter tables (twiddles + kernel spectrum) per
// (device, W, pad, filter), shared by the operator layer and batches.
#include <map>
#include <mutex>
#include <tuple>

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

}  // namespace ctb
