// Batches of independent scans (ctb_batch_*): per-scan filtering into padded
// filtered-projection buffers, then one persistent backprojection launch over
// all (scan, tile) work items, captured once as a CUDA graph.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <new>
#include <string>
#include <vector>

#include "../ctb_internal.h"
#include "autotune.h"

struct ctb_batch {
    int device = 0;
    int store = CTB_FP32;
    std::vector<ctb_scan> scans;
    std::vector<void*> filtered;     // per scan, V x H x pitch
    std::vector<float4*> views;      // per scan view tables
    std::vector<int> pitch;
    std::vector<ctb::FilterTables> tables;
    std::vector<ctb::BpBatchScan> bp;
    ctb::BpBatchPlan plan;
    void* d_desc = nullptr;
    long long* d_tile_start = nullptr;
    unsigned long long* d_queue = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int zc = 16, nbuf = 0;
    double ms32 = -1, ms16 = -1, ms8 = -1;   // best time per z voxels per thread
    std::vector<int> cand_zc, cand_nbuf;     // every timed candidate
    std::vector<double> cand_ms;
    // side stream and events of the scans left out of the persistent kernel
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;

    ~ctb_batch() {
        cudaSetDevice(device);
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (ev_fork) cudaEventDestroy(ev_fork);
        if (ev_join) cudaEventDestroy(ev_join);
        if (side) cudaStreamDestroy(side);
        for (void* p : filtered) cudaFree(p);
        for (float4* p : views) cudaFree(p);
        cudaFree(d_desc);
        cudaFree(d_tile_start);
        cudaFree(d_queue);
    }
};

namespace ctb {
namespace {

int fail(const std::string& m, int st) {
    set_global_error(m);
    return st;
}

// Filter every scan into its padded buffer.
int enqueue_filters(ctb_batch* b, cudaStream_t s) {
    for (size_t i = 0; i < b->scans.size(); ++i) {
        const ctb_scan& sc = b->scans[i];
        const float scale = b->store == CTB_FP32 ? 1.0f : 1.0f / float(sc.det.width);
        FilterArgs a = filter_args(sc.det, sc.raw_type, b->tables[i].M, b->tables[i].logM, sc.n_views, scale);
        a.out_pitch = b->pitch[i];
        const int st = filter_launch(sc.raw, sc.raw_type, b->filtered[i], b->store, a, b->tables[i].tw,
                                     b->tables[i].K, s);
        if (st != CTB_OK) return st;
    }
    return CTB_OK;
}

int upload_plan(ctb_batch* b, cudaStream_t s) {
    cudaFree(b->d_desc);
    cudaFree(b->d_tile_start);
    b->d_desc = nullptr;
    b->d_tile_start = nullptr;
    if (b->plan.desc.empty()) return CTB_OK;
    CTB_CUDA_TRY(cudaMalloc(&b->d_desc, b->plan.desc.size()));
    CTB_CUDA_TRY(cudaMalloc(&b->d_tile_start, sizeof(long long) * b->plan.tile_start.size()));
    CTB_CUDA_TRY(cudaMemcpyAsync(b->d_desc, b->plan.desc.data(), b->plan.desc.size(), cudaMemcpyHostToDevice, s));
    CTB_CUDA_TRY(cudaMemcpyAsync(b->d_tile_start, b->plan.tile_start.data(),
                                 sizeof(long long) * b->plan.tile_start.size(), cudaMemcpyHostToDevice, s));
    return CTB_OK;
}

int enqueue_batch(ctb_batch* b, cudaStream_t s) {
    int st = enqueue_filters(b, s);
    if (st != CTB_OK) return st;
    // scans left out of the persistent kernel (box beyond its budget): one launch
    // each, shared-memory kernel with its own buffer size when possible, else
    // global gathers. They go on a side stream forked here, so their few long
    // CTAs run beside the persistent kernel's instead of after it (the
    // persistent kernel takes its work from a queue, so CTAs that start late
    // only take fewer items); the side stream joins back before the end.
    const bool fork = !b->plan.excluded.empty() && b->side;
    cudaStream_t sx = fork ? b->side : s;
    if (fork) {
        CTB_CUDA_TRY(cudaEventRecord(b->ev_fork, s));
        CTB_CUDA_TRY(cudaStreamWaitEvent(sx, b->ev_fork, 0));
    }
    for (int i : b->plan.excluded) {
        st = backproject_launch(b->filtered[i], b->store, b->views[i], b->bp[i].n_views, b->bp[i].g, b->bp[i].hmax,
                                b->bp[i].vol, 0, sx);
        if (st != CTB_OK) return st;
    }
    if (fork) CTB_CUDA_TRY(cudaEventRecord(b->ev_join, sx));
    CTB_CUDA_TRY(cudaMemsetAsync(b->d_queue, 0, sizeof(unsigned long long), s));
    st = bp_batch_launch(b->plan, b->d_desc, b->d_tile_start, int(b->plan.included.size()), b->d_queue, s);
    if (st != CTB_OK) return st;
    if (fork) CTB_CUDA_TRY(cudaStreamWaitEvent(s, b->ev_join, 0));
    return CTB_OK;
}

}  // namespace
}  // namespace ctb

extern "C" {

int ctb_batch_create(ctb_batch** out, int n, const ctb_scan* scans, int store_type, void* stream) {
    using namespace ctb;
    if (!out || n <= 0 || !scans) return fail("ctb_batch_create: invalid arguments", CTB_ERR_ARG);
    if (store_type != CTB_FP32 && store_type != CTB_FP16 && store_type != CTB_BF16)
        return fail("ctb_batch_create: unknown storage type", CTB_ERR_ARG);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    ctb_batch* b = new (std::nothrow) ctb_batch();
    if (!b) return CTB_ERR_ALLOC;
    auto bail = [&](int st) {
        delete b;
        return st;
    };
    cudaGetDevice(&b->device);
    b->store = store_type;
    b->scans.assign(scans, scans + n);
    const size_t es = store_bytes(store_type);
    for (int i = 0; i < n; ++i) {
        const ctb_scan& sc = b->scans[i];
        if (!sc.raw || !sc.vol || !sc.angles_deg || sc.n_views <= 0 || sc.det.width <= 1 || sc.det.height <= 1 ||
            !(sc.det.fcd > float(sc.det.width)) || sc.det.radius <= 0 || (sc.pad != 1 && sc.pad != 2) ||
            sc.filter < CTB_RAMLAK || sc.filter > CTB_HANN ||
            (sc.raw_type != CTB_U8 && sc.raw_type != CTB_U16 && sc.raw_type != CTB_F32) ||
            sc.grid.x_to <= sc.grid.x_from || sc.grid.y_to <= sc.grid.y_from || sc.grid.z_to <= sc.grid.z_from ||
            sc.grid.voxel_pitch <= 0)
            return bail(fail("ctb_batch_create: invalid scan " + std::to_string(i), CTB_ERR_ARG));
        // filtered rows padded to a 16-byte multiple for the tensor maps
        const int pitch = (sc.det.width + 7) / 8 * 8;
        b->pitch.push_back(pitch);
        void* f = nullptr;
        if (cudaMalloc(&f, es * size_t(sc.n_views) * sc.det.height * pitch) != cudaSuccess) {
            cudaGetLastError();
            return bail(fail("ctb_batch_create: out of device memory for filtered projections", CTB_ERR_ALLOC));
        }
        b->filtered.push_back(f);
        FilterTables t;
        int st = filter_tables(sc.det.width, sc.pad, sc.filter, s, &t);
        if (st != CTB_OK) return bail(st);
        b->tables.push_back(t);
        // preprocessing tables now: the filters are captured into a graph later
        FilterArgs pa = filter_args(sc.det, sc.raw_type, t.M, t.logM, sc.n_views, 1.0f);
        st = pre_tables(&pa, s, true);
        if (st != CTB_OK) return bail(st);
        // view table (FP64 geometry kernel)
        float4* v = nullptr;
        double* tmp = nullptr;
        if (cudaMalloc(&v, sizeof(float4) * sc.n_views) != cudaSuccess ||
            cudaMalloc(&tmp, sizeof(double) * 2 * sc.n_views) != cudaSuccess) {
            cudaGetLastError();
            cudaFree(v);
            return bail(fail("ctb_batch_create: out of device memory for view tables", CTB_ERR_ALLOC));
        }
        b->views.push_back(v);
        double hmax = 0;
        cudaMemcpyAsync(tmp, sc.angles_deg, sizeof(double) * sc.n_views, cudaMemcpyHostToDevice, s);
        if (sc.height_offsets_px) {
            cudaMemcpyAsync(tmp + sc.n_views, sc.height_offsets_px, sizeof(double) * sc.n_views,
                            cudaMemcpyHostToDevice, s);
            for (int k = 0; k < sc.n_views; ++k) hmax = std::max(hmax, std::fabs(sc.height_offsets_px[k]));
        } else {
            cudaMemsetAsync(tmp + sc.n_views, 0, sizeof(double) * sc.n_views, s);
        }
        st = view_table_build(tmp, tmp + sc.n_views, sc.n_views, v, s);
        cudaStreamSynchronize(s);
        cudaFree(tmp);
        if (st != CTB_OK) return bail(st);
        BpBatchScan bs;
        bs.proj = f;
        bs.views = v;
        bs.n_views = sc.n_views;
        const int Z = sc.grid.z_to - sc.grid.z_from;
        bs.g = proj_geom(sc.det, sc.grid, 0, Z, store_type == CTB_FP32 ? 1.0f : float(sc.det.width));
        bs.g.pitch = pitch;
        bs.g.view_stride = (long long)pitch * sc.det.height;
        bs.hmax = hmax;
        bs.vol = sc.vol;
        bs.accumulate = 0;
        b->bp.push_back(bs);
    }
    if (cudaStreamCreateWithFlags(&b->side, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->ev_join, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        return bail(fail("ctb_batch_create: stream or events could not be created", CTB_ERR_CUDA));
    }
    if (cudaMalloc(&b->d_queue, sizeof(unsigned long long)) != cudaSuccess) {
        cudaGetLastError();
        return bail(fail("ctb_batch_create: out of device memory", CTB_ERR_ALLOC));
    }
    // autotuner: the persistent kernel's block tile height (z voxels per thread)
    // and views in flight (projection boxes staged per CTA), timed on this batch
    std::string key = "batch:" + std::to_string(store_type) + ":" + std::to_string(n);
    for (const ctb_scan& sc : b->scans)
        key += ":" + std::to_string(sc.det.width) + "x" + std::to_string(sc.det.height) + "x" +
               std::to_string(sc.n_views) + "/" + std::to_string(sc.grid.x_to - sc.grid.x_from) + "x" +
               std::to_string(sc.grid.y_to - sc.grid.y_from) + "x" + std::to_string(sc.grid.z_to - sc.grid.z_from);
    std::vector<double> times;
    int plan_err = CTB_OK;
    // candidates zc * 10 + boxes in flight (0: the built-in choice for the box size)
    const std::vector<int> cands = {320, 322, 324, 160, 162, 164, 80};
    const int choice = Autotuner::instance().pick(
        key, cands,
        [&](int c) -> double {
            const int zc = c / 10, nb = c % 10;
            BpBatchPlan plan;
            if (bp_batch_plan(store_type, zc, b->bp.data(), n, &plan, nb) != CTB_OK) return -1.0;
            b->plan = plan;
            if (upload_plan(b, s) != CTB_OK) return -1.0;
            cudaEvent_t e0, e1;
            cudaEventCreate(&e0);
            cudaEventCreate(&e1);
            int st = enqueue_batch(b, s);  // warm-up (also fills the volumes)
            cudaEventRecord(e0, s);
            if (st == CTB_OK) st = enqueue_batch(b, s);
            cudaEventRecord(e1, s);
            cudaStreamSynchronize(s);
            float ms = -1;
            if (st == CTB_OK) cudaEventElapsedTime(&ms, e0, e1);
            else plan_err = st;
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            return st == CTB_OK ? double(ms) : -1.0;
        },
        &times);
    b->zc = choice / 10;
    b->nbuf = choice % 10;
    for (size_t i = 0; i < times.size() && i < cands.size(); ++i) {
        const int zc = cands[i] / 10;
        b->cand_zc.push_back(zc);
        b->cand_nbuf.push_back(cands[i] % 10);
        b->cand_ms.push_back(times[i]);
        double& best = zc == 32 ? b->ms32 : zc == 16 ? b->ms16 : b->ms8;
        if (times[i] >= 0 && (best < 0 || times[i] < best)) best = times[i];
    }
    int st = bp_batch_plan(store_type, b->zc, b->bp.data(), n, &b->plan, b->nbuf);
    if (st != CTB_OK)
        return bail(fail("ctb_batch_create: a scan does not suit the persistent backprojector", plan_err ? plan_err : st));
    st = upload_plan(b, s);
    if (st != CTB_OK) return bail(st);
    CTB_CUDA_TRY(cudaStreamSynchronize(s));
    // capture: queue reset + per-scan filters + persistent backprojection
    cudaStream_t cap;
    CTB_CUDA_TRY(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    if (cudaStreamBeginCapture(cap, cudaStreamCaptureModeRelaxed) != cudaSuccess) {
        cudaStreamDestroy(cap);
        return bail(cuda_status(cudaGetLastError(), "cudaStreamBeginCapture"));
    }
    st = enqueue_batch(b, cap);
    const cudaError_t ce = cudaStreamEndCapture(cap, &b->graph);
    cudaStreamDestroy(cap);
    if (st != CTB_OK) return bail(st);
    if (ce != cudaSuccess) return bail(cuda_status(ce, "cudaStreamEndCapture"));
    st = cuda_status(cudaGraphInstantiate(&b->exec, b->graph, 0), "cudaGraphInstantiate");
    if (st != CTB_OK) return bail(st);
    *out = b;
    return CTB_OK;
}

int ctb_batch_run(ctb_batch* b, void* stream) {
    if (!b || !b->exec) return ctb::fail("ctb_batch_run: invalid batch", CTB_ERR_ARG);
    return ctb::cuda_status(cudaGraphLaunch(b->exec, static_cast<cudaStream_t>(stream)), "cudaGraphLaunch");
}

int ctb_batch_run_sequential(ctb_batch* b, void* stream) {
    using namespace ctb;
    if (!b) return fail("ctb_batch_run_sequential: invalid batch", CTB_ERR_ARG);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    for (size_t i = 0; i < b->scans.size(); ++i) {
        const ctb_scan& sc = b->scans[i];
        const float scale = b->store == CTB_FP32 ? 1.0f : 1.0f / float(sc.det.width);
        FilterArgs a = filter_args(sc.det, sc.raw_type, b->tables[i].M, b->tables[i].logM, sc.n_views, scale);
        a.out_pitch = b->pitch[i];
        int st = filter_launch(sc.raw, sc.raw_type, b->filtered[i], b->store, a, b->tables[i].tw, b->tables[i].K, s);
        if (st != CTB_OK) return st;
        st = backproject_launch(b->filtered[i], b->store, b->views[i], sc.n_views, b->bp[i].g, b->bp[i].hmax,
                                sc.vol, 0, s);
        if (st != CTB_OK) return st;
    }
    return CTB_OK;
}

int ctb_batch_tuning(const ctb_batch* b, int* zc, double* ms32, double* ms16, double* ms8, int* n_persistent) {
    if (!b) return ctb::fail("ctb_batch_tuning: invalid batch", CTB_ERR_ARG);
    if (zc) *zc = b->zc;
    if (ms32) *ms32 = b->ms32;
    if (ms16) *ms16 = b->ms16;
    if (ms8) *ms8 = b->ms8;
    if (n_persistent) *n_persistent = int(b->plan.included.size());
    return CTB_OK;
}

int ctb_batch_tuning_detail(const ctb_batch* b, int max, int* zc, int* views_in_flight, double* ms, int* n) {
    if (!b || !n) return ctb::fail("ctb_batch_tuning_detail: invalid arguments", CTB_ERR_ARG);
    const int k = int(b->cand_ms.size());
    *n = k;
    for (int i = 0; i < k && i < max; ++i) {
        if (zc) zc[i] = b->cand_zc[i];
        if (views_in_flight) views_in_flight[i] = b->cand_nbuf[i];
        if (ms) ms[i] = b->cand_ms[i];
    }
    return CTB_OK;
}

void ctb_batch_destroy(ctb_batch* b) { delete b; }

}  // extern "C"
