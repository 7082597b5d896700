// The context's matched projector pair: A (forward projection, fp_kernel) and
// its exact transpose A^T (the backprojector with load scale 1), applied to
// host volumes and projections on the context's scan geometry and box, and
// the gradient of the least-squares data term f(x) = ||A x - p||^2,
// 2 A^T (A x - p). No counterpart in the reference, which has no forward
// model. The volume moves through the device one z-slab at a time and A x is
// accumulated slab by slab: no intermediate volume is stored, the adjoint
// recomputes per slab what it needs.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "../ctb_internal.h"
#include "reconstructor.h"

namespace ctb {

// A failed CUDA call ends the operation with CTB_ERR_CUDA and its message on
// the context (ctb_last_error), as the facade's other operations do.
#define OP_TRY(expr)                                                                              \
    do {                                                                                          \
        const cudaError_t _e = (expr);                                                            \
        if (_e != cudaSuccess) {                                                                  \
            cudaGetLastError();                                                                   \
            return fail(CTB_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(_e));     \
        }                                                                                         \
    } while (0)

namespace {
constexpr size_t kSlabBytes = size_t(512) << 20;   // device slab buffer (volume slices)

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int d) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        cudaSetDevice(d);
    }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};
}  // namespace

// A bounded wait in a backprojection kernel gave up: the result is incomplete.
static int wait_status(const std::string& what) {
    unsigned gave_up = 0;
    if (device_wait_timeouts(&gave_up, 1) == CTB_OK && gave_up) {
        set_global_error("A device wait of the backprojection gave up (" + std::to_string(gave_up) + " times); " +
                         what + " is incomplete.");
        return CTB_ERR_TIMEOUT;
    }
    return CTB_OK;
}

OpWork::~OpWork() {
    if (device >= 0) {
        DeviceGuard g(device);
        if (s) cudaStreamDestroy(s);
        d_proj.release();
        d_data.release();
        d_slab.release();
        d_views.release();
        d_angles.release();
        d_heights.release();
        d_sum.release();
    }
}

// Buffers, stream and view table on the first active device; the slab height
// that fits the slab buffer.
int Reconstructor::op_prepare(int* slab) {
    if (!have_scan_) return fail(CTB_ERR_ARG, "No projections are loaded.");
    const int dev = devices_.empty() ? 0 : devices_[0];
    if (!op_ || op_->device != dev) op_.reset(new OpWork(dev));
    OpWork& w = *op_;
    OP_TRY(cudaSetDevice(dev));
    if (!w.s && cudaStreamCreateWithFlags(&w.s, cudaStreamNonBlocking) != cudaSuccess)
        return fail(CTB_ERR_CUDA, "stream creation failed");
    const int V = int(angles_.size());
    const int X = grid_.x_to - grid_.x_from, Y = grid_.y_to - grid_.y_from, Z = grid_.z_to - grid_.z_from;
    if (X <= 0 || Y <= 0 || Z <= 0) return fail(CTB_ERR_ARG, "The reconstructed box is empty.");
    const size_t plane = size_t(X) * Y * sizeof(float);
    *slab = int(std::max<size_t>(1, std::min<size_t>(size_t(Z), kSlabBytes / plane)));
    int st;
    if ((st = w.d_proj.ensure(sizeof(float) * size_t(V) * det_.height * det_.width, "projections")) ||
        (st = w.d_slab.ensure(plane * size_t(*slab), "volume slab")) ||
        (st = w.d_views.ensure(sizeof(float4) * V, "view table")) ||
        (st = w.d_angles.ensure(sizeof(double) * V, "angles")) ||
        (st = w.d_heights.ensure(sizeof(double) * V, "height offsets")) ||
        (st = w.d_sum.ensure(sizeof(double), "sum")))
        return fail(st, global_error());
    OP_TRY(cudaMemcpyAsync(w.d_angles.p, angles_.data(), sizeof(double) * V, cudaMemcpyHostToDevice, w.s));
    OP_TRY(cudaMemcpyAsync(w.d_heights.p, heights_px_.data(), sizeof(double) * V, cudaMemcpyHostToDevice, w.s));
    st = view_table_build(static_cast<const double*>(w.d_angles.p), static_cast<const double*>(w.d_heights.p), V,
                          static_cast<float4*>(w.d_views.p), w.s);
    return st == CTB_OK ? CTB_OK : fail(st, global_error());
}

// A x into op_->d_proj (overwritten), x from host memory slab by slab.
int Reconstructor::op_forward(const float* host_vol, int slab) {
    OpWork& w = *op_;
    const int V = int(angles_.size());
    const int X = grid_.x_to - grid_.x_from, Y = grid_.y_to - grid_.y_from, Z = grid_.z_to - grid_.z_from;
    const size_t plane = size_t(X) * Y;
    float* proj = static_cast<float*>(w.d_proj.p);
    float* dslab = static_cast<float*>(w.d_slab.p);
    OP_TRY(cudaMemsetAsync(proj, 0, sizeof(float) * size_t(V) * det_.height * det_.width, w.s));
    for (int z0 = 0; z0 < Z; z0 += slab) {
        if (stop_) return fail(CTB_INTERRUPTED, "User interrupted. Stopping.");
        const int z1 = std::min(Z, z0 + slab);
        OP_TRY(cudaMemcpyAsync(dslab, host_vol + plane * z0, sizeof(float) * plane * (z1 - z0),
                                     cudaMemcpyHostToDevice, w.s));
        const ProjGeom g = proj_geom(det_, grid_, z0, z1, 1.0f);
        const int st = forward_launch(dslab, static_cast<const float4*>(w.d_views.p), V, g, proj, 1, w.s);
        if (st != CTB_OK) return fail(st, global_error());
        // the slab buffer is reused by the next slab's copy (same stream: ordered)
    }
    return CTB_OK;
}

// scale * A^T of the device projections into host memory, slab by slab.
int Reconstructor::op_backward(const float* d_proj, float* host_vol, float scale, int slab) {
    OpWork& w = *op_;
    const int V = int(angles_.size());
    const int X = grid_.x_to - grid_.x_from, Y = grid_.y_to - grid_.y_from, Z = grid_.z_to - grid_.z_from;
    const size_t plane = size_t(X) * Y;
    float* dslab = static_cast<float*>(w.d_slab.p);
    double hmax = 0;
    for (double h : heights_px_) hmax = std::max(hmax, std::fabs(h));
    for (int z0 = 0; z0 < Z; z0 += slab) {
        if (stop_) return fail(CTB_INTERRUPTED, "User interrupted. Stopping.");
        const int z1 = std::min(Z, z0 + slab);
        const ProjGeom g = proj_geom(det_, grid_, z0, z1, scale);
        const int st = backproject_launch(d_proj, CTB_FP32, static_cast<const float4*>(w.d_views.p), V, g, hmax,
                                          dslab, 0, w.s);
        if (st != CTB_OK) return fail(st, global_error());
        OP_TRY(cudaMemcpyAsync(host_vol + plane * z0, dslab, sizeof(float) * plane * (z1 - z0),
                                     cudaMemcpyDeviceToHost, w.s));
        OP_TRY(cudaStreamSynchronize(w.s));
    }
    return CTB_OK;
}

int Reconstructor::forward(const float* host_vol, float* host_proj) {
    std::lock_guard<std::mutex> lk(mtx_);
    stop_ = false;
    if (!host_vol || !host_proj) return fail(CTB_ERR_ARG, "null pointer");
    DeviceGuard guard(devices_.empty() ? 0 : devices_[0]);
    int slab = 0, st;
    if ((st = op_prepare(&slab)) != CTB_OK) return st;
    if ((st = op_forward(host_vol, slab)) != CTB_OK) return st;
    const size_t n = size_t(angles_.size()) * det_.height * det_.width;
    OP_TRY(cudaMemcpyAsync(host_proj, op_->d_proj.p, sizeof(float) * n, cudaMemcpyDeviceToHost, op_->s));
    OP_TRY(cudaStreamSynchronize(op_->s));
    return CTB_OK;
}

int Reconstructor::backward(const float* host_proj, float* host_vol) {
    std::lock_guard<std::mutex> lk(mtx_);
    stop_ = false;
    if (!host_vol || !host_proj) return fail(CTB_ERR_ARG, "null pointer");
    DeviceGuard guard(devices_.empty() ? 0 : devices_[0]);
    int slab = 0, st;
    if ((st = op_prepare(&slab)) != CTB_OK) return st;
    const size_t n = size_t(angles_.size()) * det_.height * det_.width;
    OP_TRY(cudaMemcpyAsync(op_->d_proj.p, host_proj, sizeof(float) * n, cudaMemcpyHostToDevice, op_->s));
    if ((st = op_backward(static_cast<const float*>(op_->d_proj.p), host_vol, 1.0f, slab)) != CTB_OK) return st;
    if ((st = wait_status("the volume")) != CTB_OK) return fail(st, global_error());
    return CTB_OK;
}

int Reconstructor::gradient(const float* host_vol, const float* host_data, float* host_grad, double* f) {
    std::lock_guard<std::mutex> lk(mtx_);
    stop_ = false;
    if (!host_vol || !host_data || !host_grad) return fail(CTB_ERR_ARG, "null pointer");
    DeviceGuard guard(devices_.empty() ? 0 : devices_[0]);
    int slab = 0, st;
    if ((st = op_prepare(&slab)) != CTB_OK) return st;
    OpWork& w = *op_;
    const size_t n = size_t(angles_.size()) * det_.height * det_.width;
    if ((st = w.d_data.ensure(sizeof(float) * n, "measured projections")) != CTB_OK) return fail(st, global_error());
    if ((st = op_forward(host_vol, slab)) != CTB_OK) return st;
    OP_TRY(cudaMemcpyAsync(w.d_data.p, host_data, sizeof(float) * n, cudaMemcpyHostToDevice, w.s));
    OP_TRY(cudaMemsetAsync(w.d_sum.p, 0, sizeof(double), w.s));
    float* r = static_cast<float*>(w.d_proj.p);
    if ((st = residual_launch(r, static_cast<const float*>(w.d_data.p), r, (long long)n,
                              static_cast<double*>(w.d_sum.p), w.s)) != CTB_OK)
        return fail(st, global_error());
    double sumsq = 0;
    OP_TRY(cudaMemcpyAsync(&sumsq, w.d_sum.p, sizeof(double), cudaMemcpyDeviceToHost, w.s));
    // the backprojector's load scale of 2 gives 2 A^T r exactly (a power of two)
    if ((st = op_backward(r, host_grad, 2.0f, slab)) != CTB_OK) return st;
    if (f) *f = sumsq;
    if ((st = wait_status("the gradient")) != CTB_OK) return fail(st, global_error());
    return CTB_OK;
}

}  // namespace ctb
