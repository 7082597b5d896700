// Reconstruction facade: the B200 counterpart of ct::CtVolume
// (Ct/CtVolume.h:57-278). One context drives one or more devices; each active
// device reconstructs its own run of z slices from all views, as the
// reference's launchCudaThreads does (Ct/CtVolume.cpp:1322-1351).
#pragma once

#include <atomic>
#include <cstdint>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../ctb_internal.h"

namespace ctb {

// Device buffer that only grows (reused across reconstructions).
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    int ensure(size_t n, const char* what);
    void release();
    ~DevBuf() { release(); }
};

// Cross section of an X-fastest X x Y x Z volume in the left-handed
// orientation (Common/Volume.h:577-648); out == nullptr only reports the size.
int cross_section_of(const float* vol, int X, int Y, int Z, int axis, int index, float* out, int* rows, int* cols);

// Page-locked host buffer.
struct HostBuf {
    void* p = nullptr;
    size_t bytes = 0;
    bool pinned = false;
    int ensure(size_t n);
    void release();
    ~HostBuf() { release(); }
};

// Per-device resources of one reconstruction worker (one host thread per
// active device). Buffers only grow and are reused across reconstructions.
struct DeviceWork {
    int device = 0;
    // uploads, backprojection (and layout), downloads; filtering on s_filt at the
    // greatest stream priority, beside the early slabs' backprojection
    cudaStream_t s_copy = nullptr, s_comp = nullptr, s_down = nullptr, s_filt = nullptr;
    DevBuf d_filtered, d_ring, d_views, d_angles, d_heights, d_tw, d_K, d_slab[3], d_conv[3];
    HostBuf h_stage[2];
    int tables_key[3] = {-1, -1, -1};  // W, pad, filter of the cached tables
    // outcome of the last run
    std::string err;
    double filter_s = 0, backproject_s = 0, upload_s = 0, download_s = 0;
    double h2d_bytes = 0, d2h_bytes = 0;
    double progress = 0;  // 0..1 of this worker's slices
    double share = 1;     // this worker's fraction of all slices
    explicit DeviceWork(int d) : device(d) {}
    ~DeviceWork();
};

// getGpuWeights (Ct/CtVolume.cpp:1353-1381): per device
// (sm_i / sum sm)^mp_coef * (bw_i / sum bw)^bw_coef, normalised to sum 1.
void gpu_weights_from(const int* sm_count, const double* bandwidth, int n, double mp_coef, double bw_coef,
                      double* weights);
// Consecutive z ranges [begin[i], begin[i+1]) of round(weight_i * z) slices
// (launchCudaThreads, Ct/CtVolume.cpp:1339-1344), clamped to z; the last
// device also takes what rounding left over, so every slice is covered once.
void split_slices(const double* weights, int n, int z, int* begin);

// Device resources of the context's operator calls (forward, backward,
// gradient) on its first active device.
struct OpWork {
    int device = -1;
    cudaStream_t s = nullptr;
    DevBuf d_proj, d_data, d_slab, d_views, d_angles, d_heights, d_sum;
    explicit OpWork(int d) : device(d) {}
    ~OpWork();
};

class Reconstructor {
   public:
    Reconstructor();
    ~Reconstructor();

    // ---- input (sinogramFromImages and its in-memory equivalent)
    int load_csv(const std::string& csv_path);
    int set_projections(const void* images, int raw_type, int n_views, int width, int height,
                        const double* angles_deg, const double* heights_mm, double pixel_size, int ccw,
                        double u_offset_mm, double fcd_mm, double base_intensity);

    // ---- settings
    int set_bounds(float xF, float xT, float yF, float yT, float zF, float zT);
    int set_filter(int f);
    int set_skip(unsigned skip) { step_ = int(skip) + 1; return CTB_OK; }
    int set_device(int d);
    int set_devices(const int* ids, int n);
    int set_gpu_coefficients(double mp, double bw) { mp_coef_ = mp; bw_coef_ = bw; return CTB_OK; }
    int gpu_weights(const int* ids, int n, double* weights);
    int set_spare_mb(size_t mb) { spare_mb_ = mb; return CTB_OK; }
    int set_precision(int t);
    int set_pad(int p);
    int set_grid(int x, int y, int z, float vs);
    int set_slab(int s) { slab_req_ = s; return CTB_OK; }
    void set_progress(ctb_progress_cb cb, void* user) { cb_ = cb; cb_user_ = user; }
    void set_preview(ctb_preview_cb cb, void* user) { preview_ = cb; preview_user_ = user; }
    int set_cross_section_axis(int axis);
    int set_cross_section_index(int index);
    int cross_section_axis() const { return cs_axis_; }
    int cross_section_index() const { return cs_index_; }
    int cross_section_size() const;
    // setEmitSignals / setUseCuda / setUseCpuPreprocessing (Ct/CtVolume.h:99-110)
    void set_emit_signals(bool v) { emit_ = v; }
    int set_use_cuda(bool v);
    void set_use_cpu_preprocessing(bool v) { cpu_pre_ = v; }

    // ---- getters
    const ctb_detector& detector() const { return det_; }
    const ctb_grid& grid() const { return grid_; }
    int views() const { return int(angles_.size()); }
    double pixel_size() const { return pixel_size_; }
    const ctb_timings& timings() const { return tm_; }
    int precision() const { return store_; }
    void settings(ctb_settings* s) const;
    size_t required_memory() const;
    // getProjectionAt: angle, relative height offset (pixels) and, if image is
    // given, the raw image as float normalised by the scan's min / max
    int projection(int index, float* image, double* angle_deg, double* height_px);

    // ---- work
    int reconstruct(float* host_out, int index_order);   // host_out == nullptr: keep internally
    int get_volume(float* host_out, int index_order) const;
    int cross_section(int axis, int index, float* out, int* rows, int* cols) const;
    int save(const std::string& path, int index_order, int byte_order);
    void stop() { stop_ = true; }

    // ---- autotuner of the backprojection launch shape and slab height
    // (host/tuning.cpp): tunes on the context's scan, remembered per shape
    void set_autotune(bool on) { autotune_on_ = on; }
    int autotune(ctb_tuning* out);
    int tuning(ctb_tuning* out) const;

    // ---- matched projector pair on the context's scan geometry and box
    // (host X-fastest volume, host V x H x W float projections; slab by slab)
    int forward(const float* host_vol, float* host_proj);
    int backward(const float* host_proj, float* host_vol);
    // f = ||A x - p||^2 and its gradient 2 A^T (A x - p)
    int gradient(const float* host_vol, const float* host_data, float* host_grad, double* f);

    const std::string& error() const { return err_; }

   private:
    int fail(int status, const std::string& msg);
    int assign_scan(const void* images, int raw_type, int n_views, int width, int height,
                    const double* angles_deg, const double* heights_mm, double pixel_size, int ccw,
                    double u_offset_mm, double fcd_mm, double base_intensity);
    void update_grid();
    int run_pipeline(DeviceWork& w, float* host_out, int index_order, int z_lo, int z_hi);
    void progress(int stage, double pct) { if (cb_ && emit_) cb_(stage, pct, cb_user_); }
    bool previews() const { return preview_ && emit_; }
    void worker_progress(DeviceWork& w, double frac, const float* preview_vol = nullptr);
    void emit_preview(const float* vol, double pct);
    int box_extent(int axis) const;

    std::mutex mtx_;                 // exclusiveFunctionsMutex (Ct/CtVolume.h:258)
    std::atomic<bool> stop_{false};  // stopActiveProcess (:245)
    std::string err_;

    // scan (reference members :225-232)
    ctb_detector det_{};
    double pixel_size_ = 0;          // stored as float by the reference
    int raw_type_ = 0;
    std::vector<double> angles_;     // degrees, direction-corrected
    std::vector<double> heights_px_; // relative, in pixels
    HostBuf images_owned_;           // decoded CSV images
    const void* images_ = nullptr;   // V x H x W raw samples (owned or caller's)
    bool have_scan_ = false;

    // settings
    int filter_ = CTB_RAMLAK;
    int step_ = 1;
    std::vector<int> devices_{0};    // activeCudaDevices (:241)
    double mp_coef_ = 1, bw_coef_ = 1;  // multiprocessor / memoryBandwidth coefficients (:243)
    size_t spare_mb_ = 200;
    int store_ = CTB_FP32;
    int pad_ = 1;
    int grid_x_ = 0, grid_y_ = 0, grid_z_ = 0;
    float grid_vs_ = 1.0f;
    int slab_req_ = 0;
    float rel_[6] = {0, 1, 0, 1, 0, 1};
    ctb_progress_cb cb_ = nullptr;
    void* cb_user_ = nullptr;
    ctb_preview_cb preview_ = nullptr;
    void* preview_user_ = nullptr;
    std::vector<float> preview_buf_;
    int cs_axis_ = CTB_AXIS_Z;       // crossSectionAxis (:239)
    int cs_index_ = 0;               // crossSectionIndex (:238)
    bool emit_ = true;               // emitSignals: progress / preview callbacks
    bool cpu_pre_ = false;           // useCpuPreprocessing (accepted, no effect)
    bool have_minmax_ = false;       // minMaxValues (:292), computed on first use
    float min_max_[2] = {0, 0};

    // geometry (updateBoundaries)
    ctb_grid grid_{};

    // result: X-fastest box volume in host memory
    HostBuf volume_;
    int vol_dims_[3] = {0, 0, 0};
    ctb_timings tm_{};

    // cached per-device resources, one entry per active device
    std::vector<std::unique_ptr<DeviceWork>> workers_;
    std::unique_ptr<OpWork> op_;
    bool autotune_on_ = false;
    int autotune_locked(ctb_tuning* out);
    std::string tune_key(int z_lo, int z_hi) const;
    bool tuned_for(int z_lo, int z_hi, BpConfig* cfg, int* slab) const;
    int op_prepare(int* slab);
    int op_forward(const float* host_vol, int slab);
    int op_backward(const float* d_proj, float* host_vol, float scale, int slab);
    std::mutex progress_mtx_;
};

}  // namespace ctb
