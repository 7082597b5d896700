// Reconstruction facade implementation (ct::CtVolume counterpart).
//
// Pipeline of one reconstruction on one B200 (all views' filtered projections
// stay resident in HBM; the volume streams out in z-slabs):
//   copy stream    : H2D of the detector rows this device's slices reach, in
//                    chunks of views, into a 3-slot ring of device buffers
//   compute stream : fused preprocess + ramp filter of each chunk (kernel a+b)
//                    into the resident filtered set (FP32/FP16/BF16); the
//                    first two slabs are backprojected every two chunks while
//                    the views arrive, every later slab in one launch over all
//                    views (kernel c); then the output layout kernel
//   download stream: D2H of each finished slab while the next slab computes
//                    (three slab buffers; a short last slab)
// The reference instead re-reads and re-filters every projection for every
// VRAM-sized chunk and launches one kernel per view (Ct/CtVolume.cpp:1155-1301).

#include "reconstructor.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <atomic>
#include <fstream>
#include <sstream>
#include <thread>

#include "image_io.h"

namespace ctb {

// ------------------------------------------------------------------ buffers
// Diagnostic allocation failure (ctb_diag_fail_allocation): while positive,
// every device or host allocation of the facade counts it down and the one
// that brings it to zero fails as if the memory were exhausted.
static std::atomic<long> g_fail_countdown{0};

void fail_allocation_after(long n) { g_fail_countdown.store(n > 0 ? n : 0); }

static bool injected_failure() {
    long c = g_fail_countdown.load();
    while (c > 0)
        if (g_fail_countdown.compare_exchange_weak(c, c - 1)) return c == 1;
    return false;
}

int DevBuf::ensure(size_t n, const char* what) {
    if (n <= bytes && p) return CTB_OK;
    release();
    if (n == 0) return CTB_OK;
    if (injected_failure()) {
        set_global_error(std::string("device allocation of ") + std::to_string(n >> 20) + " MB for " + what +
                         " failed (injected)");
        return CTB_ERR_ALLOC;
    }
    cudaError_t e = cudaMalloc(&p, n);
    if (e != cudaSuccess) {
        p = nullptr;
        cudaGetLastError();
        set_global_error(std::string("device allocation of ") + std::to_string(n >> 20) + " MB for " + what +
                         " failed: " + cudaGetErrorString(e));
        return CTB_ERR_ALLOC;
    }
    bytes = n;
    return CTB_OK;
}
void DevBuf::release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
}

int HostBuf::ensure(size_t n) {
    if (n <= bytes && p) return CTB_OK;
    release();
    if (n == 0) return CTB_OK;
    if (injected_failure()) return CTB_ERR_ALLOC;
    if (cudaHostAlloc(&p, n, cudaHostAllocPortable) == cudaSuccess) {
        pinned = true;
    } else {
        cudaGetLastError();
        p = std::malloc(n);
        pinned = false;
        if (!p) return CTB_ERR_ALLOC;
    }
    bytes = n;
    return CTB_OK;
}
void HostBuf::release() {
    if (p) {
        if (pinned) cudaFreeHost(p);
        else std::free(p);
    }
    p = nullptr;
    bytes = 0;
    pinned = false;
}

namespace {

bool is_pinned(const void* p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

// Multi-threaded host loop over [0, n).
template <typename F>
void parallel_for(size_t n, F&& f) {
    const size_t T = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    if (n < 2 * T) {
        for (size_t i = 0; i < n; ++i) f(i);
        return;
    }
    std::vector<std::thread> th;
    for (size_t t = 0; t < T; ++t)
        th.emplace_back([&, t] {
            for (size_t i = t * n / T; i < (t + 1) * n / T; ++i) f(i);
        });
    for (auto& x : th) x.join();
}

// QString::toDouble semantics: the whole field must be a number (surrounding
// whitespace allowed).
bool to_double(const std::string& s, double* out) {
    const char* b = s.c_str();
    char* e = nullptr;
    *out = std::strtod(b, &e);
    if (e == b) return false;
    while (*e == ' ' || *e == '\t' || *e == '\r' || *e == '\n') ++e;
    return *e == '\0';
}

std::string first_field(const std::string& line) { return line.substr(0, line.find('\t')); }

std::vector<std::string> split_tabs(const std::string& line) {
    std::vector<std::string> f;
    size_t a = 0;
    while (true) {
        size_t b = line.find('\t', a);
        f.push_back(line.substr(a, b == std::string::npos ? std::string::npos : b - a));
        if (b == std::string::npos) break;
        a = b + 1;
    }
    return f;
}

std::string dirname_of(const std::string& p) {
    size_t k = p.find_last_of('/');
    return k == std::string::npos ? std::string(".") : p.substr(0, k);
}

std::string join_path(const std::string& dir, const std::string& name) {
    if (!name.empty() && name[0] == '/') return name;
    if (dir.empty()) return name;
    return dir.back() == '/' ? dir + name : dir + "/" + name;
}

unsigned cylinder_radius(int W, float FCD) {
    // getReconstructionCylinderRadius (Ct/CtVolume.cpp:370-373)
    double radius = unsigned(W) / 2;
    return unsigned(std::sqrt((double(FCD) * FCD * radius * radius) / (double(FCD) * FCD + radius * radius)));
}

}  // namespace

DeviceWork::~DeviceWork() {
    // device buffers belong to this worker's device
    cudaSetDevice(device);
    if (s_copy) {
        cudaStreamDestroy(s_copy);
        cudaStreamDestroy(s_comp);
        cudaStreamDestroy(s_down);
        cudaStreamDestroy(s_filt);
    }
    for (DevBuf* b : {&d_filtered, &d_ring, &d_views, &d_angles, &d_heights, &d_tw, &d_K, &d_slab[0], &d_slab[1],
                      &d_slab[2], &d_conv[0], &d_conv[1], &d_conv[2]})
        b->release();
}

void gpu_weights_from(const int* sm_count, const double* bandwidth, int n, double mp_coef, double bw_coef,
                      double* weights) {
    double sm_total = 0, bw_total = 0;
    for (int i = 0; i < n; ++i) { sm_total += sm_count[i]; bw_total += bandwidth[i]; }
    double sum = 0;
    for (int i = 0; i < n; ++i) {
        weights[i] = std::pow(double(sm_count[i]) / sm_total, mp_coef) * std::pow(bandwidth[i] / bw_total, bw_coef);
        sum += weights[i];
    }
    for (int i = 0; i < n; ++i) weights[i] /= sum;
}

void split_slices(const double* weights, int n, int z, int* begin) {
    int cur = 0;
    for (int i = 0; i < n; ++i) {
        begin[i] = cur;
        cur = std::min(z, cur + int(std::lround(weights[i] * double(z))));
    }
    begin[n] = z;
}

Reconstructor::Reconstructor() {}

Reconstructor::~Reconstructor() {}

int Reconstructor::fail(int status, const std::string& msg) {
    err_ = msg;
    set_global_error(msg);
    return status;
}

// updateBoundaries (Ct/CtVolume.cpp:1399-1424) on the reference grid rule
// (:311-316) or on the overriding grid.
void Reconstructor::update_grid() {
    const unsigned radius = cylinder_radius(det_.width, det_.fcd);
    det_.radius = float(radius);
    ctb_grid g{};
    if (grid_x_ > 0) {
        g.x_size = grid_x_; g.y_size = grid_y_; g.z_size = grid_z_;
        g.voxel_pitch = grid_vs_;
    } else {
        g.x_size = int(radius * 2); g.y_size = int(radius * 2); g.z_size = det_.height;
        g.voxel_pitch = 1.0f;
    }
    g.x_from = int(unsigned(rel_[0] * g.x_size + 0.5)); g.x_to = int(unsigned(rel_[1] * g.x_size + 0.5));
    g.y_from = int(unsigned(rel_[2] * g.y_size + 0.5)); g.y_to = int(unsigned(rel_[3] * g.y_size + 0.5));
    g.z_from = int(unsigned(rel_[4] * g.z_size + 0.5)); g.z_to = int(unsigned(rel_[5] * g.z_size + 0.5));
    grid_ = g;
    // keep the cross-section index inside the box (:1411-1417)
    const int ext = box_extent(cs_axis_);
    if (cs_index_ >= ext) cs_index_ = ext / 2;
}

int Reconstructor::box_extent(int axis) const {
    if (axis == CTB_AXIS_X) return grid_.x_to - grid_.x_from;
    if (axis == CTB_AXIS_Y) return grid_.y_to - grid_.y_from;
    return grid_.z_to - grid_.z_from;
}

int Reconstructor::cross_section_size() const { return std::max(0, box_extent(cs_axis_)); }

// setCrossSectionAxis (:401-410): the index moves to the middle of the axis.
int Reconstructor::set_cross_section_axis(int axis) {
    if (axis < CTB_AXIS_X || axis > CTB_AXIS_Z) return fail(CTB_ERR_ARG, "unknown axis");
    cs_axis_ = axis;
    cs_index_ = std::max(0, box_extent(axis)) / 2;
    return CTB_OK;
}

// setCrossSectionIndex (:395-399): ignored unless inside the box.
int Reconstructor::set_cross_section_index(int index) {
    if (index >= 0 && index < box_extent(cs_axis_)) cs_index_ = index;
    return CTB_OK;
}

// reconstructionProgress / reconstructionFinished with the cross section of
// the volume as it stands (Ct/CtVolume.cpp:952, :1479-1483, :615).
void Reconstructor::emit_preview(const float* vol, double pct) {
    const int X = grid_.x_to - grid_.x_from, Y = grid_.y_to - grid_.y_from, Z = grid_.z_to - grid_.z_from;
    int rows = 0, cols = 0;
    if (cross_section_of(vol, X, Y, Z, cs_axis_, cs_index_, nullptr, &rows, &cols) != CTB_OK) return;
    preview_buf_.resize(size_t(rows) * cols);
    cross_section_of(vol, X, Y, Z, cs_axis_, cs_index_, preview_buf_.data(), nullptr, nullptr);
    preview_(pct, preview_buf_.data(), rows, cols, preview_user_);
}

// setVolumeBounds (Ct/CtVolume.cpp:487-500), including the reference's clamp
// of the y/z upper bounds against xFrom.
int Reconstructor::set_bounds(float xF, float xT, float yF, float yT, float zF, float zT) {
    std::lock_guard<std::mutex> lk(mtx_);
    if (xF == xT || yF == yT || zF == zT)
        return fail(CTB_ERR_ARG, "ERROR: the lower and upper bounds must not be identical.");
    rel_[0] = std::max(0.0f, std::min(1.0f, xF));
    rel_[1] = std::max(rel_[0], std::min(1.0f, xT));
    rel_[2] = std::max(0.0f, std::min(1.0f, yF));
    rel_[3] = std::max(rel_[0], std::min(1.0f, yT));
    rel_[4] = std::max(0.0f, std::min(1.0f, zF));
    rel_[5] = std::max(rel_[0], std::min(1.0f, zT));
    if (have_scan_) update_grid();
    return CTB_OK;
}

int Reconstructor::set_filter(int f) {
    if (f < CTB_RAMLAK || f > CTB_HANN) return fail(CTB_ERR_ARG, "unknown filter type");
    filter_ = f;
    return CTB_OK;
}

// setUseCuda (:502-504): the reconstruction runs on the GPU only.
int Reconstructor::set_use_cuda(bool v) {
    if (!v) return fail(CTB_ERR_UNSUPPORTED, "CPU reconstruction is not part of this engine; it reconstructs on the GPU.");
    return CTB_OK;
}

void Reconstructor::settings(ctb_settings* s) const {
    *s = ctb_settings{};
    s->skip_projections = unsigned(std::max(1, step_) - 1);  // getSkipProjections (:438-440)
    s->use_cuda = 1;
    s->use_cpu_preprocessing = cpu_pre_ ? 1 : 0;
    s->emit_signals = emit_ ? 1 : 0;
    s->gpu_spare_memory_mb = spare_mb_;
    s->multiprocessor_coefficient = mp_coef_;
    s->memory_bandwidth_coefficient = bw_coef_;
    s->n_devices = int(std::min<size_t>(devices_.size(), 16));
    for (int i = 0; i < s->n_devices; ++i) s->devices[i] = devices_[i];
}

// getRequiredMemoryUpperBound (:469-481), CUDA branch: the float volume plus
// three float images per active device.
size_t Reconstructor::required_memory() const {
    const size_t X = size_t(std::max(0, grid_.x_to - grid_.x_from));
    const size_t Y = size_t(std::max(0, grid_.y_to - grid_.y_from));
    const size_t Z = size_t(std::max(0, grid_.z_to - grid_.z_from));
    return X * Y * Z * sizeof(float) +
           size_t(det_.width) * size_t(det_.height) * sizeof(float) * devices_.size() * 3;
}

// getProjectionAt (:332-341): the image converted to float as convertTo32bit
// does (:802-812) and normalised by the scan's minimum and maximum, which the
// reference gathers while loading (:270-292): raw extremes divided by 2^8 for
// 8-bit images and by 2^16 otherwise.
int Reconstructor::projection(int index, float* image, double* angle_deg, double* height_px) {
    if (!have_scan_ || index < 0 || index >= int(angles_.size())) return fail(CTB_ERR_ARG, "Index out of bounds.");
    if (angle_deg) *angle_deg = angles_[index];
    if (height_px) *height_px = heights_px_[index];
    if (!image) return CTB_OK;
    const size_t n = size_t(det_.width) * det_.height;
    auto sample = [&](size_t v, size_t i) -> double {
        if (raw_type_ == CTB_U8) return static_cast<const uint8_t*>(images_)[v * n + i];
        if (raw_type_ == CTB_U16) return static_cast<const uint16_t*>(images_)[v * n + i];
        return static_cast<const float*>(images_)[v * n + i];
    };
    if (!have_minmax_) {
        const size_t V = angles_.size();
        std::vector<double> lo(V), hi(V);
        parallel_for(V, [&](size_t v) {
            double a = sample(v, 0), b = a;
            for (size_t i = 1; i < n; ++i) {
                const double x = sample(v, i);
                a = std::min(a, x);
                b = std::max(b, x);
            }
            lo[v] = a;
            hi[v] = b;
        });
        const double scale = raw_type_ == CTB_U8 ? 256.0 : 65536.0;
        min_max_[0] = float(*std::min_element(lo.begin(), lo.end()) / scale);
        min_max_[1] = float(*std::max_element(hi.begin(), hi.end()) / scale);
        have_minmax_ = true;
    }
    const float alpha = float(raw_type_ == CTB_U8 ? 1.0 / 255.0 : 1.0 / 65535.0);
    const float beta = float(0.000001 * double(det_.base_intensity));
    const float lo = min_max_[0], span = min_max_[1] - min_max_[0];
    for (size_t i = 0; i < n; ++i) {
        float p = float(sample(size_t(index), i));
        if (raw_type_ != CTB_F32) {
            const float scaled = p * alpha;  // separate statements: no fused multiply-add
            p = scaled + beta;
        }
        image[i] = (p - lo) / span;
    }
    return CTB_OK;
}

int Reconstructor::set_device(int d) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || d < 0 || d >= n) {
        cudaGetLastError();
        return fail(CTB_ERR_ARG, "Active CUDA device was not set because the device ID is not valid.");
    }
    devices_.assign(1, d);
    return CTB_OK;
}

// setActiveCudaDevices (Ct/CtVolume.cpp:506-520): IDs beyond the device count
// are dropped; with none left the previous selection stays. A device may be
// listed more than once: each entry is its own worker with its own buffers.
int Reconstructor::set_devices(const int* ids, int n) {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess) {
        cudaGetLastError();
        count = 0;
    }
    std::vector<int> keep;
    for (int i = 0; i < n; ++i)
        if (ids[i] >= 0 && ids[i] < count) keep.push_back(ids[i]);
    if (keep.empty())
        return fail(CTB_ERR_ARG, "Active CUDA devices were not set because vector did not contain any valid device ID.");
    devices_ = keep;
    return CTB_OK;
}

int Reconstructor::gpu_weights(const int* ids, int n, double* weights) {
    std::vector<int> sm(n);
    std::vector<double> bw(n);
    for (int i = 0; i < n; ++i) {
        int s = 0, bus = 0, clk = 0;
        if (cudaDeviceGetAttribute(&s, cudaDevAttrMultiProcessorCount, ids[i]) != cudaSuccess ||
            cudaDeviceGetAttribute(&bus, cudaDevAttrGlobalMemoryBusWidth, ids[i]) != cudaSuccess ||
            cudaDeviceGetAttribute(&clk, cudaDevAttrMemoryClockRate, ids[i]) != cudaSuccess) {
            cudaGetLastError();
            return fail(CTB_ERR_ARG, "device properties could not be queried");
        }
        sm[i] = s;
        bw[i] = double(bus) * double(clk);
    }
    gpu_weights_from(sm.data(), bw.data(), n, mp_coef_, bw_coef_, weights);
    return CTB_OK;
}

int Reconstructor::set_precision(int t) {
    if (t != CTB_FP32 && t != CTB_FP16 && t != CTB_BF16) return fail(CTB_ERR_ARG, "unknown storage type");
    store_ = t;
    return CTB_OK;
}

int Reconstructor::set_pad(int p) {
    if (p != 1 && p != 2) return fail(CTB_ERR_ARG, "pad must be 1 or 2");
    pad_ = p;
    return CTB_OK;
}

int Reconstructor::set_grid(int x, int y, int z, float vs) {
    if (x == 0 && y == 0 && z == 0) {
        grid_x_ = grid_y_ = grid_z_ = 0;
        grid_vs_ = 1.0f;
    } else {
        if (x <= 0 || y <= 0 || z <= 0 || !(vs > 0)) return fail(CTB_ERR_ARG, "invalid grid");
        grid_x_ = x; grid_y_ = y; grid_z_ = z; grid_vs_ = vs;
    }
    if (have_scan_) update_grid();
    return CTB_OK;
}

// sinogramFromImages (Ct/CtVolume.cpp:136-330).
int Reconstructor::load_csv(const std::string& csv_path) {
    std::lock_guard<std::mutex> lk(mtx_);
    stop_ = false;
    have_scan_ = false;
    angles_.clear();
    heights_px_.clear();
    std::ifstream in(csv_path);
    if (!in.good()) return fail(CTB_ERR_IO, "Could not open the config file.");
    std::vector<std::string> lines;
    {
        std::string l;
        while (std::getline(in, l)) {
            if (!l.empty() && l.back() == '\r') l.pop_back();
            lines.push_back(l);
        }
    }
    auto line_at = [&](size_t i) { return i < lines.size() ? lines[i] : std::string(); };
    // header :157-168
    std::string image_dir = first_field(line_at(0));
    double pix = 0, uoff = 0, fcd = 0, base = 0;
    bool ok = to_double(first_field(line_at(1)), &pix);
    const std::string rotation = first_field(line_at(2));
    ok = to_double(first_field(line_at(3)), &uoff) && ok;
    ok = to_double(first_field(line_at(4)), &fcd) && ok;
    ok = to_double(first_field(line_at(5)), &base) && ok;
    if (!ok) return fail(CTB_ERR_CSV, "Could not read the parameters from the CSV file successfully.");
    if (float(base) == 0.0f)
        return fail(CTB_ERR_CSV,
                    "Error: The base intensity given in the configuration file must not be equal to zero.");
    // relative image directory is resolved against the CSV's directory (:185-187)
    if (image_dir.empty() || image_dir[0] != '/') image_dir = join_path(dirname_of(csv_path), image_dir);

    // image lines :197-213 (a line with fewer than two fields repeats the
    // previous file name and angle, as in the reference)
    std::vector<std::string> paths;
    std::vector<double> ang, hmm;
    std::string fname;
    double a = 0, h = 0;
    bool all_ok = true;
    for (size_t i = 7; i < lines.size(); ++i) {
        const std::vector<std::string> f = split_tabs(lines[i]);
        if (f.size() >= 2) {
            fname = f[0];
            double v;
            const bool s = to_double(f[1], &v);
            all_ok = all_ok && s;
            a = v;
        }
        if (f.size() >= 3) {
            double v;
            const bool s = to_double(f[2], &v);
            all_ok = all_ok && s;
            h = v;
        } else {
            h = 0;
        }
        paths.push_back(join_path(image_dir, fname));
        ang.push_back(a);
        hmm.push_back(h);
    }
    if (!all_ok) return fail(CTB_ERR_CSV, "Could not read the image parameters from the CSV file successfully.");
    if (paths.empty()) return fail(CTB_ERR_CSV, "Apparently the config file does not contain any images.");

    // probe the first image, then decode all into pinned host memory (:227-292)
    int W = 0, H = 0, type = 0;
    std::string e;
    if (!probe_image(paths[0], &W, &H, &type, &e))
        return fail(CTB_ERR_IMAGE, "Error loading the image \"" + paths[0] +
                                       "\". Maybe it does not exist, permissions are missing or the format is "
                                       "not supported. (" + e + ")");
    const size_t bytes_per = size_t(W) * H * raw_bytes(type);
    if (images_owned_.ensure(bytes_per * paths.size()) != CTB_OK)
        return fail(CTB_ERR_ALLOC, "Host memory for the projections could not be allocated.");
    std::atomic<int> bad{-1};
    std::vector<std::string> errs(paths.size());
    std::atomic<size_t> done{0};
    parallel_for(paths.size(), [&](size_t i) {
        if (bad.load() >= 0 || stop_) return;
        std::string er;
        const int r = load_image_into(paths[i], W, H, type, (char*)images_owned_.p + i * bytes_per, &er);
        if (r == kLoadOtherSize) er = "dims";
        if (r == kLoadOtherDepth) er = "depth";
        if (r != kLoadOk) {
            errs[i] = er;
            int expect = -1;
            bad.compare_exchange_strong(expect, int(i));
        }
        done++;
    });
    if (stop_) return fail(CTB_INTERRUPTED, "User interrupted. Stopping.");
    if (bad.load() >= 0) {
        const size_t i = size_t(bad.load());
        if (errs[i] == "dims")
            return fail(CTB_ERR_IMAGE, "Error loading the image \"" + paths[i] +
                                           "\", its dimensions differ from the images before.");
        if (errs[i] == "depth")
            return fail(CTB_ERR_IMAGE, "Error loading the image \"" + paths[i] +
                                           "\". All images must have the same depth (8bit, 16bit or 32bit).");
        return fail(CTB_ERR_IMAGE, "Error loading the image \"" + paths[i] +
                                       "\". Maybe it does not exist, permissions are missing or the format is "
                                       "not supported. (" + errs[i] + ")");
    }
    progress(0, 100.0);
    images_ = images_owned_.p;
    return assign_scan(images_owned_.p, type, int(paths.size()), W, H, ang.data(), hmm.data(), pix,
                       rotation == "ccw" ? 1 : (rotation == "cw" ? 0 : -1), uoff, fcd, base);
}

int Reconstructor::set_projections(const void* images, int raw_type, int n_views, int width, int height,
                                   const double* angles_deg, const double* heights_mm, double pixel_size,
                                   int ccw, double u_offset_mm, double fcd_mm, double base_intensity) {
    std::lock_guard<std::mutex> lk(mtx_);
    stop_ = false;
    have_scan_ = false;
    return assign_scan(images, raw_type, n_views, width, height, angles_deg, heights_mm, pixel_size, ccw,
                       u_offset_mm, fcd_mm, base_intensity);
}

// Shared tail of the CSV path and the in-memory entry point: FCD/uOffset in
// pixels (:170-172), the W >= FCD check (:294-301), relative height offsets
// (:742-753), direction correction (:755-767) and the grid (:311-316).
// ccw: 1 = "ccw", 0 = "cw", -1 = any other string (no correction).
int Reconstructor::assign_scan(const void* images, int raw_type, int n_views, int width, int height,
                               const double* angles_deg, const double* heights_mm, double pixel_size, int ccw,
                               double u_offset_mm, double fcd_mm, double base_intensity) {
    if (!images || n_views <= 0 || width <= 1 || height <= 1 || !angles_deg)
        return fail(CTB_ERR_ARG, "invalid projection set");
    if (raw_type != CTB_U8 && raw_type != CTB_U16 && raw_type != CTB_F32)
        return fail(CTB_ERR_IMAGE, "The image depth must be either 8bit, 16bit or 32bit.");
    if (float(base_intensity) == 0.0f)
        return fail(CTB_ERR_CSV,
                    "Error: The base intensity given in the configuration file must not be equal to zero.");
    const float pix = float(pixel_size);
    float FCD = float(fcd_mm);
    FCD /= pix;
    float uOffset = float(u_offset_mm);
    uOffset /= pix;
    if (float(width) >= FCD) {
        have_scan_ = false;
        return fail(CTB_ERR_ARG, "Error: the FCD must be greater than the image width.");
    }
    det_.width = width;
    det_.height = height;
    det_.fcd = FCD;
    det_.u_offset = uOffset;
    det_.base_intensity = float(base_intensity);
    pixel_size_ = pix;
    raw_type_ = raw_type;
    images_ = images;
    angles_.assign(angles_deg, angles_deg + n_views);
    heights_px_.assign(n_views, 0.0);
    if (heights_mm) heights_px_.assign(heights_mm, heights_mm + n_views);
    double sum = 0;
    for (double v : heights_px_) sum += v;
    sum /= double(n_views);
    for (double& v : heights_px_) { v -= sum; v /= double(pix); }
    if (n_views > 1 && ccw >= 0) {
        const double diff = angles_[1] - angles_[0];
        if ((ccw == 0 && diff > 0) || (ccw == 1 && diff < 0))
            for (double& v : angles_) v *= -1;
    }
    have_scan_ = true;
    have_minmax_ = false;
    update_grid();
    cs_index_ = std::max(0, box_extent(cs_axis_)) / 2;  // (:317-326)
    return CTB_OK;
}

int Reconstructor::reconstruct(float* host_out, int index_order) {
    std::lock_guard<std::mutex> lk(mtx_);
    stop_ = false;
    if (!have_scan_)
        return fail(CTB_ERR_ARG, "Volume was not reconstructed, because the sinogram seems to be empty. Please "
                                 "load some images first.");
    const int X = grid_.x_to - grid_.x_from, Y = grid_.y_to - grid_.y_from, Z = grid_.z_to - grid_.z_from;
    if (X <= 0 || Y <= 0 || Z <= 0) return fail(CTB_ERR_ARG, "The reconstructed box is empty.");
    const auto t_start = std::chrono::steady_clock::now();
    float* target = host_out;
    if (!target) {
        if (volume_.ensure(sizeof(float) * size_t(X) * Y * Z) != CTB_OK)
            return fail(CTB_ERR_ALLOC,
                        "The memory allocation for the volume failed. Maybe there is not enought free RAM.");
        target = static_cast<float*>(volume_.p);
        index_order = CTB_X_FASTEST;
        if (previews()) {  // previews show the unfinished part as zeros (reinitialise, :555)
            const size_t n = size_t(X) * Y * Z, parts = 16;
            parallel_for(parts, [&](size_t p) {
                std::memset(target + p * n / parts, 0, sizeof(float) * ((p + 1) * n / parts - p * n / parts));
            });
        }
    }

    // the first reconstruction of a shape tunes the backprojection when asked
    // to (single device; a failed tuning leaves the built-in choices)
    if (autotune_on_ && devices_.size() == 1) {
        ctb_tuning t;
        if (autotune_locked(&t) != CTB_OK) err_.clear();
    }

    // one worker per active device entry; workers keep their buffers while
    // the device list stays the same
    const int n = int(devices_.size());
    for (int i = 0; i < n; ++i)
        if (i >= int(workers_.size()) || workers_[i]->device != devices_[i]) {
            if (i < int(workers_.size())) workers_[i].reset(new DeviceWork(devices_[i]));
            else workers_.emplace_back(new DeviceWork(devices_[i]));
        }
    workers_.resize(n);
    std::vector<double> weights(n, 1.0);
    if (n > 1 && gpu_weights(devices_.data(), n, weights.data()) != CTB_OK) return CTB_ERR_ARG;
    std::vector<int> begin(n + 1);
    split_slices(weights.data(), n, Z, begin.data());
    for (int i = 0; i < n; ++i) {
        workers_[i]->progress = 0;
        workers_[i]->share = double(begin[i + 1] - begin[i]) / double(Z);
    }

    std::vector<int> st(n, CTB_OK);
    auto work = [&](int i) {
        st[i] = run_pipeline(*workers_[i], target, index_order, begin[i], begin[i + 1]);
        if (st[i] != CTB_OK && st[i] != CTB_INTERRUPTED) stop_ = true;  // the other workers end early
    };
    if (n == 1) {
        work(0);
    } else {
        std::vector<std::thread> threads;
        for (int i = 0; i < n; ++i) threads.emplace_back(work, i);
        for (auto& t : threads) t.join();
    }
    int status = CTB_OK;
    std::string msg;
    for (int i = 0; i < n; ++i)
        if (st[i] != CTB_OK && (status == CTB_OK || status == CTB_INTERRUPTED)) {
            status = st[i];
            msg = workers_[i]->err;
        }
    if (status != CTB_OK) {
        if (!host_out) vol_dims_[0] = vol_dims_[1] = vol_dims_[2] = 0;  // volume.clear() (:617)
        return fail(status, msg);
    }
    if (!host_out) {
        vol_dims_[0] = X; vol_dims_[1] = Y; vol_dims_[2] = Z;
        if (previews()) emit_preview(target, 100.0);  // reconstructionFinished (:615)
    }

    ctb_timings t{};
    for (auto& w : workers_) {
        t.filter_s = std::max(t.filter_s, w->filter_s);
        t.backproject_s = std::max(t.backproject_s, w->backproject_s);
        t.upload_s = std::max(t.upload_s, w->upload_s);
        t.download_s = std::max(t.download_s, w->download_s);
        t.h2d_bytes += w->h2d_bytes;
        t.d2h_bytes += w->d2h_bytes;
    }
    t.total_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
    const int step = std::max(1, step_);
    t.voxel_views = double(X) * Y * Z * double((int(angles_.size()) + step - 1) / step);
    tm_ = t;
    return CTB_OK;
}

// emitGlobalCudaProgress (Ct/CtVolume.cpp:1469-1485): the total is each
// worker's completion weighted by its share of the slices.
void Reconstructor::worker_progress(DeviceWork& w, double frac, const float* preview_vol) {
    std::lock_guard<std::mutex> lk(progress_mtx_);
    w.progress = frac;
    double total = 0;
    for (auto& o : workers_) total += o->progress * o->share;
    progress(1, 100.0 * total);
    if (previews() && preview_vol) emit_preview(preview_vol, 100.0 * total);
}

// Reconstructs box slices [z_lo, z_hi) on worker w's device into out, which
// holds the whole box in the requested index order (cudaReconstructionCore,
// Ct/CtVolume.cpp:1155-1320, for one device's part of the volume).
void row_band(const ctb_detector& det, const ctb_grid& grid, int z_begin, int z_end, const double* heights_px,
              int n_views, int* r_lo, int* rows) {
    const int H = det.height;
    *r_lo = 0;
    *rows = H;
    if (z_end <= z_begin) return;
    const ProjGeom ga = proj_geom(det, grid, z_begin, z_end, 1.0f);
    double hlo = 0, hhi = 0;
    for (int i = 0; i < n_views && heights_px; ++i) {
        hlo = std::min(hlo, heights_px[i]);
        hhi = std::max(hhi, heights_px[i]);
    }
    const double R = std::sqrt(double(ga.r2)) + 2.0 * double(ga.vs), D = ga.D;
    if (!(R < 0.9 * D)) return;
    // row vi = H/2 - (zw + h) U with zw = (j - zPre) vs, U = D / (D - s), |s| <= R
    const double Umin = D / (D + R), Umax = D / (D - R);
    const double a = (0.0 - double(ga.zPre)) * ga.vs + hlo;
    const double b = (double(z_end - z_begin) - 1.0 - double(ga.zPre)) * ga.vs + hhi;
    const double vmin = std::min(a * Umin, a * Umax), vmax = std::max(b * Umin, b * Umax);
    const int lo = std::max(0, int(std::floor(std::max(-1.0e9, double(H) / 2.0 - vmax))) - 3);
    const int hi = std::min(H - 1, int(std::floor(std::min(1.0e9, double(H) / 2.0 - vmin))) + 4);
    if (hi >= lo) {
        *r_lo = lo;
        *rows = hi - lo + 1;
    }
}

int Reconstructor::run_pipeline(DeviceWork& w, float* out, int order, int z_lo, int z_hi) {
    const auto t_start = std::chrono::steady_clock::now();
    auto fail = [&w](int status, const std::string& msg) {
        w.err = msg;
        return status;
    };
    w.filter_s = w.backproject_s = w.upload_s = w.download_s = 0;
    w.h2d_bytes = w.d2h_bytes = 0;
    if (z_hi <= z_lo) return CTB_OK;
    if (cudaSetDevice(w.device) != cudaSuccess) {
        cudaGetLastError();
        return fail(CTB_ERR_CUDA, "CUDA device could not be selected.");
    }
    if (!w.s_copy) {
        int prio_lo = 0, prio_hi = 0;   // prio_hi: the greatest priority (numerically lowest)
        cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi);
        if (cudaStreamCreateWithFlags(&w.s_copy, cudaStreamNonBlocking) != cudaSuccess ||
            cudaStreamCreateWithFlags(&w.s_comp, cudaStreamNonBlocking) != cudaSuccess ||
            cudaStreamCreateWithFlags(&w.s_down, cudaStreamNonBlocking) != cudaSuccess ||
            cudaStreamCreateWithPriority(&w.s_filt, cudaStreamNonBlocking, prio_hi) != cudaSuccess) {
            cudaGetLastError();
            return fail(CTB_ERR_CUDA, "CUDA streams could not be created.");
        }
    }
    const int W = det_.width, H = det_.height;
    const int X = grid_.x_to - grid_.x_from, Y = grid_.y_to - grid_.y_from, Z = grid_.z_to - grid_.z_from;
    const int Zw = z_hi - z_lo;  // this worker's slices

    // views used (setSkipProjections: projectionStep, :945)
    std::vector<int> used;
    for (int p = 0; p < int(angles_.size()); p += std::max(1, step_)) used.push_back(p);
    const int V = int(used.size());
    std::vector<double> ang(V), hp(V);
    double hmax = 0;
    for (int i = 0; i < V; ++i) {
        ang[i] = angles_[used[i]];
        hp[i] = heights_px_[used[i]];
        hmax = std::max(hmax, std::fabs(hp[i]));
    }

    const int M = filter_transform_length(W, pad_);
    if (M == 0) return fail(CTB_ERR_UNSUPPORTED, "Detector width exceeds the largest supported FFT length.");
    int logM = 0;
    while ((1 << logM) < M) ++logM;

    // storage scale: FP16/BF16 keep values near unit magnitude (x 1/W)
    const float store_scale = store_ == CTB_FP32 ? 1.0f : 1.0f / float(W);
    const float load_scale = store_ == CTB_FP32 ? 1.0f : float(W);

    // ---- detector row band: rows r_lo .. r_lo + Hb - 1 hold every row that
    // this worker's slices reach (every view, every column of the
    // reconstruction cylinder, the height offsets, a margin of a few rows).
    // Only those rows are uploaded, filtered and kept: workers that split z
    // between devices each move a share of the projections, and a z sub-box
    // moves only the rows it needs. Rows are filtered independently, so the
    // filtered values do not change; the backprojector's row coordinates are
    // rounded from the band's first row (differences of a few ulps).
    int r_lo = 0, Hb = H;
    row_band(det_, grid_, z_lo, z_hi, hp.data(), V, &r_lo, &Hb);

    // ---- sizing
    const size_t row_raw = size_t(W) * raw_bytes(raw_type_);
    const size_t view_raw_full = row_raw * H;   // one view in the caller's images
    const size_t view_raw = row_raw * Hb;       // its band on the device
    // filtered rows padded to a 16-byte multiple so every width can use the
    // shared-memory (TMA) backprojector
    const int pitch = (W + 7) / 8 * 8;
    const size_t view_filt = size_t(pitch) * Hb * store_bytes(store_);
    const int chunk = int(std::max<size_t>(1, std::min<size_t>(size_t(V), (size_t(256) << 20) / view_raw)));
    const size_t plane = size_t(X) * Y;
    // default: about a quarter of the slices per slab, a multiple of 16 (1440
    // views of 2048^2 into 1024^3, end to end: 256 slices 0.6 % faster than
    // 128, fewer launch tails, while two slabs still cover the upload and the
    // cut last slab keeps the final download short)
    // the autotuner's choice for this shape when there is one (host/tuning.cpp)
    BpConfig bpc;
    int tuned_slab = 0;
    const bool tuned = tuned_for(z_lo, z_hi, &bpc, &tuned_slab);
    int slab = slab_req_ > 0 ? slab_req_ : tuned ? tuned_slab : std::max(16, ((Zw + 3) / 4 + 15) / 16 * 16);
    slab = std::min(slab, Zw);
    const bool convert = order == CTB_Z_FASTEST;
    {
        size_t freeb = 0, total = 0;
        cudaMemGetInfo(&freeb, &total);
        const size_t spare = spare_mb_ << 20;
        auto need = [&](int sl) {
            const size_t nb = std::min<size_t>(3, (Zw + sl - 1) / sl);
            return view_filt * V + 3 * view_raw * chunk + nb * plane * sl * 4 * (convert ? 2 : 1) + 64 * V +
                   size_t(M) * 12;
        };
        size_t have = w.d_filtered.bytes + w.d_ring.bytes;
        for (int b = 0; b < 3; ++b) have += w.d_slab[b].bytes + w.d_conv[b].bytes;
        while (slab > 16 && need(slab) > freeb + have - std::min(freeb + have, spare)) slab = std::max(16, slab / 2);
        if (need(slab) + spare > freeb + have)
            return fail(CTB_ERR_ALLOC,
                        "An error occured during allocation of memory for the volume in the VRAM. Maybe the amount "
                        "of free VRAM was insufficient. You can try changing the GPU spare memory setting.");
    }
    int st;
    if ((st = w.d_filtered.ensure(view_filt * V, "filtered projections")) ||
        (st = w.d_ring.ensure(3 * view_raw * chunk, "projection upload ring")) ||
        (st = w.d_views.ensure(sizeof(float4) * V, "view table")) ||
        (st = w.d_angles.ensure(sizeof(double) * V, "angles")) ||
        (st = w.d_heights.ensure(sizeof(double) * V, "height offsets")) ||
        (st = w.d_tw.ensure(sizeof(float2) * M, "twiddles")) || (st = w.d_K.ensure(sizeof(float) * M, "filter")))
        return fail(st, global_error());
    // Slab boundaries: slabs of `slab` slices, and a last one of 32 slices cut
    // from a full-height last slab, so that the download no backprojection
    // hides is short.
    std::vector<int> zbound;
    for (int z = z_lo; z < z_hi; z += slab) zbound.push_back(z);
    zbound.push_back(z_hi);
    if (zbound.size() >= 3 && zbound[zbound.size() - 1] - zbound[zbound.size() - 2] >= 64)
        zbound.insert(zbound.end() - 1, z_hi - 32);
    const int nslabs = int(zbound.size()) - 1;
    // device slab buffers: the first `pre` slabs are backprojected while the
    // views arrive (the upload alone would leave the GPU idle), a third buffer
    // lets the next slab start before the first one has gone to the host
    const int nbufs = std::min(3, nslabs);
    const int pre = std::min(2, nslabs);
    for (int b = 0; b < nbufs; ++b) {
        if ((st = w.d_slab[b].ensure(sizeof(float) * plane * slab, "volume slab"))) return fail(st, global_error());
        if (convert && (st = w.d_conv[b].ensure(sizeof(float) * plane * slab, "layout slab")))
            return fail(st, global_error());
    }
    const bool out_pinned = is_pinned(out);
    if (!out_pinned)
        for (auto& hb : w.h_stage)
            if (hb.ensure(sizeof(float) * plane * slab) != CTB_OK || !hb.pinned)
                return fail(CTB_ERR_ALLOC, "Pinned staging memory could not be allocated.");

    // ---- events
    cudaEvent_t ev_up[3], ev_free[3], ev_bp[3], ev_down[3], e_f0, e_f1, e_b0, e_b1, e_tab;
    const int nchunks = (V + chunk - 1) / chunk;
    std::vector<cudaEvent_t> tf(2 * nchunks), tb(2 * (nslabs + pre * nchunks)), ev_fd(nchunks);
    for (auto& e : tf) cudaEventCreate(&e);
    for (auto& e : ev_fd) cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
    cudaEventCreateWithFlags(&e_tab, cudaEventDisableTiming);
    for (auto& e : tb) cudaEventCreate(&e);
    for (auto& e : ev_up) cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
    for (auto& e : ev_free) cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
    for (auto& e : ev_bp) cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
    for (auto& e : ev_down) cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
    cudaEventCreate(&e_f0); cudaEventCreate(&e_f1); cudaEventCreate(&e_b0); cudaEventCreate(&e_b1);
    auto cleanup = [&]() {
        for (auto& e : ev_up) cudaEventDestroy(e);
        for (auto& e : ev_free) cudaEventDestroy(e);
        for (auto& e : ev_bp) cudaEventDestroy(e);
        for (auto& e : ev_down) cudaEventDestroy(e);
        cudaEventDestroy(e_f0); cudaEventDestroy(e_f1); cudaEventDestroy(e_b0); cudaEventDestroy(e_b1);
        cudaEventDestroy(e_tab);
        for (auto& e : tf) cudaEventDestroy(e);
        for (auto& e : tb) cudaEventDestroy(e);
        for (auto& e : ev_fd) cudaEventDestroy(e);
    };
    auto cuda_fail = [&](const char* what) {
        cudaStreamSynchronize(w.s_copy); cudaStreamSynchronize(w.s_comp); cudaStreamSynchronize(w.s_down);
        cudaStreamSynchronize(w.s_filt);
        cleanup();
        // the launch helpers record their own message when the CUDA error was
        // already taken (or when a launch was refused without one)
        const cudaError_t e = cudaGetLastError();
        return fail(CTB_ERR_CUDA, std::string(what) + ": " + (e != cudaSuccess ? cudaGetErrorString(e) : global_error()));
    };

    // ---- geometry tables (FP64 kernels)
    if (cudaMemcpyAsync(w.d_angles.p, ang.data(), sizeof(double) * V, cudaMemcpyHostToDevice, w.s_comp) ||
        cudaMemcpyAsync(w.d_heights.p, hp.data(), sizeof(double) * V, cudaMemcpyHostToDevice, w.s_comp))
        return cuda_fail("geometry upload");
    if (view_table_build((double*)w.d_angles.p, (double*)w.d_heights.p, V, (float4*)w.d_views.p, w.s_comp))
        return cuda_fail("view table");
    if (w.tables_key[0] != W || w.tables_key[1] != pad_ || w.tables_key[2] != filter_) {
        if (filter_build_tables(W, pad_, filter_, M, (float2*)w.d_tw.p, (float*)w.d_K.p, w.s_comp))
            return cuda_fail("filter tables");
        w.tables_key[0] = W; w.tables_key[1] = pad_; w.tables_key[2] = filter_;
    }
    // the ring slots start free; the filter stream starts after the tables
    for (auto& e : ev_free) cudaEventRecord(e, w.s_comp);
    cudaEventRecord(e_tab, w.s_comp);
    cudaStreamWaitEvent(w.s_filt, e_tab, 0);

    // ---- upload + filter; the first `pre` slabs are backprojected group by
    // group of views as they arrive, so the host-to-device transfer overlaps
    // with their backprojection. Filtering runs on its own stream at the
    // greatest priority (its blocks are scheduled ahead of the backprojection's
    // waiting ones), so it neither waits behind nor stalls the backprojection.
    // The groups grow while backprojecting the views so far takes longer than
    // uploading the next group (a nominal 1.7 TGUPS against 50 GB/s pinned):
    // fewer launches, each of which reads and writes the slabs once (1440
    // views of 2048^2 into 1024^3 end to end: 0.914 s against 0.925 s with a
    // launch every two chunks and the filter on the backprojection's stream).
    const bool in_pinned = is_pinned(images_);
    const double t_bp_view = double(pre) * double(slab) * double(plane) / 1.7e12;
    const double t_up_view = double(view_raw) / (in_pinned ? 50e9 : 10e9);
    const double growth = std::min(2.0, std::max(1.0, 0.9 * t_bp_view / t_up_view));
    int next_at = 2 * chunk;   // views that end the next early-slab group
    auto slab_geom = [&](int zb, int ze) {
        ProjGeom g = proj_geom(det_, grid_, zb, ze, load_scale);
        g.pitch = pitch;
        // rows of the band: row r of the band is detector row r + r_lo
        g.H = Hb;
        g.vPre = float(double(H) / 2.0 - double(r_lo));
        g.vi_hi = float(double(H) - 1 - 0.1 - double(r_lo));
        g.view_stride = (long long)pitch * Hb;
        return g;
    };
    ProjGeom gpre[2];
    for (int p = 0; p < pre; ++p) gpre[p] = slab_geom(zbound[p], zbound[p + 1]);
    int nb_ev = 0;  // backprojection event pairs used
    cudaEventRecord(e_f0, w.s_comp);
    int slot = 0;
    int bp_from = 0;  // first view not yet backprojected into the early slabs
    for (int c0 = 0; c0 < V; c0 += chunk, slot = (slot + 1) % 3) {
        if (stop_) { cuda_fail("stop"); return fail(CTB_INTERRUPTED, "User interrupted. Stopping."); }
        const int n = std::min(chunk, V - c0);
        char* dst = (char*)w.d_ring.p + size_t(slot) * view_raw * chunk;
        cudaStreamWaitEvent(w.s_copy, ev_free[slot], 0);
        const char* band0 = (const char*)images_ + size_t(r_lo) * row_raw;
        if (step_ <= 1 && Hb == H) {
            if (cudaMemcpyAsync(dst, (const char*)images_ + size_t(c0) * view_raw, view_raw * n,
                                cudaMemcpyHostToDevice, w.s_copy))
                return cuda_fail("projection upload");
        } else if (step_ <= 1) {
            // the band of n consecutive views: n rows of view_raw bytes, view_raw_full apart
            if (cudaMemcpy2DAsync(dst, view_raw, band0 + size_t(c0) * view_raw_full, view_raw_full, view_raw, n,
                                  cudaMemcpyHostToDevice, w.s_copy))
                return cuda_fail("projection upload");
        } else {
            for (int i = 0; i < n; ++i)
                if (cudaMemcpyAsync(dst + size_t(i) * view_raw, band0 + size_t(used[c0 + i]) * view_raw_full,
                                    view_raw, cudaMemcpyHostToDevice, w.s_copy))
                    return cuda_fail("projection upload");
        }
        cudaEventRecord(ev_up[slot], w.s_copy);
        cudaStreamWaitEvent(w.s_filt, ev_up[slot], 0);
        FilterArgs fa = filter_args(det_, raw_type_, M, logM, n, store_scale);
        fa.out_pitch = pitch;
        fa.H = Hb;                                         // the band's rows,
        fa.vPre = float(double(H) / 2.0 - double(r_lo));  // weighted as detector rows r + r_lo
        cudaEventRecord(tf[2 * (c0 / chunk)], w.s_filt);
        char* fdst = (char*)w.d_filtered.p + size_t(c0) * view_filt;
        if (filter_launch(dst, raw_type_, fdst, store_, fa, (const float2*)w.d_tw.p, (const float*)w.d_K.p, w.s_filt))
            return cuda_fail("filter launch");
        cudaEventRecord(tf[2 * (c0 / chunk) + 1], w.s_filt);
        cudaEventRecord(ev_free[slot], w.s_filt);
        cudaEventRecord(ev_fd[c0 / chunk], w.s_filt);
        if (c0 + n >= next_at || c0 + n == V) {
            // the group's views are filtered (those of earlier chunks before them)
            cudaStreamWaitEvent(w.s_comp, ev_fd[c0 / chunk], 0);
            for (int p = 0; p < pre; ++p) {
                cudaEventRecord(tb[2 * nb_ev], w.s_comp);
                if (backproject_launch((const char*)w.d_filtered.p + size_t(bp_from) * view_filt, store_,
                                       (const float4*)w.d_views.p + bp_from, c0 + n - bp_from, gpre[p], hmax,
                                       (float*)w.d_slab[p].p, bp_from > 0, w.s_comp, bpc))
                    return cuda_fail("backprojection launch");
                cudaEventRecord(tb[2 * nb_ev + 1], w.s_comp);
                ++nb_ev;
            }
            const int done = c0 + n - bp_from;
            bp_from = c0 + n;
            next_at = bp_from + std::max(2 * chunk, int(done * growth));
        }
        if (!in_pinned) cudaStreamSynchronize(w.s_copy);
    }
    cudaEventRecord(e_f1, w.s_comp);
    const int nb_early = nb_ev;  // backprojection launches of the upload phase

    // ---- backprojection per slab + layout + download
    cudaEventRecord(e_b0, w.s_comp);
    auto host_copy = [&](int k) {
        // pageable output: staged slab k (staging buffer k % 2) -> final position
        const int zb = zbound[k], zs = zbound[k + 1] - zb;
        cudaEventSynchronize(ev_down[k % nbufs]);
        const float* src = (const float*)w.h_stage[k % 2].p;
        if (order == CTB_Z_FASTEST) {
            parallel_for(plane, [&](size_t i) {
                std::memcpy(out + i * Z + zb, src + i * zs, sizeof(float) * zs);
            });
        } else {
            const size_t n = plane * zs;
            const size_t parts = 16;
            parallel_for(parts, [&](size_t p) {
                const size_t a = p * n / parts, e = (p + 1) * n / parts;
                std::memcpy(out + size_t(zb) * plane + a, src + a, sizeof(float) * (e - a));
            });
        }
    };
    for (int k = 0; k < nslabs; ++k) {
        if (stop_) { cuda_fail("stop"); return fail(CTB_INTERRUPTED, "User interrupted. Stopping."); }
        const int b = k % nbufs;
        const int zb = zbound[k], ze = zbound[k + 1], zs = ze - zb;
        if (k >= nbufs) cudaStreamWaitEvent(w.s_comp, ev_down[b], 0);
        if (k >= pre) {  // the first slabs were backprojected during the upload
            const ProjGeom g = slab_geom(zb, ze);
            cudaEventRecord(tb[2 * nb_ev], w.s_comp);
            if (backproject_launch(w.d_filtered.p, store_, (const float4*)w.d_views.p, V, g, hmax,
                                   (float*)w.d_slab[b].p, 0, w.s_comp, bpc))
                return cuda_fail("backprojection launch");
            cudaEventRecord(tb[2 * nb_ev + 1], w.s_comp);
            ++nb_ev;
        }
        const float* src = (const float*)w.d_slab[b].p;
        if (convert) {
            if (layout_launch(src, X, Y, zs, CTB_Z_FASTEST, CTB_LITTLE_ENDIAN, w.d_conv[b].p, w.s_comp))
                return cuda_fail("layout launch");
            src = (const float*)w.d_conv[b].p;
        }
        cudaEventRecord(ev_bp[b], w.s_comp);
        cudaStreamWaitEvent(w.s_down, ev_bp[b], 0);
        cudaError_t ce;
        if (out_pinned) {
            if (convert)
                ce = cudaMemcpy2DAsync(out + zb, sizeof(float) * Z, src, sizeof(float) * zs, sizeof(float) * zs,
                                       plane, cudaMemcpyDeviceToHost, w.s_down);
            else
                ce = cudaMemcpyAsync(out + size_t(zb) * plane, src, sizeof(float) * plane * zs,
                                     cudaMemcpyDeviceToHost, w.s_down);
        } else {
            if (k >= 2) host_copy(k - 2);  // frees staging buffer k % 2
            ce = cudaMemcpyAsync(w.h_stage[k % 2].p, src, sizeof(float) * plane * zs, cudaMemcpyDeviceToHost,
                                 w.s_down);
        }
        if (ce != cudaSuccess) return cuda_fail("volume download");
        cudaEventRecord(ev_down[b], w.s_down);
        // previews read the context's own volume up to the previous slab, which
        // has landed by now (waiting for this one would stall the next launch)
        const bool preview = previews() && out == static_cast<float*>(volume_.p) && out_pinned && k >= 1;
        if (preview) cudaEventSynchronize(ev_down[(k - 1) % nbufs]);
        worker_progress(w, double(k + 1) / double(nslabs), preview ? out : nullptr);
    }
    cudaEventRecord(e_b1, w.s_comp);
    if (!out_pinned)
        for (int k = std::max(0, nslabs - 2); k < nslabs; ++k) host_copy(k);
    if (cudaStreamSynchronize(w.s_down) != cudaSuccess || cudaStreamSynchronize(w.s_comp) != cudaSuccess ||
        cudaStreamSynchronize(w.s_copy) != cudaSuccess || cudaStreamSynchronize(w.s_filt) != cudaSuccess)
        return cuda_fail("reconstruction");
    unsigned gave_up = 0;
    if (device_wait_timeouts(&gave_up, 1) == CTB_OK && gave_up) {
        cleanup();
        return fail(CTB_ERR_TIMEOUT, "A device wait of the backprojection gave up (" + std::to_string(gave_up) +
                                         " times); the volume is incomplete.");
    }
    float phase_ms = 0, tail_ms = 0;
    double f_ms = 0, b_ms = 0;
    cudaEventElapsedTime(&phase_ms, e_f0, e_f1);
    for (int i = 0; i < nchunks; ++i) { float t = 0; cudaEventElapsedTime(&t, tf[2 * i], tf[2 * i + 1]); f_ms += t; }
    double bp0_ms = 0;
    for (int i = 0; i < nb_ev; ++i) {
        float t = 0;
        cudaEventElapsedTime(&t, tb[2 * i], tb[2 * i + 1]);
        b_ms += t;
        if (i < nb_early) bp0_ms += t;
    }
    cudaEventElapsedTime(&tail_ms, e_b0, e_b1);
    cleanup();
    const double total = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
    w.filter_s = f_ms * 1e-3;
    w.backproject_s = b_ms * 1e-3;
    // the backprojection stream's idle time in the upload phase (filtering runs beside it)
    w.upload_s = std::max(0.0, (phase_ms - bp0_ms) * 1e-3);
    w.download_s = std::max(0.0, total - (phase_ms + tail_ms) * 1e-3);
    w.h2d_bytes = double(view_raw) * V;
    w.d2h_bytes = double(plane) * Zw * sizeof(float);
    return CTB_OK;
}

int Reconstructor::get_volume(float* host_out, int index_order) const {
    const int X = vol_dims_[0], Y = vol_dims_[1], Z = vol_dims_[2];
    if (X == 0 || !volume_.p) return CTB_ERR_ARG;
    const float* v = static_cast<const float*>(volume_.p);
    if (index_order == CTB_X_FASTEST) {
        std::memcpy(host_out, v, sizeof(float) * size_t(X) * Y * Z);
    } else {
        parallel_for(size_t(X), [&](size_t x) {
            for (int y = 0; y < Y; ++y)
                for (int z = 0; z < Z; ++z)
                    host_out[(x * Y + y) * Z + z] = v[(size_t(z) * Y + y) * X + x];
        });
    }
    return CTB_OK;
}

}  // namespace ctb
