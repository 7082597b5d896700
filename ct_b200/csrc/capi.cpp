// extern "C" entry points of libctb (declared in include/ctb.h).

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <new>
#include <string>

#include "ctb_internal.h"
#include "host/image_io.h"
#include "host/reconstructor.h"

struct ctb_ctx {
    ctb::Reconstructor r;
};

namespace {

using ctb::valid_detector;
using ctb::valid_grid;

int arg_error(const char* msg) {
    ctb::set_global_error(msg);
    return CTB_ERR_ARG;
}

// Device view table {sin, cos, h} from host angle / height arrays.
int upload_views(const double* ang, const double* h, int n, cudaStream_t s, float4** views) {
    double* d = nullptr;
    CTB_CUDA_TRY(cudaMallocAsync((void**)&d, sizeof(double) * 2 * n, s));
    CTB_CUDA_TRY(cudaMallocAsync((void**)views, sizeof(float4) * n, s));
    CTB_CUDA_TRY(cudaMemcpyAsync(d, ang, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    if (h) {
        CTB_CUDA_TRY(cudaMemcpyAsync(d + n, h, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    } else {
        CTB_CUDA_TRY(cudaMemsetAsync(d + n, 0, sizeof(double) * n, s));
    }
    int st = ctb::view_table_build(d, d + n, n, *views, s);
    CTB_CUDA_TRY(cudaFreeAsync(d, s));
    return st;
}

}  // namespace

extern "C" {

// ------------------------------------------------------------ operator layer
int ctb_device_count(int* count) {
    if (!count) return arg_error("null pointer");
    return ctb::cuda_status(cudaGetDeviceCount(count), "cudaGetDeviceCount");
}

int ctb_device_name(int device, char* buf, size_t buf_len) {
    if (!buf || buf_len == 0) return arg_error("null buffer");
    cudaDeviceProp p;
    CTB_CUDA_TRY(cudaGetDeviceProperties(&p, device));
    std::strncpy(buf, p.name, buf_len - 1);
    buf[buf_len - 1] = '\0';
    return CTB_OK;
}

int ctb_free_memory(int device, size_t* free_bytes, size_t* total_bytes) {
    int cur = 0;
    CTB_CUDA_TRY(cudaGetDevice(&cur));
    CTB_CUDA_TRY(cudaSetDevice(device));
    size_t f = 0, t = 0;
    const cudaError_t e = cudaMemGetInfo(&f, &t);
    cudaSetDevice(cur);
    CTB_CUDA_TRY(e);
    if (free_bytes) *free_bytes = f;
    if (total_bytes) *total_bytes = t;
    return CTB_OK;
}

int ctb_reference_grid(ctb_detector* det, const float rel6[6], ctb_grid* grid) {
    if (!det || !grid || det->width <= 1 || det->height <= 1) return arg_error("invalid detector");
    float r[6] = {0, 1, 0, 1, 0, 1};
    if (rel6) {
        if (rel6[0] == rel6[1] || rel6[2] == rel6[3] || rel6[4] == rel6[5])
            return arg_error("ERROR: the lower and upper bounds must not be identical.");
        r[0] = std::max(0.0f, std::min(1.0f, rel6[0]));
        r[1] = std::max(r[0], std::min(1.0f, rel6[1]));
        r[2] = std::max(0.0f, std::min(1.0f, rel6[2]));
        r[3] = std::max(r[0], std::min(1.0f, rel6[3]));
        r[4] = std::max(0.0f, std::min(1.0f, rel6[4]));
        r[5] = std::max(r[0], std::min(1.0f, rel6[5]));
    }
    const double rad = unsigned(det->width) / 2;
    const double D = det->fcd;
    const unsigned radius = unsigned(std::sqrt((D * D * rad * rad) / (D * D + rad * rad)));
    det->radius = float(radius);
    grid->x_size = int(2 * radius);
    grid->y_size = int(2 * radius);
    grid->z_size = det->height;
    grid->x_from = int(unsigned(r[0] * grid->x_size + 0.5)); grid->x_to = int(unsigned(r[1] * grid->x_size + 0.5));
    grid->y_from = int(unsigned(r[2] * grid->y_size + 0.5)); grid->y_to = int(unsigned(r[3] * grid->y_size + 0.5));
    grid->z_from = int(unsigned(r[4] * grid->z_size + 0.5)); grid->z_to = int(unsigned(r[5] * grid->z_size + 0.5));
    grid->voxel_pitch = 1.0f;
    return CTB_OK;
}

int ctb_row_band(const ctb_detector* det, const ctb_grid* grid, int z_begin, int z_end,
                 const double* height_offsets_px, int n_views, int* r_lo, int* rows) {
    if (!det || !grid || !r_lo || !rows || !valid_detector(det) || !valid_grid(grid) || n_views < 0)
        return arg_error("invalid row band arguments");
    if (det->radius <= 0) return arg_error("detector radius not set (use ctb_reference_grid)");
    if (z_begin < 0 || z_end <= z_begin || z_end > grid->z_to - grid->z_from) return arg_error("invalid z range");
    ctb::row_band(*det, *grid, z_begin, z_end, height_offsets_px, n_views, r_lo, rows);
    return CTB_OK;
}

int ctb_filter_projections(const void* raw, int raw_type, int n_views, const ctb_detector* det, int filter,
                           int pad, void* filtered, int store_type, float store_scale, void* stream) {
    if (!raw || !filtered || n_views < 0 || !valid_detector(det)) return arg_error("invalid filter arguments");
    if (raw_type != CTB_U8 && raw_type != CTB_U16 && raw_type != CTB_F32) return arg_error("unknown raw type");
    if (filter < CTB_RAMLAK || filter > CTB_HANN) return arg_error("unknown filter type");
    if (pad != 1 && pad != 2) return arg_error("pad must be 1 or 2");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    ctb::FilterTables t;
    int st = ctb::filter_tables(det->width, pad, filter, s, &t);
    if (st != CTB_OK) return st;
    const ctb::FilterArgs a = ctb::filter_args(*det, raw_type, t.M, t.logM, n_views, store_scale);
    return ctb::filter_launch(raw, raw_type, filtered, store_type, a, t.tw, t.K, s);
}

int ctb_backproject(const void* filtered, int store_type, int n_views, const double* angles_deg,
                    const double* height_offsets_px, const ctb_detector* det, const ctb_grid* grid, int z_begin,
                    int z_end, float load_scale, float* vol, int accumulate, void* stream) {
    if (!filtered || !vol || !angles_deg || n_views <= 0 || !valid_detector(det) || !valid_grid(grid))
        return arg_error("invalid backprojection arguments");
    if (z_begin < 0 || z_end <= z_begin || z_end > grid->z_to - grid->z_from) return arg_error("invalid z range");
    if (det->radius <= 0) return arg_error("detector radius not set (use ctb_reference_grid)");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    float4* views = nullptr;
    int st = upload_views(angles_deg, height_offsets_px, n_views, s, &views);
    if (st != CTB_OK) return st;
    const ctb::ProjGeom g = ctb::proj_geom(*det, *grid, z_begin, z_end, load_scale);
    double hmax = 0;
    if (height_offsets_px)
        for (int i = 0; i < n_views; ++i) hmax = std::max(hmax, std::fabs(height_offsets_px[i]));
    st = ctb::backproject_launch(filtered, store_type, views, n_views, g, hmax, vol, accumulate, s);
    cudaFreeAsync(views, s);
    return st;
}

int ctb_read_image(const char* path, int* width, int* height, int* raw_type, void* out) {
    if (!path || !width || !height || !raw_type) return arg_error("null pointer");
    std::string err;
    if (!ctb::probe_image(path, width, height, raw_type, &err)) {
        ctb::set_global_error(err);
        return CTB_ERR_IMAGE;
    }
    if (out && !ctb::decode_image_into(path, *width, *height, *raw_type, out, &err)) {
        ctb::set_global_error(err);
        return CTB_ERR_IMAGE;
    }
    return CTB_OK;
}

int ctb_device_wait_timeouts(int device, unsigned* count, int reset) {
    if (!count) return arg_error("null pointer");
    int prev = 0;
    CTB_CUDA_TRY(cudaGetDevice(&prev));
    CTB_CUDA_TRY(cudaSetDevice(device));
    const int st = ctb::device_wait_timeouts(count, reset);
    cudaSetDevice(prev);
    return st;
}

int ctb_diag_bounded_wait(int device, unsigned limit) {
    int prev = 0;
    CTB_CUDA_TRY(cudaGetDevice(&prev));
    CTB_CUDA_TRY(cudaSetDevice(device));
    const int st = ctb::bounded_wait_probe_run(limit, nullptr);
    cudaSetDevice(prev);
    return st;
}

void ctb_diag_force_overflow(int every) { ctb::bp_force_overflow(every); }

void ctb_diag_fail_allocation(long nth) { ctb::fail_allocation_after(nth); }

int ctb_diag_bounds_status(int device, int* checked_build, unsigned* violations, unsigned long long* first,
                           int reset) {
    if (!checked_build || !violations || !first) return arg_error("null pointer");
#ifdef CTB_BOUNDS_CHECK
    *checked_build = 1;
#else
    *checked_build = 0;
#endif
    int prev = 0;
    CTB_CUDA_TRY(cudaGetDevice(&prev));
    CTB_CUDA_TRY(cudaSetDevice(device));
    unsigned c1 = 0, c2 = 0;
    unsigned long long f1 = 0, f2 = 0;
    int st = ctb::bounds_status_tma(&c1, &f1, reset);
    if (st == CTB_OK) st = ctb::bounds_status_gather(&c2, &f2, reset);
    cudaSetDevice(prev);
    *violations = c1 + c2;
    *first = f1 ? f1 : f2;
    return st;
}

int ctb_forward_project(const float* vol, const double* angles_deg, const double* height_offsets_px, int n_views,
                        const ctb_detector* det, const ctb_grid* grid, int z_begin, int z_end, float* proj,
                        int accumulate, void* stream) {
    if (!vol || !proj || !angles_deg || n_views <= 0 || !valid_detector(det) || !valid_grid(grid))
        return arg_error("invalid forward projection arguments");
    if (z_begin < 0 || z_end <= z_begin || z_end > grid->z_to - grid->z_from) return arg_error("invalid z range");
    if (det->radius <= 0) return arg_error("detector radius not set (use ctb_reference_grid)");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    float4* views = nullptr;
    int st = upload_views(angles_deg, height_offsets_px, n_views, s, &views);
    if (st != CTB_OK) return st;
    const ctb::ProjGeom g = ctb::proj_geom(*det, *grid, z_begin, z_end, 1.0f);
    st = ctb::forward_launch(vol, views, n_views, g, proj, accumulate, s);
    cudaFreeAsync(views, s);
    return st;
}

int ctb_convert_layout(const float* src, int x, int y, int zs, int index_order, int byte_order, void* dst,
                       void* stream) {
    if (!src || !dst) return arg_error("null pointer");
    return ctb::layout_launch(src, x, y, zs, index_order, byte_order, dst, static_cast<cudaStream_t>(stream));
}

int ctb_phantom_project(const double* ellipsoids_dev, int n_ellipsoids, const double* angles_deg,
                        const double* height_offsets_mm, int n_views, int width, int height, double pixel_mm,
                        double fcd_mm, double u_offset_mm, double* out_dev, void* stream) {
    if (!ellipsoids_dev || !angles_deg || !out_dev || n_ellipsoids < 0) return arg_error("invalid phantom args");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    double* d = nullptr;
    CTB_CUDA_TRY(cudaMallocAsync((void**)&d, sizeof(double) * 2 * n_views, s));
    CTB_CUDA_TRY(cudaMemcpyAsync(d, angles_deg, sizeof(double) * n_views, cudaMemcpyHostToDevice, s));
    if (height_offsets_mm)
        CTB_CUDA_TRY(cudaMemcpyAsync(d + n_views, height_offsets_mm, sizeof(double) * n_views, cudaMemcpyHostToDevice, s));
    else
        CTB_CUDA_TRY(cudaMemsetAsync(d + n_views, 0, sizeof(double) * n_views, s));
    int st = ctb::phantom_launch(ellipsoids_dev, n_ellipsoids, d, d + n_views, n_views, width, height, pixel_mm,
                                 fcd_mm, u_offset_mm, out_dev, s);
    cudaFreeAsync(d, s);
    return st;
}

// ------------------------------------------------------------ facade layer
int ctb_create(ctb_ctx** ctx) {
    if (!ctx) return arg_error("null pointer");
    *ctx = new (std::nothrow) ctb_ctx();
    return *ctx ? CTB_OK : CTB_ERR_ALLOC;
}

void ctb_destroy(ctb_ctx* ctx) { delete ctx; }

const char* ctb_last_error(const ctb_ctx* ctx) { return ctx ? ctx->r.error().c_str() : ""; }
const char* ctb_last_error_global(void) { return ctb::global_error().c_str(); }

#define CTX_CHECK(ctx) \
    if (!(ctx)) return arg_error("null context")

int ctb_load_csv(ctb_ctx* ctx, const char* csv_path) {
    CTX_CHECK(ctx);
    if (!csv_path) return arg_error("null path");
    return ctx->r.load_csv(csv_path);
}

int ctb_set_projections(ctb_ctx* ctx, const void* host_images, int raw_type, int n_views, int width, int height,
                        const double* angles_deg, const double* height_offsets_mm, double pixel_size, int ccw,
                        double u_offset_mm, double fcd_mm, double base_intensity) {
    CTX_CHECK(ctx);
    return ctx->r.set_projections(host_images, raw_type, n_views, width, height, angles_deg, height_offsets_mm,
                                  pixel_size, ccw, u_offset_mm, fcd_mm, base_intensity);
}

int ctb_set_volume_bounds(ctb_ctx* ctx, float xmin, float xmax, float ymin, float ymax, float zmin, float zmax) {
    CTX_CHECK(ctx);
    return ctx->r.set_bounds(xmin, xmax, ymin, ymax, zmin, zmax);
}
int ctb_set_filter(ctb_ctx* ctx, int filter) { CTX_CHECK(ctx); return ctx->r.set_filter(filter); }
int ctb_set_skip_projections(ctb_ctx* ctx, unsigned skip) { CTX_CHECK(ctx); return ctx->r.set_skip(skip); }
int ctb_set_device(ctb_ctx* ctx, int device) { CTX_CHECK(ctx); return ctx->r.set_device(device); }
int ctb_set_gpu_spare_memory(ctb_ctx* ctx, size_t mb) { CTX_CHECK(ctx); return ctx->r.set_spare_mb(mb); }
int ctb_set_devices(ctb_ctx* ctx, const int* ids, int n) {
    CTX_CHECK(ctx);
    if (!ids || n <= 0) return arg_error("empty device list");
    return ctx->r.set_devices(ids, n);
}
int ctb_set_gpu_coefficients(ctb_ctx* ctx, double mp, double bw) {
    CTX_CHECK(ctx);
    return ctx->r.set_gpu_coefficients(mp, bw);
}
int ctb_get_gpu_weights(ctb_ctx* ctx, const int* ids, int n, double* weights) {
    CTX_CHECK(ctx);
    if (!ids || !weights || n <= 0) return arg_error("empty device list");
    return ctx->r.gpu_weights(ids, n, weights);
}
int ctb_gpu_weights_from(const int* sm_count, const double* bandwidth, int n, double mp, double bw, double* weights) {
    if (!sm_count || !bandwidth || !weights || n <= 0) return arg_error("empty device list");
    ctb::gpu_weights_from(sm_count, bandwidth, n, mp, bw, weights);
    return CTB_OK;
}
int ctb_split_slices(const double* weights, int n, int z, int* begin) {
    if (!weights || !begin || n <= 0 || z < 0) return arg_error("invalid split arguments");
    ctb::split_slices(weights, n, z, begin);
    return CTB_OK;
}
int ctb_set_precision(ctb_ctx* ctx, int store_type) { CTX_CHECK(ctx); return ctx->r.set_precision(store_type); }
int ctb_set_pad(ctb_ctx* ctx, int pad) { CTX_CHECK(ctx); return ctx->r.set_pad(pad); }
int ctb_set_grid(ctb_ctx* ctx, int x, int y, int z, float vs) { CTX_CHECK(ctx); return ctx->r.set_grid(x, y, z, vs); }
int ctb_set_slab_height(ctb_ctx* ctx, int slices) { CTX_CHECK(ctx); return ctx->r.set_slab(slices); }
int ctb_set_progress_callback(ctb_ctx* ctx, ctb_progress_cb cb, void* user) {
    CTX_CHECK(ctx);
    ctx->r.set_progress(cb, user);
    return CTB_OK;
}

int ctb_get_detector(const ctb_ctx* ctx, ctb_detector* det) {
    CTX_CHECK(ctx);
    if (!det) return arg_error("null pointer");
    *det = ctx->r.detector();
    return CTB_OK;
}
int ctb_get_grid(const ctb_ctx* ctx, ctb_grid* grid) {
    CTX_CHECK(ctx);
    if (!grid) return arg_error("null pointer");
    *grid = ctx->r.grid();
    return CTB_OK;
}
int ctb_get_volume_size(const ctb_ctx* ctx, int* x, int* y, int* z) {
    CTX_CHECK(ctx);
    const ctb_grid& g = ctx->r.grid();
    if (x) *x = g.x_to - g.x_from;
    if (y) *y = g.y_to - g.y_from;
    if (z) *z = g.z_to - g.z_from;
    return CTB_OK;
}
int ctb_get_sinogram_size(const ctb_ctx* ctx, int* n) {
    CTX_CHECK(ctx);
    if (n) *n = ctx->r.views();
    return CTB_OK;
}
double ctb_get_pixel_size(const ctb_ctx* ctx) { return ctx ? ctx->r.pixel_size() : 0.0; }

int ctb_reconstruct(ctb_ctx* ctx) { CTX_CHECK(ctx); return ctx->r.reconstruct(nullptr, CTB_X_FASTEST); }

int ctb_reconstruct_into(ctb_ctx* ctx, float* host_volume, int index_order) {
    CTX_CHECK(ctx);
    if (!host_volume) return arg_error("null output buffer");
    if (index_order != CTB_X_FASTEST && index_order != CTB_Z_FASTEST) return arg_error("unknown index order");
    return ctx->r.reconstruct(host_volume, index_order);
}

int ctb_get_volume(const ctb_ctx* ctx, float* host_volume, int index_order) {
    CTX_CHECK(ctx);
    if (!host_volume) return arg_error("null output buffer");
    return ctx->r.get_volume(host_volume, index_order);
}

int ctb_save_volume(ctb_ctx* ctx, const char* path, int index_order, int byte_order) {
    CTX_CHECK(ctx);
    if (!path) return arg_error("null path");
    return ctx->r.save(path, index_order, byte_order);
}

int ctb_set_cross_section_axis(ctb_ctx* ctx, int axis) {
    CTX_CHECK(ctx);
    return ctx->r.set_cross_section_axis(axis);
}
int ctb_set_cross_section_index(ctb_ctx* ctx, int index) {
    CTX_CHECK(ctx);
    return ctx->r.set_cross_section_index(index);
}
int ctb_get_cross_section_info(const ctb_ctx* ctx, int* axis, int* index, int* size) {
    CTX_CHECK(ctx);
    if (axis) *axis = ctx->r.cross_section_axis();
    if (index) *index = ctx->r.cross_section_index();
    if (size) *size = ctx->r.cross_section_size();
    return CTB_OK;
}
int ctb_set_preview_callback(ctb_ctx* ctx, ctb_preview_cb cb, void* user) {
    CTX_CHECK(ctx);
    ctx->r.set_preview(cb, user);
    return CTB_OK;
}
int ctb_get_cross_section(const ctb_ctx* ctx, int axis, int index, float* out, int* rows, int* cols) {
    CTX_CHECK(ctx);
    if (axis < CTB_AXIS_X || axis > CTB_AXIS_Z) return arg_error("unknown axis");
    const int st = ctx->r.cross_section(axis, index, out, rows, cols);
    if (st != CTB_OK) ctb::set_global_error("no reconstructed volume or index out of bounds");
    return st;
}

int ctb_set_autotune(ctb_ctx* ctx, int on) {
    if (!ctx) return arg_error("null context");
    ctx->r.set_autotune(on != 0);
    return CTB_OK;
}

int ctb_autotune(ctb_ctx* ctx, ctb_tuning* out) {
    if (!ctx) return arg_error("null context");
    return ctx->r.autotune(out);
}

int ctb_get_tuning(const ctb_ctx* ctx, ctb_tuning* out) {
    if (!ctx || !out) return arg_error("null pointer");
    return ctx->r.tuning(out);
}

int ctb_forward(ctb_ctx* ctx, const float* host_volume, float* host_projections) {
    if (!ctx) return arg_error("null context");
    return ctx->r.forward(host_volume, host_projections);
}

int ctb_backward(ctb_ctx* ctx, const float* host_projections, float* host_volume) {
    if (!ctx) return arg_error("null context");
    return ctx->r.backward(host_projections, host_volume);
}

int ctb_gradient(ctb_ctx* ctx, const float* host_volume, const float* host_data, float* host_gradient,
                 double* loss) {
    if (!ctx) return arg_error("null context");
    return ctx->r.gradient(host_volume, host_data, host_gradient, loss);
}

int ctb_batch_reconstruct(ctb_ctx* ctx, int n_scans, const ctb_scan* scans, void* stream) {
    if (!ctx) return arg_error("null context");
    ctb_batch* b = nullptr;
    int st = ctb_batch_create(&b, n_scans, scans, ctx->r.precision(), stream);
    if (st == CTB_OK) st = ctb_batch_run(b, stream);
    if (b) {
        // the graph reads the batch's buffers until it has run
        const cudaError_t e = cudaStreamSynchronize(static_cast<cudaStream_t>(stream));
        if (st == CTB_OK && e != cudaSuccess) st = ctb::cuda_status(e, "ctb_batch_reconstruct");
        ctb_batch_destroy(b);
    }
    return st;
}

void ctb_stop(ctb_ctx* ctx) {
    if (ctx) ctx->r.stop();
}

int ctb_set_use_cuda(ctb_ctx* ctx, int v) { CTX_CHECK(ctx); return ctx->r.set_use_cuda(v != 0); }
int ctb_set_use_cpu_preprocessing(ctb_ctx* ctx, int v) {
    CTX_CHECK(ctx);
    ctx->r.set_use_cpu_preprocessing(v != 0);
    return CTB_OK;
}
int ctb_set_emit_signals(ctb_ctx* ctx, int v) {
    CTX_CHECK(ctx);
    ctx->r.set_emit_signals(v != 0);
    return CTB_OK;
}
int ctb_get_settings(const ctb_ctx* ctx, ctb_settings* s) {
    CTX_CHECK(ctx);
    if (!s) return arg_error("null pointer");
    ctx->r.settings(s);
    return CTB_OK;
}
int ctb_get_required_memory(const ctb_ctx* ctx, size_t* bytes) {
    CTX_CHECK(ctx);
    if (!bytes) return arg_error("null pointer");
    *bytes = ctx->r.required_memory();
    return CTB_OK;
}
int ctb_get_projection(ctb_ctx* ctx, int index, float* image, double* angle_deg, double* height_offset_px) {
    CTX_CHECK(ctx);
    return ctx->r.projection(index, image, angle_deg, height_offset_px);
}

int ctb_get_timings(const ctb_ctx* ctx, ctb_timings* t) {
    CTX_CHECK(ctx);
    if (!t) return arg_error("null pointer");
    *t = ctx->r.timings();
    return CTB_OK;
}

}  // extern "C"
