/*
 * ctb.h -- C ABI of the B200 FDK cone-beam reconstruction engine.
 *
 * Two layers, mirroring the two layers of the reference (bastian-weber/Ct):
 *
 *  1. Operator layer (device pointers + a CUDA stream), replacing the
 *     reference's kernel API in Ct/cuda_ct.h:18-69 and the OpenCV/cuFFT glue in
 *     Ct/CtVolume.cpp:887-921.  Callers own all device memory they pass.
 *
 *  2. Reconstruction facade (opaque context), replacing the public surface of
 *     ct::CtVolume (Ct/CtVolume.h:63-121): load the CSV + images, set bounds and
 *     filter, reconstruct, save.  The context owns its device memory.
 *
 * Conventions
 *  - Every function returns an int status (CTB_OK == 0) unless stated; a
 *    human-readable message for the last failure is kept per context
 *    (ctb_last_error) or per thread for context-free calls
 *    (ctb_last_error_global).  No C++ exception crosses this boundary.
 *    Reference: bool& success out-params + lastErrorMessage +
 *    CompletionStatus (Ct/cuda_ct.cu:95-99, Ct/CtVolume.h:260, Common/types.h:11-20).
 *  - Units follow the reference: detector coordinates in pixels of the virtual
 *    detector at the rotation axis (CSV pixel size), FCD and uOffset divided by
 *    the pixel size (Ct/CtVolume.cpp:170-172), angles in degrees.
 *  - Volumes on the device are X-fastest (idx = z*X*Y + y*X + x), as the
 *    reference's GPU path (Ct/cuda_ct.cu:193-199).
 *  - cudaStream_t is passed as void* so this header needs no CUDA include.
 */
#ifndef CTB_H
#define CTB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------ status codes */
enum {
    CTB_OK = 0,
    CTB_ERR_ARG = 1,         /* invalid argument / state */
    CTB_ERR_IO = 2,          /* file could not be opened, read or written */
    CTB_ERR_CSV = 3,         /* configuration file could not be parsed */
    CTB_ERR_IMAGE = 4,       /* image missing, unsupported depth or size mismatch */
    CTB_ERR_ALLOC = 5,       /* device or pinned host allocation failed */
    CTB_ERR_CUDA = 6,        /* CUDA runtime error */
    CTB_ERR_TIMEOUT = 7,     /* a bounded device wait gave up */
    CTB_INTERRUPTED = 8,     /* ctb_stop() was called (CompletionStatus::interrupted) */
    CTB_ERR_UNSUPPORTED = 9  /* size or option beyond what this build supports */
};

/* FilterType, Ct/CtVolume.h:50-54 (same numeric values). */
enum { CTB_RAMLAK = 0, CTB_SHEPPLOGAN = 1, CTB_HANN = 2 };

/* IndexOrder, Common/Volume.h:29-32. */
enum { CTB_X_FASTEST = 0, CTB_Z_FASTEST = 1 };

/* QDataStream::ByteOrder as used by saveVolumeToBinaryFile. */
enum { CTB_LITTLE_ENDIAN = 0, CTB_BIG_ENDIAN = 1 };

/* Storage type of raw / filtered projections; arithmetic is always FP32. */
enum { CTB_FP32 = 0, CTB_FP16 = 1, CTB_BF16 = 2 };

/* Raw projection pixel types accepted (cv::imread depths the reference accepts,
 * Ct/CtVolume.cpp:247). */
enum { CTB_U8 = 8, CTB_U16 = 16, CTB_F32 = 32 };

/* -------------------------------------------------------- geometry records */

/* Per-scan detector/orbit geometry in reference units. */
typedef struct {
    int32_t width;          /* W, detector columns */
    int32_t height;         /* H, detector rows */
    float fcd;              /* focus-centre distance in pixels (CSV FCD / pixelSize) */
    float u_offset;         /* rotation axis offset in pixels (CSV uOffset / pixelSize) */
    float base_intensity;   /* air intensity (CSV line 6), normalised scale */
    float radius;           /* reconstruction cylinder radius in pixels */
} ctb_detector;

/* Reconstructed box inside the full grid, plus the voxel pitch. The reference
 * grid is xSize = ySize = 2*radius, zSize = H, voxel pitch 1 pixel
 * (Ct/CtVolume.cpp:311-316); from/to follow updateBoundaries (:1399-1409). */
typedef struct {
    int32_t x_size, y_size, z_size;          /* full grid */
    int32_t x_from, x_to, y_from, y_to, z_from, z_to;  /* box, half-open */
    float voxel_pitch;                       /* voxel edge in detector pixels (1 = reference) */
} ctb_grid;

/* ------------------------------------------------------- operator layer */

/* Device queries, Ct/cuda_ct.h:18-23. */
int ctb_device_count(int* count);
int ctb_device_name(int device, char* buf, size_t buf_len);
int ctb_free_memory(int device, size_t* free_bytes, size_t* total_bytes);

/* Reference grid for a detector (grid rule Ct/CtVolume.cpp:311-316 and
 * cylinder radius :370-373) with relative bounds rel6 = {xmin,xmax,ymin,ymax,
 * zmin,zmax} clamped like setVolumeBounds (:487-500). det->radius is set. */
int ctb_reference_grid(ctb_detector* det, const float rel6[6], ctb_grid* grid);

/* Detector rows [*r_lo, *r_lo + *rows) that the voxels of box slices
 * [z_begin, z_end) reach in any of n views with the given height offsets
 * (pixels; NULL = none), bilinear neighbours and a margin included: the rows a
 * device reconstructing only those slices needs to upload and filter (the
 * facade does so per device). No reference counterpart: the reference
 * uploads and filters every row on every device. det->radius must be set. */
int ctb_row_band(const ctb_detector* det, const ctb_grid* grid, int z_begin, int z_end,
                 const double* height_offsets_px, int n_views, int* r_lo, int* rows);

/* Preprocess and ramp-filter n_views raw projections in one launch sequence:
 * -ln of the normalised intensity, Feldkamp cosine weight, and the row-wise
 * ramp filter (ramlak / shepplogan / hann) applied in frequency with the
 * reference's window sampling. Replaces cudaPreprocessImage
 * (Ct/CtVolume.cpp:887-921) = convertTo/log/multiply + applyFeldkampWeightFiltering
 * (Ct/cuda_ct.h:28-33) + cuFFT R2C + applyFrequencyFiltering (Ct/cuda_ct.h:24-27)
 * + cuFFT C2R.
 *   raw:       device, n_views x H x W of raw_type (CTB_U8/U16/F32), dense.
 *   filtered:  device, n_views x H x W of store_type (CTB_FP32/FP16/BF16).
 *   pad:       1 = reference-exact circular filter of length W (no padding);
 *              2 = linear filter zero-padded to the next power of two >= 2W.
 *   store_scale: filtered values are multiplied by this before storage
 *              (1 for FP32; FP16/BF16 use a scale that keeps values near 1). */
int ctb_filter_projections(const void* raw, int raw_type, int n_views, const ctb_detector* det,
                           int filter, int pad, void* filtered, int store_type, float store_scale,
                           void* stream);

/* Voxel-driven FDK backprojection of n_views filtered projections into the
 * z-slab [z_begin, z_end) of the box (indices relative to grid->z_from),
 * X-fastest, slab-local: vol[(z - z_begin)*X*Y + y*X + x].
 * Replaces startReconstruction / reconstructionKernel (Ct/cuda_ct.h:47-69,
 * Ct/cuda_ct.cu:201-352), which adds one view per launch into a pitched chunk.
 *   angles_deg / height_offsets_px: host arrays (n_views), after the
 *     reference's direction correction and relative height offsets.
 *   load_scale: multiplies every sample (1/store_scale of the filter).
 *   accumulate: 0 = overwrite the slab, 1 = add to it. */
int ctb_backproject(const void* filtered, int store_type, int n_views, const double* angles_deg,
                    const double* height_offsets_px, const ctb_detector* det, const ctb_grid* grid,
                    int z_begin, int z_end, float load_scale, float* vol, int accumulate, void* stream);

/* ctb_backproject for callers that cannot allocate device memory. No
 * counterpart in the reference. Same arguments and result as ctb_backproject,
 * but the per-view geometry table that ctb_backproject allocates on the stream
 * at every call lives in a static 256 KB device array of the library instead,
 * so this call allocates nothing (the caller passes the filtered projections
 * and the volume, as before). At most CTB_NOALLOC_MAX_VIEWS views per call
 * (CTB_ERR_UNSUPPORTED beyond that); larger sets of views are split into
 * several calls with accumulate = 1. Arguments are checked as ctb_backproject
 * checks them. The first call on a device looks up the array's address, which
 * with lazy module loading also loads the library's kernels onto the device
 * (device memory taken once): make it at start-up, before any stream capture.
 * All calls share the array: calls that overlap on the GPU race, so serialise
 * them. */
#define CTB_NOALLOC_MAX_VIEWS 8192
int ctb_backproject_noalloc(const void* filtered, int store_type, int n_views, const double* angles_deg,
                            const double* height_offsets_px, const ctb_detector* det, const ctb_grid* grid,
                            int z_begin, int z_end, float load_scale, float* vol, int accumulate, void* stream);

/* Matched forward projector: the exact transpose of ctb_backproject with
 * load_scale = 1 (same bilinear footprint, U^2 weight, cylinder and bounds
 * masks). Input slab as ctb_backproject's output; output n_views x H x W FP32
 * projections (overwritten when accumulate == 0). No counterpart in the
 * reference (which has no forward model). */
int ctb_forward_project(const float* vol, const double* angles_deg, const double* height_offsets_px,
                        int n_views, const ctb_detector* det, const ctb_grid* grid, int z_begin,
                        int z_end, float* proj, int accumulate, void* stream);

/* Convert an X-fastest device slab (X x Y x Zs floats) into the requested
 * index order and byte order, into dst (device). Replaces the layout/byte-order
 * walk of Volume::saveToBinaryFile (Common/Volume.h:476-574) for one slab;
 * for Z_FASTEST the slab is written with row length zs (the caller scatters
 * slabs into the full z extent). */
int ctb_convert_layout(const float* src, int x, int y, int zs, int index_order, int byte_order,
                       void* dst, void* stream);

/* ------------------------------------------------------ batches of scans */

/* One scan of a batch. Device pointers are the caller's; host arrays are read
 * during ctb_batch_create only. */
typedef struct {
    const void* raw;                  /* device, n_views x H x W raw projections */
    int32_t raw_type;                 /* CTB_U8 / CTB_U16 / CTB_F32 */
    int32_t n_views;
    const double* angles_deg;         /* host, n_views (direction-corrected) */
    const double* height_offsets_px;  /* host, n_views (relative, pixels) or NULL */
    ctb_detector det;                 /* radius set (ctb_reference_grid) */
    ctb_grid grid;
    int32_t filter;                   /* CTB_RAMLAK / CTB_SHEPPLOGAN / CTB_HANN */
    int32_t pad;                      /* 1 or 2 */
    float* vol;                       /* device, X-fastest box volume (overwritten) */
} ctb_scan;

typedef struct ctb_batch ctb_batch;
typedef struct ctb_ctx ctb_ctx;   /* reconstruction context (facade layer below) */

/* Many independent scans of different detector, view and volume sizes
 * reconstructed together: per-scan filtering followed by ONE persistent
 * backprojection launch whose CTAs take (scan, tile) items from a device work
 * counter, the whole sequence captured once as a CUDA graph. Allocates the
 * filtered projections and view tables of every scan, picks the kernel's
 * z-voxels-per-thread with the built-in autotuner (timing both candidates on
 * this batch) and captures the graph. No counterpart in the reference, which
 * reconstructs one scan per process. */
int ctb_batch_create(ctb_batch** batch, int n_scans, const ctb_scan* scans, int store_type, void* stream);
int ctb_batch_run(ctb_batch* batch, void* stream);             /* replay the graph */
int ctb_batch_run_sequential(ctb_batch* batch, void* stream);  /* scan by scan, separate launches */
/* Autotuner outcome: chosen z voxels per thread, the timed candidates (ms, z = 32, 16 and 8; -1
 * where a candidate could not run) and how many scans the persistent kernel takes (scans with
 * voxels so coarse that a tile's footprint box exceeds the persistent kernel's shared-memory
 * budget get their own launch inside the same graph). */
int ctb_batch_tuning(const ctb_batch* batch, int* zc, double* ms_zc32, double* ms_zc16, double* ms_zc8,
                     int* n_persistent);
/* Every candidate the batch autotuner timed: z voxels per thread, views in
 * flight (projection boxes staged per CTA; 0 = the built-in choice) and ms;
 * *n receives the count, at most max entries are written. */
int ctb_batch_tuning_detail(const ctb_batch* batch, int max, int* zc, int* views_in_flight, double* ms, int* n);
void ctb_batch_destroy(ctb_batch* batch);
/* One call for a batch on a context: ctb_batch_create with the context's
 * precision (ctb_set_precision), ctb_batch_run, a synchronisation of the
 * stream and ctb_batch_destroy. For repeated batches of the same scans keep
 * a ctb_batch instead (the tuning and the graph capture are done once). */
int ctb_batch_reconstruct(ctb_ctx* ctx, int n_scans, const ctb_scan* scans, void* stream);

/* ------------------------------------------------------ facade layer */


/* Progress callback: stage 0 = loading, 1 = reconstruction, 2 = saving;
 * percent 0..100 (Ct/CtVolume.h:271-276 signals). Fires on the calling thread. */
typedef void (*ctb_progress_cb)(int stage, double percent, void* user);

int ctb_create(ctb_ctx** ctx);                 /* CtVolume() */
void ctb_destroy(ctb_ctx* ctx);
const char* ctb_last_error(const ctb_ctx* ctx);
const char* ctb_last_error_global(void);

/* sinogramFromImages (Ct/CtVolume.cpp:136-330): parse the CSV, decode and
 * validate every image (8/16-bit PGM or TIFF, 32-bit float TIFF), apply the
 * direction correction and relative height offsets, set the reference grid. */
int ctb_load_csv(ctb_ctx* ctx, const char* csv_path);

/* In-memory equivalent of ctb_load_csv for callers that already hold the
 * images: n_views raw images (raw_type) of width x height, host memory (pinned
 * or pageable), angles in degrees and height offsets in mm exactly as they
 * would appear in the CSV, plus the CSV header values. */
int ctb_set_projections(ctb_ctx* ctx, const void* host_images, int raw_type, int n_views, int width,
                        int height, const double* angles_deg, const double* height_offsets_mm,
                        double pixel_size, int ccw, double u_offset_mm, double fcd_mm,
                        double base_intensity);

int ctb_set_volume_bounds(ctb_ctx* ctx, float xmin, float xmax, float ymin, float ymax, float zmin,
                          float zmax);        /* setVolumeBounds */
int ctb_set_filter(ctb_ctx* ctx, int filter);             /* setFrequencyFilterType */
int ctb_set_skip_projections(ctb_ctx* ctx, unsigned skip);  /* setSkipProjections */
int ctb_set_device(ctb_ctx* ctx, int device);             /* setActiveCudaDevices({d}) */
/* setActiveCudaDevices (Ct/CtVolume.h:107, Ct/CtVolume.cpp:506-520): IDs at or
 * beyond the device count are dropped; with none left the selection is kept
 * and CTB_ERR_ARG returned. Each listed device reconstructs its own run of z
 * slices from all views; a device listed twice runs two workers. */
int ctb_set_devices(ctb_ctx* ctx, const int* device_ids, int n);
/* setGpuCoefficients (Ct/CtVolume.h:109-110): exponents of the multiprocessor
 * and memory-bandwidth shares in the per-device weights. */
int ctb_set_gpu_coefficients(ctb_ctx* ctx, double multiprocessor_coefficient, double bandwidth_coefficient);
/* getGpuWeights (Ct/CtVolume.cpp:1353-1381) for the given devices with the
 * context's coefficients; weights[n] sums to 1. */
int ctb_get_gpu_weights(ctb_ctx* ctx, const int* device_ids, int n, double* weights);
/* The same weights from given properties (no device query):
 * (sm_i/sum sm)^mp * (bw_i/sum bw)^bwc, normalised. */
int ctb_gpu_weights_from(const int* sm_count, const double* bandwidth, int n, double multiprocessor_coefficient,
                         double bandwidth_coefficient, double* weights);
/* Slice split of launchCudaThreads (Ct/CtVolume.cpp:1339-1344): device i gets
 * [begin[i], begin[i+1]) with round(weight_i * z) slices, clamped to z; the
 * last device also takes what rounding left over (the reference can leave
 * slices unassigned there). begin has n + 1 entries. */
int ctb_split_slices(const double* weights, int n, int z, int* begin);
int ctb_set_gpu_spare_memory(ctb_ctx* ctx, size_t megabytes);  /* setGpuSpareMemory */
/* Engine extensions (no reference counterpart). */
int ctb_set_precision(ctb_ctx* ctx, int store_type);      /* CTB_FP32 / FP16 / BF16 */
int ctb_set_pad(ctb_ctx* ctx, int pad);                   /* 1 (reference) or 2 */
/* Override the grid: x_size,y_size,z_size voxels of voxel_pitch detector
 * pixels, centred like the reference grid; bounds apply on top. 0 restores the
 * reference grid. */
int ctb_set_grid(ctb_ctx* ctx, int x_size, int y_size, int z_size, float voxel_pitch);
int ctb_set_slab_height(ctb_ctx* ctx, int slices);        /* 0 = automatic */

/* Autotuner of the backprojection (no reference counterpart; the reference
 * sizes its z-chunks by free memory only, getMaxChunkSize,
 * Ct/CtVolume.cpp:1385-1397). ctb_autotune times, on the loaded scan and box
 * and the first active device, the block tile height (z voxels per thread),
 * the views in flight (projection boxes staged per CTA) and the slab height
 * over an evenly spaced subset of the views, and keeps the fastest for every
 * later reconstruction of the same scan/box shape in this process (single
 * device; with several devices the built-in choices apply). With
 * ctb_set_autotune(ctx, 1) the first reconstruction of each shape tunes by
 * itself. 0 in a field means the built-in choice. */
typedef struct {
    int slab_slices;        /* z slices per backprojection launch */
    int zc;                 /* z voxels per thread */
    int views_in_flight;    /* projection boxes staged per CTA */
    double backproject_ms;  /* tuned device time of the whole backprojection (estimated from the subset) */
    int tuned;              /* 1 if a tuning exists for the context's current shape */
} ctb_tuning;
int ctb_set_autotune(ctb_ctx* ctx, int on);
int ctb_autotune(ctb_ctx* ctx, ctb_tuning* out);
int ctb_get_tuning(const ctb_ctx* ctx, ctb_tuning* out);
int ctb_set_progress_callback(ctb_ctx* ctx, ctb_progress_cb cb, void* user);

/* setUseCuda (Ct/CtVolume.h:104): 0 is refused (CTB_ERR_UNSUPPORTED), the
 * engine reconstructs on the GPU only. setUseCpuPreprocessing (:111) is
 * accepted and has no effect: preprocessing always runs on the GPU.
 * setEmitSignals (:100): 0 silences the progress and preview callbacks, as
 * the reference silences its Qt signals. */
int ctb_set_use_cuda(ctb_ctx* ctx, int use_cuda);
int ctb_set_use_cpu_preprocessing(ctb_ctx* ctx, int value);
int ctb_set_emit_signals(ctb_ctx* ctx, int value);

/* Getters (Ct/CtVolume.h:69-94). */
int ctb_get_detector(const ctb_ctx* ctx, ctb_detector* det);
int ctb_get_grid(const ctb_ctx* ctx, ctb_grid* grid);
int ctb_get_volume_size(const ctb_ctx* ctx, int* x, int* y, int* z); /* getX/Y/ZSize */
int ctb_get_sinogram_size(const ctb_ctx* ctx, int* n);
double ctb_get_pixel_size(const ctb_ctx* ctx);

/* reconstructVolume (Ct/CtVolume.cpp:543-632). The volume stays in host
 * memory owned by the context (X-fastest) until the next call. */
int ctb_reconstruct(ctb_ctx* ctx);

/* Reconstruct straight into a caller buffer of x*y*z floats in index_order
 * (host memory, pinned buffers are used without staging). */
int ctb_reconstruct_into(ctb_ctx* ctx, float* host_volume, int index_order);

/* Copy the last reconstructed volume into a caller buffer in index_order. */
int ctb_get_volume(const ctb_ctx* ctx, float* host_volume, int index_order);

/* saveVolumeToBinaryFile (Ct/CtVolume.cpp:634-721): <base>.txt info file,
 * <base>.vgi header, raw float32 in index_order / byte_order. */
int ctb_save_volume(ctb_ctx* ctx, const char* path, int index_order, int byte_order);

/* The matched projector pair on the context's scan (detector, views, height
 * offsets, all views regardless of the skip setting) and box (grid and
 * bounds), host memory in and out, on the first active device; the volume
 * moves through the device one z-slab at a time, nothing else is kept.
 * Volumes are X-fastest box volumes (x*y*z floats), projections n_views x H x
 * W floats. No counterpart in the reference (which has no forward model).
 *   ctb_forward:  projections = A volume (the forward projector, fp_kernel)
 *   ctb_backward: volume = A^T projections (the backprojector, load scale 1,
 *                 unfiltered: the exact transpose of A)
 *   ctb_gradient: loss = ||A volume - data||^2 and gradient = 2 A^T (A volume
 *                 - data), with A volume accumulated slab by slab and the
 *                 adjoint recomputed per slab (no stored intermediates). */
int ctb_forward(ctb_ctx* ctx, const float* host_volume, float* host_projections);
int ctb_backward(ctb_ctx* ctx, const float* host_projections, float* host_volume);
int ctb_gradient(ctb_ctx* ctx, const float* host_volume, const float* host_data, float* host_gradient,
                 double* loss);

/* stop() (Ct/CtVolume.cpp:723-726): thread-safe, polled per slab / view group. */
void ctb_stop(ctb_ctx* ctx);

/* Stage timings of the last ctb_reconstruct* call (seconds, CUDA events and
 * steady clock). */
typedef struct {
    double upload_s;        /* host->device copies not hidden behind filtering */
    double filter_s;        /* preprocessing + ramp filter kernels */
    double backproject_s;   /* backprojection kernels */
    double download_s;      /* device->host copies not hidden behind backprojection */
    double total_s;         /* wall time of the whole call */
    double voxel_views;     /* x*y*z*views processed */
    double h2d_bytes;       /* projection bytes copied host->device (each device
                               copies only the detector rows its slices reach) */
    double d2h_bytes;       /* volume bytes copied device->host */
} ctb_timings;
int ctb_get_timings(const ctb_ctx* ctx, ctb_timings* t);

/* getSkipProjections, getUseCuda, getUseCpuPreprocessing, getEmitSignals,
 * getGpuSpareMemory, getMultiprocessorCoefficient,
 * getMemoryBandwidthCoefficient, getActiveCudaDevices (Ct/CtVolume.h:86-95). */
typedef struct {
    unsigned skip_projections;
    int use_cuda;                 /* always 1 */
    int use_cpu_preprocessing;
    int emit_signals;
    size_t gpu_spare_memory_mb;
    double multiprocessor_coefficient;
    double memory_bandwidth_coefficient;
    int n_devices;                /* active devices (the first 16 listed) */
    int devices[16];
} ctb_settings;
int ctb_get_settings(const ctb_ctx* ctx, ctb_settings* s);
/* getRequiredMemoryUpperBound (Ct/CtVolume.cpp:469-481): bytes of host memory
 * the reference would need: the float volume plus three float images per
 * active device. */
int ctb_get_required_memory(const ctb_ctx* ctx, size_t* bytes);
/* getProjectionAt (Ct/CtVolume.cpp:332-341): the view's angle (degrees,
 * direction-corrected), its relative height offset (pixels) and, if image is
 * not NULL, width*height floats: the raw image scaled as the reference's
 * convertTo32bit and normalised by the scan's minimum and maximum sample
 * (divided by 2^8 for 8-bit scans, 2^16 otherwise, as the reference does).
 * CTB_ERR_ARG for an index out of bounds. */
int ctb_get_projection(ctb_ctx* ctx, int index, float* image, double* angle_deg, double* height_offset_px);

/* --------------------------------------------------- device waits */

/* Every wait inside the backprojection kernels (for a box load, for a free
 * buffer) is bounded; a wait that gives up makes its tile stop, leaves that
 * part of the volume incomplete and is counted here. Returns the count on
 * `device` since the last reset (reset != 0 clears it). ctb_reconstruct checks
 * it and fails with CTB_ERR_TIMEOUT; callers of ctb_backproject check it after
 * synchronising. No reference counterpart. */
int ctb_device_wait_timeouts(int device, unsigned* count, int reset);
/* Diagnostic of that path: one warp waits on a barrier that can never
 * complete, with at most `limit` tries, and must give up: returns
 * CTB_ERR_TIMEOUT (and adds 1 to the count) with the device still usable. */
int ctb_diag_bounded_wait(int device, unsigned limit);

/* Diagnostic of the backprojector's overflow path: from the next launch on,
 * the shared-memory backprojector (single scans and batches) reads every view
 * whose index is a multiple of `every` through global memory, the path taken by
 * views whose footprint does not fit the staged box. The result must not
 * change; 0 turns it off. Process-wide. No reference counterpart. */
void ctb_diag_force_overflow(int every);

/* Diagnostic of the facade's allocation failure path: from now on the nth
 * device or host buffer the facade allocates (1 = the next one) fails as if
 * the memory were exhausted, so ctb_reconstruct* returns CTB_ERR_ALLOC (the
 * reference's VRAM / RAM failure branches, Ct/CtVolume.cpp:554-557,
 * :1133-1147). 0 turns it off. Process-wide; no GPU fault is involved. */
void ctb_diag_fail_allocation(long nth);

/* Bounds-checked build (libctb_checked.so, compiled with CTB_BOUNDS_CHECK):
 * the backprojection kernels check every texel fetch against the buffer it
 * reads (the staged box in shared memory, or the projections in global
 * memory), skip a fetch out of range and record it: *violations counts them
 * on `device` since the last reset and *first encodes the first one
 * (site << 56 | index). *checked_build is 0 in the normal library, whose
 * kernels carry no checks (the counts are then 0). reset != 0 clears them.
 * No reference counterpart (compute-sanitizer's memcheck is not used). */
int ctb_diag_bounds_status(int device, int* checked_build, unsigned* violations, unsigned long long* first,
                           int reset);

/* ------------------------------------------------------ projection images */

/* Projection::getImage (Ct/CtVolume.cpp:20-33): decode one projection image
 * the way cv::imread(IMREAD_GRAYSCALE | IMREAD_ANYDEPTH) does for the formats
 * read here: binary PGM (8/16-bit), TIFF strips (8/16-bit integer, 32-bit
 * float; uncompressed, LZW, Deflate or PackBits, with or without horizontal
 * differencing; gray, or RGB/RGBA converted to gray), PNG (8/16-bit gray,
 * gray + alpha, RGB, RGBA). With out == NULL only the size and the sample
 * type (CTB_U8 / CTB_U16 / CTB_F32) are returned; otherwise out receives
 * width * height samples, row-major. */
int ctb_read_image(const char* path, int* width, int* height, int* raw_type, void* out);

/* ------------------------------------------------------ volume files */

/* DataType, Common/types.h:27-36 (same order). */
enum { CTB_DT_FLOAT32 = 0, CTB_DT_DOUBLE64, CTB_DT_UINT8, CTB_DT_INT8, CTB_DT_UINT16, CTB_DT_INT16,
       CTB_DT_UINT32, CTB_DT_INT32 };

/* Axis, Common/Volume.h:18-22. */
enum { CTB_AXIS_X = 0, CTB_AXIS_Y = 1, CTB_AXIS_Z = 2 };

/* Read the dimensions, byte order and index order from a reconstruction's
 * .txt info file, as the viewer does (CtViewer/ViewerInterface.cpp:486-523):
 * lines containing "X size:", "Y size:", "Z size:", "Byte order:" ("Big
 * endian") and "Index order:" ("X fastest"), case-insensitive. CTB_ERR_ARG if
 * any of the five is missing. */
int ctb_read_volume_info(const char* txt_path, int* x, int* y, int* z, int* index_order, int* byte_order);

/* Volume<float>::loadFromBinaryFile (Common/Volume.h:336-472): read x*y*z
 * samples of data_type after header_offset bytes in index_order / byte_order,
 * optionally mirrored per axis, into an X-fastest float volume. */
int ctb_load_volume(const char* raw_path, int x, int y, int z, int index_order, int byte_order, int data_type,
                    size_t header_offset, int mirror_x, int mirror_y, int mirror_z, float* out_xfastest);

/* Volume::getVolumeCrossSection with the left-handed orientation CtVolume
 * uses (Common/Volume.h:577-648, Ct/CtVolume.cpp:391-393) of the last
 * reconstructed volume: axis X -> Z rows x Y columns, Y -> Z x X, Z -> X x Y.
 * out holds rows*cols floats (row-major); rows/cols are returned. */
int ctb_get_cross_section(const ctb_ctx* ctx, int axis, int index, float* out, int* rows, int* cols);

/* Cross-section settings (setCrossSectionAxis / setCrossSectionIndex,
 * Ct/CtVolume.cpp:395-429): changing the axis moves the index to the middle
 * of the box along it; an index outside the box is ignored; loading a scan
 * and changing the bounds re-centre or clamp it as the reference does
 * (:317-326, :1411-1417). */
int ctb_set_cross_section_axis(ctb_ctx* ctx, int axis);
int ctb_set_cross_section_index(ctb_ctx* ctx, int index);
/* getCrossSectionAxis / Index / Size (size = box extent along the axis). */
int ctb_get_cross_section_info(const ctb_ctx* ctx, int* axis, int* index, int* size);
/* Progress previews (reconstructionProgress / reconstructionFinished with the
 * cross section, Ct/CtVolume.cpp:952, :1479-1483, :615): while
 * ctb_reconstruct fills the context's own volume, cb receives the completion
 * percentage and the current cross section (rows x cols floats, library-owned,
 * valid during the call) after every downloaded z-slab, and once more at
 * 100 % with the finished volume. Called from the reconstructing thread(s),
 * one call at a time. */
typedef void (*ctb_preview_cb)(double percent, const float* section, int rows, int cols, void* user);
int ctb_set_preview_callback(ctb_ctx* ctx, ctb_preview_cb cb, void* user);

/* ------------------------------------------------------ synthetic data */

/* Analytic line integrals of a sum of ellipsoids (test phantoms), one value
 * per detector pixel, FP64 on the device. ellipsoids: n x 16 doubles
 * {cx,cy,cz, a,b,c, R00..R22 (row-major rotation, body->world), density} in
 * mm; geometry as the reference model with source-axis distance fcd_mm and
 * detector pitch pixel_mm at the axis. out: device, n_views x H x W doubles. */
int ctb_phantom_project(const double* ellipsoids_dev, int n_ellipsoids, const double* angles_deg,
                        const double* height_offsets_mm, int n_views, int width, int height,
                        double pixel_mm, double fcd_mm, double u_offset_mm, double* out_dev,
                        void* stream);

#ifdef __cplusplus
}
#endif

#endif /* CTB_H */
