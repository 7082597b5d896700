"""ctypes declarations of libctb (include/ctb.h).

The library is required: importing a function that needs it raises when
libctb.so is missing instead of falling back to anything else.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# CTB_LIBRARY=checked loads the bounds-checked build (libctb_checked.so,
# kernels compiled with CTB_BOUNDS_CHECK) instead of libctb.so.
LIB_PATH = os.path.join(HERE, "libctb_checked.so" if os.environ.get("CTB_LIBRARY") == "checked" else "libctb.so")

# status codes
CTB_OK, CTB_ERR_ARG, CTB_ERR_IO, CTB_ERR_CSV, CTB_ERR_IMAGE, CTB_ERR_ALLOC, CTB_ERR_CUDA, CTB_ERR_TIMEOUT, \
    CTB_INTERRUPTED, CTB_ERR_UNSUPPORTED = range(10)
STATUS_NAMES = {0: "OK", 1: "ERR_ARG", 2: "ERR_IO", 3: "ERR_CSV", 4: "ERR_IMAGE", 5: "ERR_ALLOC", 6: "ERR_CUDA",
                7: "ERR_TIMEOUT", 8: "INTERRUPTED", 9: "ERR_UNSUPPORTED"}
RAMLAK, SHEPPLOGAN, HANN = 0, 1, 2
X_FASTEST, Z_FASTEST = 0, 1
AXIS_X, AXIS_Y, AXIS_Z = 0, 1, 2
LITTLE_ENDIAN, BIG_ENDIAN = 0, 1
FP32, FP16, BF16 = 0, 1, 2
U8, U16, F32 = 8, 16, 32


class Detector(ctypes.Structure):
    _fields_ = [("width", ctypes.c_int32), ("height", ctypes.c_int32), ("fcd", ctypes.c_float),
                ("u_offset", ctypes.c_float), ("base_intensity", ctypes.c_float), ("radius", ctypes.c_float)]


class Grid(ctypes.Structure):
    _fields_ = [("x_size", ctypes.c_int32), ("y_size", ctypes.c_int32), ("z_size", ctypes.c_int32),
                ("x_from", ctypes.c_int32), ("x_to", ctypes.c_int32), ("y_from", ctypes.c_int32),
                ("y_to", ctypes.c_int32), ("z_from", ctypes.c_int32), ("z_to", ctypes.c_int32),
                ("voxel_pitch", ctypes.c_float)]

    @property
    def box(self):
        return (self.x_to - self.x_from, self.y_to - self.y_from, self.z_to - self.z_from)


class Scan(ctypes.Structure):
    _fields_ = [("raw", ctypes.c_void_p), ("raw_type", ctypes.c_int32), ("n_views", ctypes.c_int32),
                ("angles_deg", ctypes.c_void_p), ("height_offsets_px", ctypes.c_void_p), ("det", Detector),
                ("grid", Grid), ("filter", ctypes.c_int32), ("pad", ctypes.c_int32), ("vol", ctypes.c_void_p)]


class Settings(ctypes.Structure):
    _fields_ = [("skip_projections", ctypes.c_uint), ("use_cuda", ctypes.c_int),
                ("use_cpu_preprocessing", ctypes.c_int), ("emit_signals", ctypes.c_int),
                ("gpu_spare_memory_mb", ctypes.c_size_t), ("multiprocessor_coefficient", ctypes.c_double),
                ("memory_bandwidth_coefficient", ctypes.c_double), ("n_devices", ctypes.c_int),
                ("devices", ctypes.c_int * 16)]


class Timings(ctypes.Structure):
    _fields_ = [("upload_s", ctypes.c_double), ("filter_s", ctypes.c_double), ("backproject_s", ctypes.c_double),
                ("download_s", ctypes.c_double), ("total_s", ctypes.c_double), ("voxel_views", ctypes.c_double),
                ("h2d_bytes", ctypes.c_double), ("d2h_bytes", ctypes.c_double)]


class Tuning(ctypes.Structure):
    _fields_ = [("slab_slices", ctypes.c_int), ("zc", ctypes.c_int), ("views_in_flight", ctypes.c_int),
                ("backproject_ms", ctypes.c_double), ("tuned", ctypes.c_int)]


PROGRESS_CB = ctypes.CFUNCTYPE(None, ctypes.c_int, ctypes.c_double, ctypes.c_void_p)
PREVIEW_CB = ctypes.CFUNCTYPE(None, ctypes.c_double, ctypes.POINTER(ctypes.c_float), ctypes.c_int, ctypes.c_int,
                              ctypes.c_void_p)

# name -> (restype, argtypes)
P, I, F, D, Z = ctypes.c_void_p, ctypes.c_int, ctypes.c_float, ctypes.c_double, ctypes.c_size_t
SIGNATURES = {
    "ctb_device_count": (I, [P]),
    "ctb_device_name": (I, [I, ctypes.c_char_p, Z]),
    "ctb_free_memory": (I, [I, P, P]),
    "ctb_reference_grid": (I, [P, P, P]),
    "ctb_row_band": (I, [P, P, I, I, P, I, P, P]),
    "ctb_filter_projections": (I, [P, I, I, P, I, I, P, I, F, P]),
    "ctb_backproject": (I, [P, I, I, P, P, P, P, I, I, F, P, I, P]),
    "ctb_backproject_noalloc": (I, [P, I, I, P, P, P, P, I, I, F, P, I, P]),
    "ctb_forward_project": (I, [P, P, P, I, P, P, I, I, P, I, P]),
    "ctb_diag_force_overflow": (None, [I]),
    "ctb_diag_fail_allocation": (None, [ctypes.c_long]),
    "ctb_diag_bounds_status": (I, [I, P, P, P, I]),
    "ctb_forward": (I, [P, P, P]),
    "ctb_backward": (I, [P, P, P]),
    "ctb_gradient": (I, [P, P, P, P, P]),
    "ctb_batch_reconstruct": (I, [P, I, P, P]),
    "ctb_batch_tuning_detail": (I, [P, I, P, P, P, P]),
    "ctb_set_autotune": (I, [P, I]),
    "ctb_autotune": (I, [P, P]),
    "ctb_get_tuning": (I, [P, P]),
    "ctb_convert_layout": (I, [P, I, I, I, I, I, P, P]),
    "ctb_create": (I, [P]),
    "ctb_destroy": (None, [P]),
    "ctb_last_error": (ctypes.c_char_p, [P]),
    "ctb_last_error_global": (ctypes.c_char_p, []),
    "ctb_load_csv": (I, [P, ctypes.c_char_p]),
    "ctb_set_projections": (I, [P, P, I, I, I, I, P, P, D, I, D, D, D]),
    "ctb_set_volume_bounds": (I, [P, F, F, F, F, F, F]),
    "ctb_set_filter": (I, [P, I]),
    "ctb_set_skip_projections": (I, [P, ctypes.c_uint]),
    "ctb_set_device": (I, [P, I]),
    "ctb_set_gpu_spare_memory": (I, [P, Z]),
    "ctb_set_devices": (I, [P, P, I]),
    "ctb_set_gpu_coefficients": (I, [P, D, D]),
    "ctb_get_gpu_weights": (I, [P, P, I, P]),
    "ctb_gpu_weights_from": (I, [P, P, I, D, D, P]),
    "ctb_split_slices": (I, [P, I, I, P]),
    "ctb_set_precision": (I, [P, I]),
    "ctb_set_pad": (I, [P, I]),
    "ctb_set_grid": (I, [P, I, I, I, F]),
    "ctb_set_slab_height": (I, [P, I]),
    "ctb_set_progress_callback": (I, [P, PROGRESS_CB, P]),
    "ctb_get_detector": (I, [P, P]),
    "ctb_get_grid": (I, [P, P]),
    "ctb_get_volume_size": (I, [P, P, P, P]),
    "ctb_get_sinogram_size": (I, [P, P]),
    "ctb_get_pixel_size": (D, [P]),
    "ctb_reconstruct": (I, [P]),
    "ctb_reconstruct_into": (I, [P, P, I]),
    "ctb_get_volume": (I, [P, P, I]),
    "ctb_save_volume": (I, [P, ctypes.c_char_p, I, I]),
    "ctb_stop": (None, [P]),
    "ctb_get_timings": (I, [P, P]),
    "ctb_phantom_project": (I, [P, I, P, P, I, I, I, D, D, D, P, P]),
    "ctb_read_volume_info": (I, [ctypes.c_char_p, P, P, P, P, P]),
    "ctb_load_volume": (I, [ctypes.c_char_p, I, I, I, I, I, I, Z, I, I, I, P]),
    "ctb_get_cross_section": (I, [P, I, I, P, P, P]),
    "ctb_set_cross_section_axis": (I, [P, I]),
    "ctb_set_cross_section_index": (I, [P, I]),
    "ctb_get_cross_section_info": (I, [P, P, P, P]),
    "ctb_set_preview_callback": (I, [P, PREVIEW_CB, P]),
    "ctb_batch_create": (I, [P, I, P, I, P]),
    "ctb_batch_run": (I, [P, P]),
    "ctb_batch_run_sequential": (I, [P, P]),
    "ctb_batch_tuning": (I, [P, P, P, P, P, P]),
    "ctb_device_wait_timeouts": (I, [I, P, I]),
    "ctb_read_image": (I, [ctypes.c_char_p, P, P, P, P]),
    "ctb_set_use_cuda": (I, [P, I]),
    "ctb_set_use_cpu_preprocessing": (I, [P, I]),
    "ctb_set_emit_signals": (I, [P, I]),
    "ctb_get_settings": (I, [P, P]),
    "ctb_get_required_memory": (I, [P, P]),
    "ctb_get_projection": (I, [P, I, P, P, P]),
    "ctb_diag_bounded_wait": (I, [I, ctypes.c_uint]),
    "ctb_batch_destroy": (None, [P]),
}

_lib = None


class CtbError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status
        self.message = message


def lib():
    """Load libctb.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{os.path.basename(LIB_PATH)} not found at {LIB_PATH}; build it with "
                               "`python -m ct_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status: int, ctx=None):
    if status != CTB_OK:
        if ctx is not None:
            msg = lib().ctb_last_error(ctx)
        else:
            msg = lib().ctb_last_error_global()
        raise CtbError(status, (msg or b"").decode(errors="replace"))
    return status
