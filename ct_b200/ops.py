"""Operator layer over device memory (torch tensors as plain device buffers).

These mirror the reference's kernel API (Ct/cuda_ct.h:18-69): callers own the
device memory and pass a stream; the functions enqueue work and return.
torch is only used for allocation, streams and pointers.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib as L
from ._lib import check, lib

STORE_DTYPES = {}
RAW_CODES = {}


def _torch():
    import torch
    if not STORE_DTYPES:
        STORE_DTYPES.update({L.FP32: torch.float32, L.FP16: torch.float16, L.BF16: torch.bfloat16})
        RAW_CODES.update({torch.uint8: L.U8, torch.uint16: L.U16, torch.float32: L.F32})
    return torch


def _stream(stream):
    torch = _torch()
    if stream is None:
        stream = torch.cuda.current_stream()
    return ctypes.c_void_p(stream.cuda_stream)


def detector(width, height, fcd, u_offset=0.0, base_intensity=1.0, rel=None):
    """Detector record plus the reference grid (radius, grid rule, bounds)."""
    d = L.Detector(width, height, fcd, u_offset, base_intensity, 0.0)
    g = L.Grid()
    r = None if rel is None else (ctypes.c_float * 6)(*rel)
    check(lib().ctb_reference_grid(ctypes.byref(d), r, ctypes.byref(g)))
    return d, g


def row_band(d: L.Detector, g: L.Grid, z_begin: int, z_end: int, heights_px=None):
    """Detector rows (r_lo, rows) that box slices [z_begin, z_end) reach (host only)."""
    h = None if heights_px is None else np.ascontiguousarray(heights_px, dtype=np.float64)
    n = 0 if h is None else len(h)
    r_lo, rows = ctypes.c_int(), ctypes.c_int()
    check(lib().ctb_row_band(ctypes.byref(d), ctypes.byref(g), int(z_begin), int(z_end),
                             None if h is None else h.ctypes.data, n, ctypes.byref(r_lo), ctypes.byref(rows)))
    return r_lo.value, rows.value


def custom_grid(d: L.Detector, size, voxel_pitch, box=None) -> L.Grid:
    x, y, z = size
    if box is None:
        box = (0, x, 0, y, 0, z)
    return L.Grid(x, y, z, *box, voxel_pitch)


def filter_projections(raw, det: L.Detector, filter_type=L.RAMLAK, pad=1, store=L.FP32, store_scale=1.0,
                       out=None, stream=None):
    """raw: (V, H, W) uint8/uint16/float32 CUDA tensor -> filtered (V, H, W) in the storage dtype."""
    torch = _torch()
    assert raw.is_cuda and raw.is_contiguous()
    V = raw.shape[0]
    if out is None:
        out = torch.empty(raw.shape, dtype=STORE_DTYPES[store], device=raw.device)
    check(lib().ctb_filter_projections(ctypes.c_void_p(raw.data_ptr()), RAW_CODES[raw.dtype], V, ctypes.byref(det),
                                       filter_type, pad, ctypes.c_void_p(out.data_ptr()), store, store_scale,
                                       _stream(stream)))
    return out


def backproject(filtered, angles_deg, heights_px, det: L.Detector, grid: L.Grid, z_begin=0, z_end=None,
                load_scale=1.0, out=None, accumulate=False, stream=None):
    """Filtered projections (V, H, W) -> X-fastest slab (Zs, Y, X) float32."""
    torch = _torch()
    store = {v: k for k, v in STORE_DTYPES.items()}[filtered.dtype]
    X, Y, Z = grid.box
    if z_end is None:
        z_end = Z
    if out is None:
        out = torch.empty((z_end - z_begin, Y, X), dtype=torch.float32, device=filtered.device)
    a = np.ascontiguousarray(angles_deg, np.float64)
    h = np.ascontiguousarray(heights_px if heights_px is not None else np.zeros_like(a), np.float64)
    check(lib().ctb_backproject(ctypes.c_void_p(filtered.data_ptr()), store, len(a), a.ctypes.data, h.ctypes.data,
                                ctypes.byref(det), ctypes.byref(grid), z_begin, z_end, load_scale,
                                ctypes.c_void_p(out.data_ptr()), int(accumulate), _stream(stream)))
    return out


def forward_project(vol, angles_deg, heights_px, det: L.Detector, grid: L.Grid, z_begin=0, z_end=None, out=None,
                    accumulate=False, stream=None):
    """X-fastest slab (Zs, Y, X) float32 -> projections (V, H, W) float32 (transpose of backproject)."""
    torch = _torch()
    X, Y, Z = grid.box
    if z_end is None:
        z_end = Z
    a = np.ascontiguousarray(angles_deg, np.float64)
    h = np.ascontiguousarray(heights_px if heights_px is not None else np.zeros_like(a), np.float64)
    if out is None:
        out = torch.empty((len(a), det.height, det.width), dtype=torch.float32, device=vol.device)
    check(lib().ctb_forward_project(ctypes.c_void_p(vol.data_ptr()), a.ctypes.data, h.ctypes.data, len(a),
                                    ctypes.byref(det), ctypes.byref(grid), z_begin, z_end,
                                    ctypes.c_void_p(out.data_ptr()), int(accumulate), _stream(stream)))
    return out


def convert_layout(src, index_order, byte_order=L.LITTLE_ENDIAN, out=None, stream=None):
    """X-fastest slab (Zs, Y, X) -> same bytes in index_order / byte_order (returned as int32 view if swapped)."""
    torch = _torch()
    zs, y, x = src.shape
    if out is None:
        out = torch.empty(src.numel(), dtype=torch.float32, device=src.device)
    check(lib().ctb_convert_layout(ctypes.c_void_p(src.data_ptr()), x, y, zs, index_order, byte_order,
                                   ctypes.c_void_p(out.data_ptr()), _stream(stream)))
    return out


def phantom_project(ellipsoids, angles_deg, heights_mm, width, height, pixel_mm, fcd_mm, u_offset_mm=0.0,
                    out=None, device="cuda", stream=None):
    """Analytic line integrals (FP64, device) of an (n, 16) ellipsoid table -> (V, H, W) float64."""
    torch = _torch()
    e = torch.as_tensor(np.ascontiguousarray(ellipsoids, np.float64), device=device)
    a = np.ascontiguousarray(angles_deg, np.float64)
    h = None if heights_mm is None else np.ascontiguousarray(heights_mm, np.float64)
    if out is None:
        out = torch.empty((len(a), height, width), dtype=torch.float64, device=device)
    check(lib().ctb_phantom_project(ctypes.c_void_p(e.data_ptr()), e.shape[0], a.ctypes.data,
                                    None if h is None else h.ctypes.data, len(a), width, height, pixel_mm, fcd_mm,
                                    u_offset_mm, ctypes.c_void_p(out.data_ptr()), _stream(stream)))
    return out


class Batch:
    """Many scans of different sizes reconstructed by one persistent
    backprojection launch under a captured CUDA graph (ctb_batch_*).

    scans: list of dicts with raw (CUDA uint8/uint16/float32 tensor V x H x W),
    angles_deg, heights_px (or None), det, grid, filter, pad, vol (CUDA float32
    tensor Z x Y x X, overwritten)."""

    def __init__(self, scans, store=L.FP32, stream=None):
        self._keep = []
        arr = (L.Scan * len(scans))()
        for i, sc in enumerate(scans):
            a = np.ascontiguousarray(sc["angles_deg"], np.float64)
            h = None if sc.get("heights_px") is None else np.ascontiguousarray(sc["heights_px"], np.float64)
            self._keep += [a, h, sc["raw"], sc["vol"]]
            arr[i] = L.Scan(ctypes.c_void_p(sc["raw"].data_ptr()), RAW_CODES_FN()[sc["raw"].dtype], len(a),
                            a.ctypes.data, None if h is None else h.ctypes.data, sc["det"], sc["grid"],
                            sc.get("filter", L.RAMLAK), sc.get("pad", 1), ctypes.c_void_p(sc["vol"].data_ptr()))
        self._h = ctypes.c_void_p()
        check(lib().ctb_batch_create(ctypes.byref(self._h), len(scans), arr, store, _stream(stream)))

    def run(self, stream=None):
        check(lib().ctb_batch_run(self._h, _stream(stream)))

    def run_sequential(self, stream=None):
        check(lib().ctb_batch_run_sequential(self._h, _stream(stream)))

    def tuning(self):
        zc, n = ctypes.c_int(), ctypes.c_int()
        t32, t16, t8 = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        check(lib().ctb_batch_tuning(self._h, ctypes.byref(zc), ctypes.byref(t32), ctypes.byref(t16), ctypes.byref(t8),
                                     ctypes.byref(n)))
        return {"zc": zc.value, "ms_zc32": t32.value, "ms_zc16": t16.value, "ms_zc8": t8.value,
                "persistent_scans": n.value}

    def tuning_detail(self):
        """Every candidate the autotuner timed: [(z voxels per thread, views in flight (0: built-in), ms)]."""
        n = ctypes.c_int()
        check(lib().ctb_batch_tuning_detail(self._h, 0, None, None, None, ctypes.byref(n)))
        zc = (ctypes.c_int * n.value)()
        nb = (ctypes.c_int * n.value)()
        ms = (ctypes.c_double * n.value)()
        check(lib().ctb_batch_tuning_detail(self._h, n.value, zc, nb, ms, ctypes.byref(n)))
        return [(zc[i], nb[i], ms[i]) for i in range(n.value)]

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and L._lib is not None:
            L._lib.ctb_batch_destroy(h)
            self._h = None


def batch_reconstruct(scans, store=L.FP32, stream=None):
    """One-shot batch (ctb_batch_reconstruct on a context of the given
    precision): create, run, synchronise and release. Same scan dicts as Batch."""
    from .ctvolume import CtVolume
    keep = []
    arr = (L.Scan * len(scans))()
    for i, sc in enumerate(scans):
        a = np.ascontiguousarray(sc["angles_deg"], np.float64)
        h = None if sc.get("heights_px") is None else np.ascontiguousarray(sc["heights_px"], np.float64)
        keep += [a, h]
        arr[i] = L.Scan(ctypes.c_void_p(sc["raw"].data_ptr()), RAW_CODES_FN()[sc["raw"].dtype], len(a),
                        a.ctypes.data, None if h is None else h.ctypes.data, sc["det"], sc["grid"],
                        sc.get("filter", L.RAMLAK), sc.get("pad", 1), ctypes.c_void_p(sc["vol"].data_ptr()))
    ctx = CtVolume()
    ctx.setPrecision(store)
    ctx._ck(lib().ctb_batch_reconstruct(ctx._ctx, len(scans), arr, _stream(stream)))


def RAW_CODES_FN():
    _torch()
    return RAW_CODES
