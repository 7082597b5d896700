"""CtVolume: the reference's reconstruction facade (Ct/CtVolume.h:57-278) over libctb.

Method names and argument meanings follow ct::CtVolume; errors raise CtbError
carrying the message the reference would have emitted with
CompletionStatus::error (user interruption raises with status INTERRUPTED).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib as L
from ._lib import check, lib

FILTER_NAMES = {"ramlak": L.RAMLAK, "shepplogan": L.SHEPPLOGAN, "hann": L.HANN}
RAW_TYPES = {np.dtype(np.uint8): L.U8, np.dtype(np.uint16): L.U16, np.dtype(np.float32): L.F32}


class CtVolume:
    def __init__(self, csv_file: str | None = None):
        self._ctx = ctypes.c_void_p()
        check(lib().ctb_create(ctypes.byref(self._ctx)))
        self._keep = None
        self._cb = None
        self._pcb = None
        if csv_file is not None:
            self.sinogramFromImages(csv_file)

    def __del__(self):
        ctx = getattr(self, "_ctx", None)
        if ctx is not None and ctx.value and L._lib is not None:
            L._lib.ctb_destroy(ctx)
            self._ctx = None

    def _ck(self, status):
        return check(status, self._ctx)

    # ---------------------------------------------------------------- input
    def sinogramFromImages(self, csv_file: str) -> bool:
        self._ck(lib().ctb_load_csv(self._ctx, str(csv_file).encode()))
        return True

    def setProjections(self, images: np.ndarray, angles_deg, height_offsets_mm=None, *, pixel_size: float,
                       rotation: str = "ccw", u_offset_mm: float = 0.0, fcd_mm: float, base_intensity: float = 1.0):
        """In-memory equivalent of sinogramFromImages: images (V, H, W) uint8/uint16/float32 in host memory."""
        images = np.ascontiguousarray(images)
        V, H, W = images.shape
        a = np.ascontiguousarray(angles_deg, np.float64)
        h = None if height_offsets_mm is None else np.ascontiguousarray(height_offsets_mm, np.float64)
        ccw = {"ccw": 1, "cw": 0}.get(rotation, -1)
        self._ck(lib().ctb_set_projections(self._ctx, images.ctypes.data, RAW_TYPES[images.dtype], V, W, H,
                                           a.ctypes.data, None if h is None else h.ctypes.data, pixel_size, ccw,
                                           u_offset_mm, fcd_mm, base_intensity))
        self._keep = images  # the context reads the images during reconstruction

    def setProjectionsPointer(self, ptr: int, raw_type: int, n_views: int, width: int, height: int, angles_deg,
                              height_offsets_mm=None, *, pixel_size: float, rotation: str = "ccw",
                              u_offset_mm: float = 0.0, fcd_mm: float, base_intensity: float = 1.0, keep=None):
        """Like setProjections for a raw host pointer (e.g. a pinned torch tensor's data_ptr())."""
        a = np.ascontiguousarray(angles_deg, np.float64)
        h = None if height_offsets_mm is None else np.ascontiguousarray(height_offsets_mm, np.float64)
        ccw = {"ccw": 1, "cw": 0}.get(rotation, -1)
        self._ck(lib().ctb_set_projections(self._ctx, ptr, raw_type, n_views, width, height, a.ctypes.data,
                                           None if h is None else h.ctypes.data, pixel_size, ccw, u_offset_mm,
                                           fcd_mm, base_intensity))
        self._keep = keep

    # ------------------------------------------------------------- settings
    def setVolumeBounds(self, xFrom, xTo, yFrom, yTo, zFrom, zTo):
        self._ck(lib().ctb_set_volume_bounds(self._ctx, xFrom, xTo, yFrom, yTo, zFrom, zTo))

    def setFrequencyFilterType(self, filter_type):
        if isinstance(filter_type, str):
            filter_type = FILTER_NAMES.get(filter_type.lower(), L.RAMLAK)
        self._ck(lib().ctb_set_filter(self._ctx, int(filter_type)))

    def setSkipProjections(self, value: int = 0):
        self._ck(lib().ctb_set_skip_projections(self._ctx, value))

    def setActiveCudaDevices(self, devices):
        """Devices that share the reconstruction, each taking a run of z slices;
        IDs beyond the device count are dropped (a device may be listed twice)."""
        ids = np.ascontiguousarray(list(devices), np.int32)
        self._ck(lib().ctb_set_devices(self._ctx, ids.ctypes.data, len(ids)))

    def setGpuCoefficients(self, multiprocessorCoefficient: float, memoryBandwidthCoefficient: float):
        self._ck(lib().ctb_set_gpu_coefficients(self._ctx, float(multiprocessorCoefficient),
                                                float(memoryBandwidthCoefficient)))

    def getGpuWeights(self, devices) -> dict:
        ids = np.ascontiguousarray(list(devices), np.int32)
        w = np.zeros(len(ids), np.float64)
        self._ck(lib().ctb_get_gpu_weights(self._ctx, ids.ctypes.data, len(ids), w.ctypes.data))
        return {int(d): float(x) for d, x in zip(ids, w)}

    def setGpuSpareMemory(self, megabytes: int):
        self._ck(lib().ctb_set_gpu_spare_memory(self._ctx, int(megabytes)))

    def setPrecision(self, store: str | int):
        t = {"fp32": L.FP32, "fp16": L.FP16, "bf16": L.BF16}.get(store, store) if isinstance(store, str) else store
        self._ck(lib().ctb_set_precision(self._ctx, int(t)))

    def setPad(self, pad: int):
        self._ck(lib().ctb_set_pad(self._ctx, int(pad)))

    def setGrid(self, x: int, y: int, z: int, voxel_pitch: float):
        self._ck(lib().ctb_set_grid(self._ctx, x, y, z, voxel_pitch))

    def setSlabHeight(self, slices: int):
        self._ck(lib().ctb_set_slab_height(self._ctx, slices))

    def setAutotune(self, on: bool):
        """Tune the backprojection on the first reconstruction of each scan/box shape (ctb_set_autotune)."""
        self._ck(lib().ctb_set_autotune(self._ctx, int(bool(on))))

    def autotune(self) -> dict:
        """Tune now on the loaded scan and box (ctb_autotune); the choice is kept for this shape."""
        t = L.Tuning()
        self._ck(lib().ctb_autotune(self._ctx, ctypes.byref(t)))
        return {k: getattr(t, k) for k, _ in L.Tuning._fields_}

    def getTuning(self) -> dict:
        t = L.Tuning()
        self._ck(lib().ctb_get_tuning(self._ctx, ctypes.byref(t)))
        return {k: getattr(t, k) for k, _ in L.Tuning._fields_}

    def setProgressCallback(self, fn):
        """fn(stage, percent); stage 0 loading, 1 reconstruction, 2 saving."""
        self._cb = L.PROGRESS_CB(lambda s, p, u: fn(s, p)) if fn else L.PROGRESS_CB()
        self._ck(lib().ctb_set_progress_callback(self._ctx, self._cb, None))

    # --------------------------------------------------------------- getters
    def detector(self) -> L.Detector:
        d = L.Detector()
        self._ck(lib().ctb_get_detector(self._ctx, ctypes.byref(d)))
        return d

    def grid(self) -> L.Grid:
        g = L.Grid()
        self._ck(lib().ctb_get_grid(self._ctx, ctypes.byref(g)))
        return g

    def getXSize(self): return self.grid().box[0]
    def getYSize(self): return self.grid().box[1]
    def getZSize(self): return self.grid().box[2]
    def getImageWidth(self): return self.detector().width
    def getImageHeight(self): return self.detector().height
    def getFCD(self): return self.detector().fcd
    def getUOffset(self): return self.detector().u_offset
    def getBaseIntensity(self): return self.detector().base_intensity
    def getPixelSize(self): return lib().ctb_get_pixel_size(self._ctx)
    def getReconstructionCylinderRadius(self): return int(self.detector().radius)

    def getSinogramSize(self) -> int:
        n = ctypes.c_int()
        self._ck(lib().ctb_get_sinogram_size(self._ctx, ctypes.byref(n)))
        return n.value

    # ------------------------------------------------------------------ work
    def reconstructVolume(self):
        self._ck(lib().ctb_reconstruct(self._ctx))

    def reconstructInto(self, out_ptr: int, index_order: int = L.X_FASTEST):
        """Reconstruct into caller host memory (pinned memory is written without staging)."""
        self._ck(lib().ctb_reconstruct_into(self._ctx, out_ptr, index_order))

    def volume(self, index_order: int = L.X_FASTEST) -> np.ndarray:
        """The last reconstructed volume: shape (Z, Y, X) for X_FASTEST, (X, Y, Z) for Z_FASTEST."""
        x, y, z = self.grid().box
        shape = (z, y, x) if index_order == L.X_FASTEST else (x, y, z)
        out = np.empty(shape, np.float32)
        self._ck(lib().ctb_get_volume(self._ctx, out.ctypes.data, index_order))
        return out

    def saveVolumeToBinaryFile(self, filename: str, indexOrder: int = L.Z_FASTEST, byteOrder: int = L.LITTLE_ENDIAN):
        self._ck(lib().ctb_save_volume(self._ctx, str(filename).encode(), indexOrder, byteOrder))

    # ------------------------------------------------ matched projector pair (no reference counterpart)
    def _proj_shape(self):
        d = self.detector()
        return (self.getSinogramSize(), d.height, d.width)

    def forwardProject(self, volume: np.ndarray) -> np.ndarray:
        """A x: the forward projector on this scan's views and box; volume (Z, Y, X) float32 -> (V, H, W)."""
        x = np.ascontiguousarray(volume, np.float32)
        out = np.empty(self._proj_shape(), np.float32)
        self._ck(lib().ctb_forward(self._ctx, x.ctypes.data, out.ctypes.data))
        return out

    def backProject(self, projections: np.ndarray) -> np.ndarray:
        """A^T y: the exact transpose of forwardProject (unfiltered); (V, H, W) float32 -> (Z, Y, X)."""
        y = np.ascontiguousarray(projections, np.float32)
        X, Y, Z = self.grid().box
        out = np.empty((Z, Y, X), np.float32)
        self._ck(lib().ctb_backward(self._ctx, y.ctypes.data, out.ctypes.data))
        return out

    def gradient(self, volume: np.ndarray, data: np.ndarray):
        """(||A x - p||^2, 2 A^T (A x - p)) for volume x (Z, Y, X) and data p (V, H, W)."""
        x = np.ascontiguousarray(volume, np.float32)
        p = np.ascontiguousarray(data, np.float32)
        g = np.empty_like(x)
        f = ctypes.c_double()
        self._ck(lib().ctb_gradient(self._ctx, x.ctypes.data, p.ctypes.data, g.ctypes.data, ctypes.byref(f)))
        return f.value, g

    def getVolumeCrossSection(self, axis: int, index: int) -> np.ndarray:
        """Cross section of the last volume, left-handed orientation (Volume::getVolumeCrossSection)."""
        rows, cols = ctypes.c_int(), ctypes.c_int()
        self._ck(lib().ctb_get_cross_section(self._ctx, axis, index, None, ctypes.byref(rows), ctypes.byref(cols)))
        out = np.empty((rows.value, cols.value), np.float32)
        self._ck(lib().ctb_get_cross_section(self._ctx, axis, index, out.ctypes.data, None, None))
        return out

    # ------------------------------------------------ remaining CtVolume getters / setters
    @staticmethod
    def getCudaDeviceCount() -> int:
        n = ctypes.c_int()
        return n.value if lib().ctb_device_count(ctypes.byref(n)) == L.CTB_OK else -1

    @staticmethod
    def cudaAvailable() -> bool:
        return CtVolume.getCudaDeviceCount() > 0

    def getCudaDeviceList(self):
        names = []
        for i in range(max(0, self.getCudaDeviceCount())):
            buf = ctypes.create_string_buffer(256)
            lib().ctb_device_name(i, buf, 256)
            names.append(buf.value.decode(errors="replace"))
        return names

    def _settings(self) -> L.Settings:
        s = L.Settings()
        self._ck(lib().ctb_get_settings(self._ctx, ctypes.byref(s)))
        return s

    def getSkipProjections(self): return self._settings().skip_projections
    def getUseCuda(self): return bool(self._settings().use_cuda)
    def getUseCpuPreprocessing(self): return bool(self._settings().use_cpu_preprocessing)
    def getEmitSignals(self): return bool(self._settings().emit_signals)
    def getGpuSpareMemory(self): return self._settings().gpu_spare_memory_mb
    def getMultiprocessorCoefficient(self): return self._settings().multiprocessor_coefficient
    def getMemoryBandwidthCoefficient(self): return self._settings().memory_bandwidth_coefficient

    def getActiveCudaDevices(self):
        s = self._settings()
        return [s.devices[i] for i in range(s.n_devices)]

    def getRequiredMemoryUpperBound(self) -> int:
        n = ctypes.c_size_t()
        self._ck(lib().ctb_get_required_memory(self._ctx, ctypes.byref(n)))
        return n.value

    def setUseCuda(self, value: bool):
        self._ck(lib().ctb_set_use_cuda(self._ctx, int(bool(value))))

    def setUseCpuPreprocessing(self, value: bool):
        self._ck(lib().ctb_set_use_cpu_preprocessing(self._ctx, int(bool(value))))

    def setEmitSignals(self, value: bool):
        self._ck(lib().ctb_set_emit_signals(self._ctx, int(bool(value))))

    def getProjectionAt(self, index: int):
        """(image normalised by the scan's min / max as float32 (H, W), angle in degrees, height offset in pixels)."""
        w, h = self.getImageWidth(), self.getImageHeight()
        img = np.empty((h, w), np.float32)
        a, o = ctypes.c_double(), ctypes.c_double()
        self._ck(lib().ctb_get_projection(self._ctx, int(index), img.ctypes.data, ctypes.byref(a), ctypes.byref(o)))
        return img, a.value, o.value

    def setCrossSectionAxis(self, axis: int):
        self._ck(lib().ctb_set_cross_section_axis(self._ctx, int(axis)))

    def setCrossSectionIndex(self, index: int):
        self._ck(lib().ctb_set_cross_section_index(self._ctx, int(index)))

    def _cs_info(self):
        a, i, n = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        self._ck(lib().ctb_get_cross_section_info(self._ctx, ctypes.byref(a), ctypes.byref(i), ctypes.byref(n)))
        return a.value, i.value, n.value

    def getCrossSectionAxis(self): return self._cs_info()[0]
    def getCrossSectionIndex(self): return self._cs_info()[1]
    def getCrossSectionSize(self): return self._cs_info()[2]

    def setPreviewCallback(self, fn):
        """fn(percent, section) after every downloaded slab of reconstructVolume and once at 100 %;
        section is a copy (rows x cols float32) of the current cross section."""
        def tramp(pct, ptr, rows, cols, user):
            fn(pct, np.ctypeslib.as_array(ptr, shape=(rows, cols)).copy())
        self._pcb = L.PREVIEW_CB(tramp) if fn else L.PREVIEW_CB()
        self._ck(lib().ctb_set_preview_callback(self._ctx, self._pcb, None))

    def stop(self):
        lib().ctb_stop(self._ctx)

    def timings(self) -> L.Timings:
        t = L.Timings()
        self._ck(lib().ctb_get_timings(self._ctx, ctypes.byref(t)))
        return t


def gpu_weights_from(sm_counts, bandwidths, multiprocessorCoefficient=1.0, memoryBandwidthCoefficient=1.0):
    """getGpuWeights' formula on given device properties (no device query)."""
    sm = np.ascontiguousarray(sm_counts, np.int32)
    bw = np.ascontiguousarray(bandwidths, np.float64)
    w = np.zeros(len(sm), np.float64)
    check(lib().ctb_gpu_weights_from(sm.ctypes.data, bw.ctypes.data, len(sm), float(multiprocessorCoefficient),
                                     float(memoryBandwidthCoefficient), w.ctypes.data))
    return w


def split_slices(weights, z: int) -> np.ndarray:
    """First slice of each device's z range plus the end (n + 1 entries)."""
    w = np.ascontiguousarray(weights, np.float64)
    b = np.zeros(len(w) + 1, np.int32)
    check(lib().ctb_split_slices(w.ctypes.data, len(w), int(z), b.ctypes.data))
    return b


def read_image(path: str) -> np.ndarray:
    """One projection image decoded as the reference reads it (Projection::getImage)."""
    w, h, t = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    check(lib().ctb_read_image(str(path).encode(), ctypes.byref(w), ctypes.byref(h), ctypes.byref(t), None))
    dt = {L.U8: np.uint8, L.U16: np.uint16, L.F32: np.float32}[t.value]
    out = np.empty((h.value, w.value), dt)
    check(lib().ctb_read_image(str(path).encode(), ctypes.byref(w), ctypes.byref(h), ctypes.byref(t), out.ctypes.data))
    return out


def read_volume_info(txt_path: str) -> dict:
    """Dimensions and orders from a reconstruction's .txt info file (as the viewer reads it)."""
    x, y, z, io, bo = (ctypes.c_int() for _ in range(5))
    check(lib().ctb_read_volume_info(str(txt_path).encode(), ctypes.byref(x), ctypes.byref(y), ctypes.byref(z),
                                     ctypes.byref(io), ctypes.byref(bo)))
    return {"x": x.value, "y": y.value, "z": z.value, "index_order": io.value, "byte_order": bo.value}


def load_volume(raw_path: str, x: int, y: int, z: int, index_order: int = L.Z_FASTEST,
                byte_order: int = L.LITTLE_ENDIAN, data_type: int = 0, header_offset: int = 0,
                mirror=(False, False, False)) -> np.ndarray:
    """Volume::loadFromBinaryFile into a (Z, Y, X) float32 array."""
    out = np.empty((z, y, x), np.float32)
    check(lib().ctb_load_volume(str(raw_path).encode(), x, y, z, index_order, byte_order, data_type, header_offset,
                                int(mirror[0]), int(mirror[1]), int(mirror[2]), out.ctypes.data))
    return out
