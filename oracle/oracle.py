"""TEST INFRASTRUCTURE ONLY -- ctypes wrapper of the CPU oracle (ct_oracle.cpp).

The oracle restates the reference's CPU FDK path (bastian-weber/Ct,
Ct/CtVolume.cpp:802-1054) in C++ and adds a double-precision version of the
same mathematics. Only tests/, __graft_entry__.smoke() and bench.py's CPU
baseline leg use this module, as the checker; the product never imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libct_oracle.so")

RAMLAK, SHEPPLOGAN, HANN = 0, 1, 2
FILTERS = {"ramlak": RAMLAK, "shepplogan": SHEPPLOGAN, "hann": HANN}


class OrcGeom(ctypes.Structure):
    _fields_ = [
        ("W", ctypes.c_int), ("H", ctypes.c_int),
        ("FCD", ctypes.c_float), ("uOffset", ctypes.c_float), ("radius", ctypes.c_float),
        ("xSize", ctypes.c_int), ("ySize", ctypes.c_int), ("zSize", ctypes.c_int),
        ("xFrom", ctypes.c_int), ("xTo", ctypes.c_int),
        ("yFrom", ctypes.c_int), ("yTo", ctypes.c_int),
        ("zFrom", ctypes.c_int), ("zTo", ctypes.c_int),
        ("vs", ctypes.c_float),
    ]

    @property
    def box(self):
        return (self.xTo - self.xFrom, self.yTo - self.yFrom, self.zTo - self.zFrom)


def build() -> str:
    """Compile the oracle library with its Makefile (g++, OpenMP)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        P = ctypes.c_void_p
        L.orc_ref_cylinder_radius.restype = ctypes.c_uint
        L.orc_ref_cylinder_radius.argtypes = [ctypes.c_int, ctypes.c_float]
        L.orc_ref_clamp_bounds.restype = ctypes.c_int
        L.orc_ref_clamp_bounds.argtypes = [ctypes.c_float] * 6 + [P]
        L.orc_ref_geom.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_float, P, P]
        L.orc_ref_fix_sinogram.argtypes = [P, P, ctypes.c_int, ctypes.c_int, ctypes.c_double]
        L.orc_ref_window.restype = ctypes.c_float
        L.orc_ref_window.argtypes = [ctypes.c_int, ctypes.c_uint, ctypes.c_uint]
        L.orc_ref_preprocess.argtypes = [P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                         ctypes.c_float, ctypes.c_int, P]
        L.orc_ref_filter_rows.argtypes = [P, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.orc_ref_backproject.argtypes = [P, ctypes.c_int, ctypes.c_int, P, P, P, ctypes.c_int, P]
        L.orc_ref_reconstruct.restype = ctypes.c_int
        L.orc_ref_reconstruct.argtypes = [P, ctypes.c_int, ctypes.c_int, ctypes.c_int, P, P, ctypes.c_float,
                                          ctypes.c_int, P, ctypes.c_int, P, P]
        L.orc_f64_preprocess.argtypes = [P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                         ctypes.c_double, ctypes.c_int, ctypes.c_int, P]
        L.orc_f64_backproject.argtypes = [P, ctypes.c_int, P, P, P, ctypes.c_int, ctypes.c_int, P]
        L.orc_f64_preprocess_rows.argtypes = [P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                              ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                              ctypes.c_int, P]
        L.orc_f64_backproject_rows.restype = ctypes.c_int
        L.orc_f64_backproject_rows.argtypes = [P, ctypes.c_int, P, P, P, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                               ctypes.c_int, P, P]
        L.orc_num_threads.restype = ctypes.c_int
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def _depth(img: np.ndarray) -> int:
    return {np.dtype(np.uint8): 8, np.dtype(np.uint16): 16, np.dtype(np.float32): 32}[img.dtype]


# ------------------------------------------------------------------ geometry
def cylinder_radius(W: int, FCD: float) -> int:
    return int(lib().orc_ref_cylinder_radius(W, FCD))


def clamp_bounds(xf, xt, yf, yt, zf, zt):
    out = np.zeros(6, np.float32)
    ok = lib().orc_ref_clamp_bounds(xf, xt, yf, yt, zf, zt, _p(out))
    return tuple(float(v) for v in out) if ok else None


def ref_geom(W, H, FCD, uOffset=0.0, rel=(0, 1, 0, 1, 0, 1)) -> OrcGeom:
    g = OrcGeom()
    r = np.asarray(rel, np.float32)
    lib().orc_ref_geom(W, H, FCD, uOffset, _p(r), ctypes.byref(g))
    return g


def custom_geom(W, H, FCD, grid, vs, uOffset=0.0, box=None, radius=None) -> OrcGeom:
    """Grid of arbitrary size and voxel pitch `vs` (in detector pixels)."""
    g = OrcGeom()
    g.W, g.H, g.FCD, g.uOffset = W, H, FCD, uOffset
    g.radius = float(cylinder_radius(W, FCD) if radius is None else radius)
    g.xSize, g.ySize, g.zSize = grid
    if box is None:
        box = (0, grid[0], 0, grid[1], 0, grid[2])
    g.xFrom, g.xTo, g.yFrom, g.yTo, g.zFrom, g.zTo = box
    g.vs = vs
    return g


def fix_sinogram(angles, heights, ccw: bool, pixel_size: float):
    a = np.array(angles, np.float64)
    h = np.array(heights, np.float64)
    lib().orc_ref_fix_sinogram(_p(a), _p(h), len(a), int(bool(ccw)), float(pixel_size))
    return a, h


# --------------------------------------------------------- reference FP32 path
def window(filter_type: int, k: int, nyq: int) -> float:
    return float(lib().orc_ref_window(filter_type, k, nyq))


def ref_preprocess(img: np.ndarray, base: float, FCD: float, filter_type: int) -> np.ndarray:
    img = np.ascontiguousarray(img)
    H, W = img.shape
    out = np.empty((H, W), np.float32)
    lib().orc_ref_preprocess(_p(img), _depth(img), W, H, base, FCD, filter_type, _p(out))
    return out


def ref_filter_rows(rows: np.ndarray, filter_type: int) -> np.ndarray:
    out = np.array(rows, np.float32, copy=True, order="C")
    H, W = out.shape
    lib().orc_ref_filter_rows(_p(out), W, H, filter_type)
    return out


def ref_backproject(proj: np.ndarray, angles, heights, g: OrcGeom, step: int = 1,
                    nthreads: int = 0) -> np.ndarray:
    """Filtered projections (V, H, W) float32 -> Z_FASTEST volume (x, y, z)."""
    proj = np.ascontiguousarray(proj, np.float32)
    a = np.ascontiguousarray(angles, np.float64)
    h = np.ascontiguousarray(heights, np.float64)
    vol = np.zeros(g.box, np.float32)
    lib().orc_ref_backproject(_p(proj), proj.shape[0], step, _p(a), _p(h), ctypes.byref(g), nthreads, _p(vol))
    return vol


def ref_reconstruct(imgs: np.ndarray, angles, heights, base: float, filter_type: int, g: OrcGeom,
                    step: int = 1, nthreads: int = 0):
    """Whole reference CPU path from raw images (V, H, W). Returns (volume x,y,z, seconds)."""
    imgs = np.ascontiguousarray(imgs)
    a = np.ascontiguousarray(angles, np.float64)
    h = np.ascontiguousarray(heights, np.float64)
    vol = np.zeros(g.box, np.float32)
    secs = ctypes.c_double(0)
    lib().orc_ref_reconstruct(_p(imgs), _depth(imgs[0]), imgs.shape[0], step, _p(a), _p(h), base,
                              filter_type, ctypes.byref(g), nthreads, _p(vol), ctypes.byref(secs))
    return vol, secs.value


# ----------------------------------------------------------------- FP64 oracle
def f64_preprocess(img: np.ndarray, base: float, FCD: float, filter_type: int, pad: int = 1) -> np.ndarray:
    img = np.ascontiguousarray(img)
    H, W = img.shape
    out = np.empty((H, W), np.float64)
    lib().orc_f64_preprocess(_p(img), _depth(img), W, H, base, FCD, filter_type, pad, _p(out))
    return out


def f64_backproject(proj: np.ndarray, angles, heights, g: OrcGeom, z0: int = 0, z1: int = 0) -> np.ndarray:
    proj = np.ascontiguousarray(proj, np.float64)
    a = np.ascontiguousarray(angles, np.float64)
    h = np.ascontiguousarray(heights, np.float64)
    bx, by, bz = g.box
    nz = (z1 - z0) if z1 > z0 else bz
    vol = np.zeros((bx, by, nz), np.float64)
    lib().orc_f64_backproject(_p(proj), proj.shape[0], _p(a), _p(h), ctypes.byref(g), z0, z1, _p(vol))
    return vol


def f64_reconstruct(imgs, angles, heights, base, filter_type, g: OrcGeom, pad=1, z0=0, z1=0):
    proj = np.stack([f64_preprocess(im, base, g.FCD, filter_type, pad) for im in imgs])
    return f64_backproject(proj, angles, heights, g, z0, z1)


def f64_slices(imgs_rows: np.ndarray, row0: int, H: int, angles, heights, base: float, filter_type: int,
               g: OrcGeom, z0: int, z1: int, pad: int = 1) -> np.ndarray:
    """FP64 reconstruction of box slices [z0, z1) from detector rows [row0, row0 + n) of every view
    (imgs_rows: (V, n, W)). Raises if a sample falls outside the row window."""
    imgs_rows = np.ascontiguousarray(imgs_rows)
    V, n, W = imgs_rows.shape
    proj = np.empty((V, n, W), np.float64)
    L = lib()
    for k in range(V):
        L.orc_f64_preprocess_rows(_p(imgs_rows[k]), _depth(imgs_rows[k]), W, H, row0, n, base, g.FCD,
                                  filter_type, pad, _p(proj[k]))
    a = np.ascontiguousarray(angles, np.float64)
    h = np.ascontiguousarray(heights, np.float64)
    bx, by, _ = g.box
    vol = np.zeros((bx, by, z1 - z0), np.float64)
    missed = ctypes.c_longlong(0)
    L.orc_f64_backproject_rows(_p(proj), V, _p(a), _p(h), ctypes.byref(g), row0, n, z0, z1, _p(vol),
                               ctypes.byref(missed))
    if missed.value:
        raise ValueError(f"{missed.value} samples outside detector rows [{row0}, {row0 + n})")
    return vol


def num_threads() -> int:
    return int(lib().orc_num_threads())


@dataclass
class RelErr:
    rel_l2: float
    max_abs: float


def rel_err(x: np.ndarray, ref: np.ndarray) -> RelErr:
    x = np.asarray(x, np.float64)
    ref = np.asarray(ref, np.float64)
    d = x - ref
    n = np.linalg.norm(ref.ravel())
    return RelErr(float(np.linalg.norm(d.ravel()) / (n if n > 0 else 1.0)), float(np.abs(d).max(initial=0.0)))


# --------------------------------------------- the reference's own CPU code
# oracle/_ref/libct_ref.so: the reference's CPU reconstruction lines of
# Ct/CtVolume.cpp compiled unchanged (oracle/Makefile target `ref`, shims in
# oracle/ref_shim.h, driver in oracle/ref_build.cpp). Built where the
# reference sources are present; the built library travels with the tree.
_REF_LIB_PATH = os.path.join(_HERE, "_ref", "libct_ref.so")
# the same lines built with <cmath> alone (libstdc++): sqrt/sin/cos of a float
# resolve to the double functions there
_REF_GCC_LIB_PATH = os.path.join(_HERE, "_ref", "libct_ref_gcc.so")
_REF_SOURCE = "/root/reference/Ct/CtVolume.cpp"
_ref_libs = {}


def build_ref() -> str | None:
    """Build oracle/_ref/libct_ref.so from the reference sources if they are
    present; returns the library path, or None when neither exists."""
    if os.path.exists(_REF_SOURCE):
        subprocess.run(["make", "-s", "-C", _HERE, "ref"], check=True)
    return _REF_LIB_PATH if os.path.exists(_REF_LIB_PATH) else None


def ref_source_available() -> bool:
    return os.path.exists(_REF_LIB_PATH) or os.path.exists(_REF_SOURCE)


def ref_lib(variant: str = "msvc"):
    """variant "msvc": float overloads of sqrt/sin/cos in the global namespace
    (the reference's Windows build); "gcc": <cmath> alone under libstdc++."""
    if variant not in _ref_libs:
        if build_ref() is None:
            raise FileNotFoundError("oracle/_ref/libct_ref.so is not built and the reference sources are absent")
        L = ctypes.CDLL(_REF_LIB_PATH if variant == "msvc" else _REF_GCC_LIB_PATH)
        P, I, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        L.ref_reconstruct.restype = I
        L.ref_reconstruct.argtypes = [P, I, I, I, I, P, P, D, D, D, D, ctypes.c_char_p, P, I, ctypes.c_uint, P, P,
                                      P, I]
        L.ref_prepare_projection.restype = I
        L.ref_prepare_projection.argtypes = [P, I, I, I, I, P, D, D, D, I, I, P]
        L.ref_fix_sinogram.restype = I
        L.ref_fix_sinogram.argtypes = [I, P, P, D, ctypes.c_char_p, P, P]
        _ref_libs[variant] = L
    return _ref_libs[variant]


def refsrc_reconstruct(imgs: np.ndarray, angles_deg, heights_mm, pixel_size: float, fcd_mm: float,
                       u_offset_mm: float = 0.0, base: float = 1.0, rotation: str = "ccw", rel=None,
                       filter_type: int = RAMLAK, skip: int = 0, dims_only: bool = False,
                       variant: str = "msvc", keep_volume: bool = True):
    """The reference's own CPU reconstruction (CSV values as they appear in the
    file: angles in degrees, heights and distances in mm). Returns
    (volume (x, y, z) Z_FASTEST, seconds of the zeroed volume and
    reconstructionCore), or the box dimensions with dims_only. keep_volume=False
    runs the reconstruction and returns (box dimensions, seconds)."""
    imgs = np.ascontiguousarray(imgs)
    V, H, W = imgs.shape
    a = np.ascontiguousarray(angles_deg, np.float64)
    h = None if heights_mm is None else np.ascontiguousarray(heights_mm, np.float64)
    r6 = None if rel is None else np.ascontiguousarray(rel, np.float32)
    dims = np.zeros(3, np.int32)
    L = ref_lib(variant)
    args = (_p(imgs), _depth(imgs[0]), V, W, H, _p(a), None if h is None else _p(h), pixel_size, u_offset_mm,
            fcd_mm, base, rotation.encode(), None if r6 is None else _p(r6), filter_type, skip)
    st = L.ref_reconstruct(*args, None, _p(dims), None, 0)
    if st != 0:
        raise RuntimeError(f"ref_reconstruct failed ({st})")
    if dims_only:
        return tuple(int(d) for d in dims)
    secs = ctypes.c_double(0)
    if not keep_volume:
        st = L.ref_reconstruct(*args, None, _p(dims), ctypes.byref(secs), 1)
        if st != 0:
            raise RuntimeError(f"ref_reconstruct failed ({st})")
        return tuple(int(d) for d in dims), secs.value
    vol = np.zeros(tuple(int(d) for d in dims), np.float32)
    st = L.ref_reconstruct(*args, _p(vol), _p(dims), ctypes.byref(secs), 1)
    if st != 0:
        raise RuntimeError(f"ref_reconstruct failed ({st})")
    return vol, secs.value


def refsrc_prepare_projection(imgs: np.ndarray, index: int, pixel_size: float, fcd_mm: float, base: float = 1.0,
                              filter_type: int = RAMLAK, variant: str = "msvc") -> np.ndarray:
    """The reference's prepareProjection of view `index` (H x W float32)."""
    imgs = np.ascontiguousarray(imgs)
    V, H, W = imgs.shape
    a = np.zeros(V, np.float64)
    out = np.empty((H, W), np.float32)
    st = ref_lib(variant).ref_prepare_projection(_p(imgs), _depth(imgs[0]), V, W, H, _p(a), pixel_size, fcd_mm, base,
                                          filter_type, index, _p(out))
    if st != 0:
        raise RuntimeError(f"ref_prepare_projection failed ({st})")
    return out


def refsrc_fix_sinogram(angles_deg, heights_mm, pixel_size: float, rotation: str):
    """The reference's makeHeightOffsetRelative + correctAngleDirection:
    (angles in degrees, relative height offsets in pixels)."""
    a = np.ascontiguousarray(angles_deg, np.float64)
    h = np.ascontiguousarray(heights_mm, np.float64)
    ao = np.empty_like(a)
    ho = np.empty_like(a)
    ref_lib().ref_fix_sinogram(len(a), _p(a), _p(h), pixel_size, rotation.encode(), _p(ao), _p(ho))
    return ao, ho
