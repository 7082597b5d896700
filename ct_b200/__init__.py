"""ct_b200 -- B200-native FDK cone-beam reconstruction behind the reference's
CtVolume surface (bastian-weber/Ct). The compute path is libctb.so (hand-written
sm_100a CUDA kernels behind a C ABI, include/ctb.h); this package is its Python
binding (ctypes), mirroring ct::CtVolume, plus device-level operators and
synthetic-scan utilities.
"""
from ._lib import (AXIS_X, AXIS_Y, AXIS_Z, BF16, BIG_ENDIAN, F32, FP16, FP32, HANN, LITTLE_ENDIAN, RAMLAK,
                   SHEPPLOGAN, U8, U16, X_FASTEST, Z_FASTEST, CtbError, Detector, Grid, lib)
from .ctvolume import CtVolume, load_volume, read_volume_info

__all__ = ["CtVolume", "load_volume", "read_volume_info", "CtbError", "Detector", "Grid", "lib", "RAMLAK", "SHEPPLOGAN", "HANN", "X_FASTEST",
           "Z_FASTEST", "LITTLE_ENDIAN", "BIG_ENDIAN", "FP32", "FP16", "BF16", "U8", "U16", "F32", "AXIS_X", "AXIS_Y",
           "AXIS_Z"]
