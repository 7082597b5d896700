"""TEST INFRASTRUCTURE ONLY -- numpy restatement of the analytic ellipsoid
projector, used to check the engine's device phantom kernel, plus a voxelised
phantom for error-to-truth measurements.

Model (the one the reference's backprojection assumes, Ct/CtVolume.cpp:989-1008):
a point maps to u = (t + uOffset) D / (D - s), v = (z + h) D / (D - s), so the ray
of pixel (r, c) (u = c - W/2, v = H/2 - r) runs from the source
S = D e_s - uOffset e_t - h e_z to Q = (u - uOffset) e_t + (v - h) e_z.
"""
from __future__ import annotations

import numpy as np


def project(ellipsoids: np.ndarray, angles_deg, heights_mm, width: int, height: int, pixel_mm: float,
            fcd_mm: float, u_offset_mm: float = 0.0) -> np.ndarray:
    ell = np.asarray(ellipsoids, np.float64)
    ang = np.asarray(angles_deg, np.float64)
    hh = np.zeros_like(ang) if heights_mm is None else np.asarray(heights_mm, np.float64)
    out = np.zeros((len(ang), height, width))
    c = np.arange(width)
    r = np.arange(height)
    u = (c[None, :] - width / 2.0) * pixel_mm
    v = (height / 2.0 - r[:, None]) * pixel_mm
    for k, (a, h) in enumerate(zip(ang, hh)):
        th = np.deg2rad(a)
        sn, cs = np.sin(th), np.cos(th)
        S = np.array([fcd_mm * cs + u_offset_mm * sn, fcd_mm * sn - u_offset_mm * cs, -h])
        tq = u - u_offset_mm
        Q = np.stack(np.broadcast_arrays(-tq * sn, tq * cs, v - h), axis=-1)
        d = Q - S
        d /= np.linalg.norm(d, axis=-1, keepdims=True)
        acc = np.zeros((height, width))
        for E in ell:
            R = E[6:15].reshape(3, 3)
            ax = E[3:6]
            pb = (R.T @ (S - E[:3])) / ax
            db = (d @ R) / ax
            a2 = np.einsum("...i,...i", db, db)
            b = db @ pb
            g = pb @ pb - 1.0
            disc = b * b - a2 * g
            acc += np.where(disc > 0, E[15] * 2.0 * np.sqrt(np.maximum(disc, 0)) / a2, 0.0)
        out[k] = acc
    return out


def voxelise(ellipsoids: np.ndarray, grid_size, voxel_mm: float, pre) -> np.ndarray:
    """Density at voxel centres, Z_FASTEST (x, y, z); world = (index - pre) * voxel_mm."""
    nx, ny, nz = grid_size
    x = (np.arange(nx) - pre[0]) * voxel_mm
    y = (np.arange(ny) - pre[1]) * voxel_mm
    z = (np.arange(nz) - pre[2]) * voxel_mm
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
    P = np.stack([X, Y, Z], -1)
    out = np.zeros(grid_size)
    for E in np.asarray(ellipsoids, np.float64):
        R = E[6:15].reshape(3, 3)
        q = ((P - E[:3]) @ R) / E[3:6]
        out += np.where((q * q).sum(-1) <= 1.0, E[15], 0.0)
    return out
