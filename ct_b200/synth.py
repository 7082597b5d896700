"""Synthetic cone-beam scans: seeded random ellipsoid phantoms, analytic
projections, conversion to 16-bit intensities (optionally with Poisson noise),
and a writer for the reference's on-disk format (CSV + 16-bit PGM images).

The CSV layout is the one Ct/CtVolume.cpp:157-213 parses: image directory,
pixel size, rotation direction, u offset, FCD, base intensity, one ignored
line, then `file<TAB>angle_deg[<TAB>heightOffset_mm]` per image.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field

import numpy as np


@dataclass
class ScanGeometry:
    """Circular orbit; distances in mm. pixel_eff = detector pitch * SOD / SDD."""
    n_views: int
    width: int
    height: int
    pitch_mm: float
    sod_mm: float
    sdd_mm: float
    arc_deg: float = 360.0
    u_offset_mm: float = 0.0
    heights_mm: np.ndarray | None = None

    @property
    def pixel_eff(self) -> float:
        return self.pitch_mm * self.sod_mm / self.sdd_mm

    @property
    def fcd_px(self) -> float:
        return self.sod_mm / self.pixel_eff

    def angles(self) -> np.ndarray:
        return np.arange(self.n_views, dtype=np.float64) * (self.arc_deg / self.n_views)


def random_rotation(rng: np.random.Generator) -> np.ndarray:
    q = rng.standard_normal(4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def random_ellipsoids(rng: np.random.Generator, n: int, fov_radius_mm: float, half_height_mm: float,
                      axes_mm=(5.0, 60.0), density=(-0.5, 1.0), n_small: int = 0, small_axes_mm=(0.5, 2.0),
                      small_density: float = 2.0) -> np.ndarray:
    """(n + n_small, 16) table {c(3), semi-axes(3), R row-major(9), density}: centres uniform in the
    inner 80% of the field of view, random rotations."""
    rows = []
    for i in range(n + n_small):
        small = i >= n
        c = np.array([rng.uniform(-0.8, 0.8) * fov_radius_mm / math.sqrt(2),
                      rng.uniform(-0.8, 0.8) * fov_radius_mm / math.sqrt(2),
                      rng.uniform(-0.8, 0.8) * half_height_mm])
        ax = rng.uniform(*(small_axes_mm if small else axes_mm), size=3)
        R = random_rotation(rng)
        rho = small_density if small else rng.uniform(*density)
        rows.append(np.concatenate([c, ax, R.ravel(), [rho]]))
    return np.array(rows, np.float64)


def fov(geom: ScanGeometry):
    """Reconstruction cylinder radius and half height in mm (reference grid rule)."""
    D = geom.fcd_px
    r = (geom.width // 2)
    radius_px = math.floor(math.sqrt(D * D * r * r / (D * D + r * r)))
    return radius_px * geom.pixel_eff, geom.height / 2 * geom.pixel_eff


def intensities_from_line_integrals(p, photons: float | None = None, seed: int = 0, scale: float = 0.02):
    """I = 65535 exp(-scale p) as uint16 (torch or numpy); with Poisson counts at `photons` per ray."""
    try:
        import torch
        is_torch = isinstance(p, torch.Tensor)
    except ImportError:  # pragma: no cover
        is_torch = False
    if is_torch:
        import torch
        t = torch.exp(-scale * p)
        if photons:
            g = torch.Generator(device=p.device)
            g.manual_seed(seed)
            t = torch.poisson(t * photons, generator=g) / photons
        return torch.clamp(torch.round(65535.0 * t), 0, 65535).to(torch.int32).to(torch.uint16)
    t = np.exp(-scale * np.asarray(p, np.float64))
    if photons:
        t = np.random.default_rng(seed).poisson(t * photons) / photons
    return np.clip(np.round(65535.0 * t), 0, 65535).astype(np.uint16)


def write_pgm16(path: str, img: np.ndarray):
    img = np.asarray(img, np.uint16)
    h, w = img.shape
    with open(path, "wb") as f:
        f.write(f"P5\n{w} {h}\n65535\n".encode())
        f.write(img.astype(">u2").tobytes())


def write_scan(dirpath: str, images: np.ndarray, geom: ScanGeometry, rotation: str = "ccw",
               base_intensity: float = 1.0, image_subdir: str = "images", heights_mm=None,
               angles_deg=None) -> str:
    """Write images as 16-bit PGM plus the CSV; returns the CSV path."""
    os.makedirs(os.path.join(dirpath, image_subdir), exist_ok=True)
    angles = geom.angles() if angles_deg is None else np.asarray(angles_deg)
    lines = [image_subdir, repr(float(geom.pixel_eff)), rotation, repr(float(geom.u_offset_mm)),
             repr(float(geom.sod_mm)), repr(float(base_intensity)), "ignored"]
    for i, img in enumerate(images):
        name = f"proj_{i:05d}.pgm"
        write_pgm16(os.path.join(dirpath, image_subdir, name), img)
        line = f"{name}\t{float(angles[i])!r}"
        if heights_mm is not None:
            line += f"\t{float(heights_mm[i])!r}"
        lines.append(line)
    csv = os.path.join(dirpath, "scan.csv")
    with open(csv, "w") as f:
        f.write("\n".join(lines) + "\n")
    return csv


@dataclass
class Scan:
    geom: ScanGeometry
    ellipsoids: np.ndarray
    images: object = None          # (V, H, W) uint16, numpy or torch
    extra: dict = field(default_factory=dict)


def make_scan(geom: ScanGeometry, n_ellipsoids: int, seed: int, photons: float | None = None, n_small: int = 0,
              device: str = "cuda", chunk_views: int = 32, out=None) -> Scan:
    """Project a seeded phantom on the GPU and convert to uint16 intensities (torch tensor on `device`)."""
    import torch

    from .ops import phantom_project
    rng = np.random.default_rng(seed)
    r_mm, hz_mm = fov(geom)
    ell = random_ellipsoids(rng, n_ellipsoids, r_mm, hz_mm, n_small=n_small)
    angles = geom.angles()
    heights = geom.heights_mm
    if out is None:
        out = torch.empty((geom.n_views, geom.height, geom.width), dtype=torch.uint16, device=device)
    for v0 in range(0, geom.n_views, chunk_views):
        v1 = min(geom.n_views, v0 + chunk_views)
        p = phantom_project(ell, angles[v0:v1], None if heights is None else heights[v0:v1], geom.width,
                            geom.height, geom.pixel_eff, geom.sod_mm, geom.u_offset_mm, device=device)
        out[v0:v1].copy_(intensities_from_line_integrals(p, photons, seed * 100003 + v0))
    return Scan(geom, ell, out)
