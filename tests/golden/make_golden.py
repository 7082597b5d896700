"""Generate the golden fixtures in tests/golden/ (run in a container with cv2).

The reference (bastian-weber/Ct) needs the Qt5 and OpenCV 3.1 C++ libraries
and cannot be built here, and it ships no test vectors. Its CPU path does its
arithmetic through OpenCV; the cv2 Python module (4.13, same flag semantics)
runs those exact calls here:
  * cv::dft(DFT_COMPLEX_OUTPUT | DFT_ROWS) / cv::idft(DFT_ROWS | DFT_REAL_OUTPUT)
    with the window multiply in between (Ct/CtVolume.cpp:832-858),
  * cv::log (Ct/CtVolume.cpp:864),
  * the whole preprocessing chain of one projection (:802-866, :814-830),
  * a tiny end-to-end reconstruction whose backprojection loops are a numpy
    restatement of reconstructionCore (:923-1046) written independently of the
    C++ oracle (float32 geometry, double bilinear blend).
The C++ oracle is checked against these files by tests/test_oracle_golden.py.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import math
import os

import cv2
import numpy as np

OUT = os.path.dirname(os.path.abspath(__file__))
f32 = np.float32


def window(filter_type: int, k: int, nyq: int) -> np.float32:
    """Ct/CtVolume.cpp:868-885 (float rl; sin/cos in double of float products)."""
    rl = f32(k) / f32(nyq)
    if filter_type == 1:
        if k == 0:
            return f32(0)
        a = float(rl * f32(0.5)) * math.pi
        return f32(float(rl) * math.sin(a) / a)
    if filter_type == 2:
        return f32(float(rl * f32(0.5)) * (1.0 + math.cos(math.pi * float(rl))))
    return rl


def cv_filter(img: np.ndarray, filter_type: int) -> np.ndarray:
    freq = cv2.dft(img, flags=cv2.DFT_COMPLEX_OUTPUT | cv2.DFT_ROWS)
    nyq = freq.shape[1] // 2 + 1
    w = np.array([window(filter_type, k, nyq) for k in range(nyq)], np.float32)
    freq[:, :nyq, :] *= w[None, :, None]
    return cv2.idft(freq, flags=cv2.DFT_ROWS | cv2.DFT_REAL_OUTPUT)


def cv_preprocess(img: np.ndarray, base: float, FCD: float, filter_type: int) -> np.ndarray:
    H, W = img.shape
    # convertTo(CV_32F, alpha, beta): float working type, mul then add
    if img.dtype == np.uint8:
        x = img.astype(f32) * f32(1.0 / 255.0) + f32(0.000001 * base)
    elif img.dtype == np.uint16:
        x = img.astype(f32) * f32(1.0 / 65535.0) + f32(0.000001 * base)
    else:
        x = img.astype(f32)
    x = x * f32(1.0 / (base + 0.000001 * base))
    x = cv2.log(x)
    x = x * f32(-1)
    uPre, vPre = f32(W / 2.0), f32(H / 2.0)
    D = f32(FCD)
    u = np.arange(W, dtype=f32) - uPre
    v = f32(-1) * np.arange(H, dtype=f32)[:, None] + vPre
    wgt = D / np.sqrt(D * D + u[None, :] * u[None, :] + v * v, dtype=f32)
    x = (x * wgt).astype(f32)
    return cv_filter(np.ascontiguousarray(x), filter_type)


def np_backproject(image: np.ndarray, vol: np.ndarray, W: int, H: int, FCD: float, uOffset: float, xSize: int,
                   ySize: int, zSize: int, box, radius: int, angle_deg: float, height: float):
    """One view of reconstructionCore into a Z_FASTEST float32 volume (x, y, z)."""
    xFrom, xTo, yFrom, yTo, zFrom, zTo = box
    xMax, yMax, zMax = xTo - xFrom, yTo - yFrom, zTo - zFrom
    uPre, vPre = f32(W / 2.0), f32(H / 2.0)
    xPre = f32(f32(xSize) / 2.0 - f32(xFrom))
    yPre = f32(f32(ySize) / 2.0 - f32(yFrom))
    zPre = f32(f32(zSize) / 2.0 - f32(zFrom))
    lbU = f32(0) - uPre
    ubU = f32(W - 1 - 0.1) - uPre
    lbV = f32(-1) * f32(H - 1 - 0.1) + vPre
    ubV = vPre
    r2 = f32(radius) * f32(radius)
    ang = f32((angle_deg / 180.0) * math.pi)
    sn, cs = f32(math.sin(float(ang))), f32(math.cos(float(ang)))
    D, uo, h = f32(FCD), f32(uOffset), f32(height)
    zs = np.arange(zMax, dtype=f32) - zPre
    for xi in range(xMax):
        x = f32(xi) - xPre
        for yi in range(yMax):
            y = f32(yi) - yPre
            if not (x * x + y * y < r2):
                continue
            t = f32(f32(-1) * x * sn + y * cs) + uo
            s = f32(x * cs + y * sn)
            U = f32(D / f32(D - s))
            u = f32(t * U)
            if u < lbU or u > ubU:
                continue
            w = f32(U * U)
            v = (zs + h) * U
            ok = (v >= lbV) & (v <= ubV)
            ui = f32(u + uPre)
            vi = f32(-1) * v + vPre
            u0 = int(ui)
            v0 = vi.astype(np.int64)
            v0c = np.where(ok, v0, 0)
            fu = f32(ui - f32(u0))
            fv = (vi - v0.astype(f32)).astype(f32)
            p00 = image[v0c, u0]; p01 = image[v0c, u0 + 1]
            p10 = image[v0c + 1, u0]; p11 = image[v0c + 1, u0 + 1]
            a = ((f32(1) - fu) * p00 + fu * p01).astype(np.float64)
            b = ((f32(1) - fu) * p10 + fu * p11).astype(np.float64)
            val = ((f32(1) - fv).astype(np.float64) * a + fv.astype(np.float64) * b).astype(f32)
            vol[xi, yi] += np.where(ok, w * val, f32(0)).astype(f32)


def main():
    rng = np.random.default_rng(20261203)
    # 1. row filter
    rows = {}
    for W in (16, 17, 64, 100, 255, 256):
        x = rng.standard_normal((4, W)).astype(f32)
        rows[f"x_{W}"] = x
        for ft in range(3):
            rows[f"y_{W}_{ft}"] = cv_filter(x, ft)
    np.savez_compressed(os.path.join(OUT, "filter_rows.npz"), **rows)
    # 2. log
    lx = np.concatenate([rng.uniform(1e-6, 1.5, 4000), rng.uniform(0.9, 1.1, 1000)]).astype(f32)
    np.savez_compressed(os.path.join(OUT, "log_values.npz"), x=lx, y=cv2.log(lx.reshape(1, -1)).ravel())
    # 3. preprocessing chain
    pre = {}
    img16 = rng.integers(200, 65535, size=(12, 20)).astype(np.uint16)
    img8 = rng.integers(5, 255, size=(12, 20)).astype(np.uint8)
    imgf = rng.uniform(0.05, 1.0, size=(12, 20)).astype(f32)
    pre.update(img16=img16, img8=img8, imgf=imgf)
    for name, img, base in (("u16", img16, 1.0), ("u8", img8, 0.9), ("f32", imgf, 1.2)):
        for ft in range(3):
            pre[f"out_{name}_{ft}"] = cv_preprocess(img, base, 55.0, ft)
    np.savez_compressed(os.path.join(OUT, "preprocess.npz"), **pre)
    # 4. tiny end-to-end reconstruction (reference grid, 24 views, ramlak)
    V, H, W, FCD = 24, 10, 16, 50.0
    imgs = rng.integers(30000, 65535, size=(V, H, W)).astype(np.uint16)
    angles = np.arange(V) * (360.0 / V)
    heights = np.zeros(V)
    rad = W // 2
    radius = int(math.sqrt((FCD * FCD * rad * rad) / (FCD * FCD + rad * rad)))
    xSize = ySize = 2 * radius
    zSize = H
    box = (0, xSize, 0, ySize, 0, zSize)
    vol = np.zeros((xSize, ySize, zSize), f32)
    for k in range(V):
        p = cv_preprocess(imgs[k], 1.0, FCD, 0)
        np_backproject(p, vol, W, H, FCD, 0.0, xSize, ySize, zSize, box, radius, angles[k], heights[k])
    # sub-box with the reference's bounds rounding: x 0.25..0.75, y 0.1..0.9, z 0.2..1
    sub = tuple(int(f * s + 0.5) for f, s in ((0.25, xSize), (0.75, xSize), (0.1, ySize), (0.9, ySize),
                                              (0.2, zSize), (1.0, zSize)))
    vsub = np.zeros((sub[1] - sub[0], sub[3] - sub[2], sub[5] - sub[4]), f32)
    for k in range(V):
        p = cv_preprocess(imgs[k], 1.0, FCD, 2)
        np_backproject(p, vsub, W, H, FCD, 1.5, xSize, ySize, zSize, sub, radius, angles[k], 0.75)
    np.savez_compressed(os.path.join(OUT, "recon_tiny.npz"), imgs=imgs, angles=angles, FCD=FCD, radius=radius,
                        vol=vol, sub=np.array(sub), vol_sub=vsub)
    print("written to", OUT)


if __name__ == "__main__":
    main()
