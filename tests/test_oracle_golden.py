"""The CPU oracle against golden vectors made with the reference's own
third-party arithmetic (OpenCV via cv2, tests/golden/make_golden.py) and
against known-answer values of the reference's formulas."""
import math
import os

import numpy as np
import pytest


def load(golden_dir, name):
    return np.load(os.path.join(golden_dir, name))


def test_filter_rows_match_opencv(oracle, golden_dir):
    g = load(golden_dir, "filter_rows.npz")
    for W in (16, 17, 64, 100, 255, 256):
        x = g[f"x_{W}"]
        for ft in range(3):
            ref = g[f"y_{W}_{ft}"]
            out = oracle.ref_filter_rows(x, ft)
            err = np.abs(out - ref).max() / np.abs(ref).max()
            assert err < 2e-6, (W, ft, err)


def test_log_matches_opencv_within_2ulp(golden_dir):
    g = load(golden_dir, "log_values.npz")
    ours = np.log(g["x"].astype(np.float64)).astype(np.float32)  # logf is correctly rounded to <1 ulp
    d = np.abs(ours.view(np.int32).astype(np.int64) - g["y"].view(np.int32).astype(np.int64))
    assert d.max() <= 2


@pytest.mark.parametrize("name,base", [("u16", 1.0), ("u8", 0.9), ("f32", 1.2)])
@pytest.mark.parametrize("ft", [0, 1, 2])
def test_preprocess_chain_matches_opencv(oracle, golden_dir, name, base, ft):
    g = load(golden_dir, "preprocess.npz")
    img = g[{"u16": "img16", "u8": "img8", "f32": "imgf"}[name]]
    ref = g[f"out_{name}_{ft}"]
    out = oracle.ref_preprocess(img, base, 55.0, ft)
    err = np.linalg.norm(out - ref) / np.linalg.norm(ref)
    assert err < 2e-6, err


def test_tiny_reconstruction_matches_golden(oracle, golden_dir):
    g = load(golden_dir, "recon_tiny.npz")
    imgs, angles, FCD = g["imgs"], g["angles"], float(g["FCD"])
    V, H, W = imgs.shape
    geom = oracle.ref_geom(W, H, FCD)
    assert geom.radius == int(g["radius"])
    vol, _ = oracle.ref_reconstruct(imgs, angles, np.zeros(V), 1.0, oracle.RAMLAK, geom, nthreads=2)
    err = oracle.rel_err(vol, g["vol"])
    assert err.rel_l2 < 1e-6, err
    # sub-box, u offset and height offset, hann
    sub = tuple(int(v) for v in g["sub"])
    gs = oracle.custom_geom(W, H, FCD, (geom.xSize, geom.ySize, geom.zSize), 1.0, uOffset=1.5, box=sub)
    proj = np.stack([oracle.ref_preprocess(im, 1.0, FCD, oracle.HANN) for im in imgs])
    vsub = oracle.ref_backproject(proj, angles, np.full(V, 0.75), gs, nthreads=2)
    err = oracle.rel_err(vsub, g["vol_sub"])
    assert err.rel_l2 < 1e-6, err


def test_window_known_answers(oracle):
    nyq = 129
    for ft in range(3):
        assert oracle.window(ft, 0, nyq) == 0.0
    assert oracle.window(0, 1, nyq) == np.float32(1) / np.float32(nyq)
    assert oracle.window(0, nyq - 1, nyq) == np.float32(nyq - 1) / np.float32(nyq)
    rl = float(np.float32(1) / np.float32(nyq))
    assert abs(oracle.window(1, 1, nyq) - rl * math.sin(rl * math.pi / 2) / (rl * math.pi / 2)) < 1e-7
    assert abs(oracle.window(2, nyq - 1, nyq) - (nyq - 1) / nyq * 0.5 * (1 + math.cos(math.pi * (nyq - 1) / nyq))) < 1e-6


def test_grid_rule_and_bounds(oracle):
    # Ct/CtVolume.cpp:311-316, :370-373 for a 256x192 detector, FCD 1000 px
    assert oracle.cylinder_radius(256, 1000.0) == 126
    g = oracle.ref_geom(256, 192, 1000.0)
    assert (g.xSize, g.ySize, g.zSize) == (252, 252, 192)
    g = oracle.ref_geom(256, 192, 1000.0, rel=(0.25, 0.75, 0.25, 0.75, 0.25, 0.75))
    assert (g.xFrom, g.xTo, g.zFrom, g.zTo) == (63, 189, 48, 144)
    # setVolumeBounds clamps yTo and zTo against xFrom (reference quirk :496,498)
    assert oracle.clamp_bounds(0.6, 1.0, 0.1, 0.3, 0.0, 0.2) == pytest.approx((0.6, 1.0, 0.1, 0.6, 0.0, 0.6))
    assert oracle.clamp_bounds(0.5, 0.5, 0, 1, 0, 1) is None


def test_sinogram_fixups(oracle):
    # cw with increasing angles -> negated; heights relative and in pixels
    a, h = oracle.fix_sinogram([0, 1, 2], [1.0, 2.0, 3.0], ccw=False, pixel_size=0.5)
    assert list(a) == [0, -1, -2]
    assert list(h) == [-2.0, 0.0, 2.0]
    a, _ = oracle.fix_sinogram([0, 1, 2], [0, 0, 0], ccw=True, pixel_size=1.0)
    assert list(a) == [0, 1, 2]
    a, _ = oracle.fix_sinogram([2, 1, 0], [0, 0, 0], ccw=True, pixel_size=1.0)
    assert list(a) == [-2, -1, 0]


def test_fp64_oracle_agrees_with_fp32_restatement(oracle, golden_dir):
    g = load(golden_dir, "recon_tiny.npz")
    imgs, angles, FCD = g["imgs"], g["angles"], float(g["FCD"])
    V, H, W = imgs.shape
    geom = oracle.ref_geom(W, H, FCD)
    v64 = oracle.f64_reconstruct(imgs, angles, np.zeros(V), 1.0, oracle.RAMLAK, geom)
    err = oracle.rel_err(g["vol"], v64)
    assert err.rel_l2 < 1e-5, err


def test_padded_filter_is_linear_convolution(oracle):
    # pad=2: filtering a row equals the linear (non-circular) convolution restricted to W
    rng = np.random.default_rng(3)
    W, H = 24, 2
    img = rng.uniform(0.2, 1.0, (H, W)).astype(np.float32)
    p1 = oracle.f64_preprocess(img, 1.0, 100.0, oracle.RAMLAK, pad=1)
    p2 = oracle.f64_preprocess(img, 1.0, 100.0, oracle.RAMLAK, pad=2)
    assert not np.allclose(p1, p2)
    assert np.all(np.isfinite(p2))
