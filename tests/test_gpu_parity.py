"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

Bars: FP32 filtering <= 1e-5 relative per projection, FP32 backprojection
<= 1e-5 relative L2 on identical filtered input, end-to-end FP32 reconstruction
<= 1e-4 relative L2 against the reference's CPU path restated by the oracle,
FP16/BF16 storage <= 1e-3 relative L2 against the FP64 oracle.
"""
import math
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import ct_b200  # noqa: E402
from ct_b200 import CtVolume, ops, synth  # noqa: E402
from ct_b200 import _lib as L  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.init()


def np_phantom_images(V, H, W, FCD_px, pix_mm, n_ell=6, seed=0, photons=None, heights_mm=None, uoff_mm=0.0):
    from oracle import phantom
    geom = synth.ScanGeometry(V, W, H, pitch_mm=pix_mm * 2, sod_mm=FCD_px * pix_mm, sdd_mm=FCD_px * pix_mm * 2)
    r_mm, hz_mm = synth.fov(geom)
    ell = synth.random_ellipsoids(np.random.default_rng(seed), n_ell, r_mm, hz_mm, axes_mm=(0.1 * r_mm, 0.6 * r_mm))
    p = phantom.project(ell, geom.angles(), heights_mm, W, H, geom.pixel_eff, geom.sod_mm, uoff_mm)
    return synth.intensities_from_line_integrals(p, photons, seed), geom, ell


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


# ------------------------------------------------------------------ phantom
def test_phantom_kernel_matches_numpy():
    from oracle import phantom
    rng = np.random.default_rng(1)
    ell = synth.random_ellipsoids(rng, 5, 10.0, 8.0, axes_mm=(2.0, 8.0))
    ang = np.array([0.0, 33.0, 190.5])
    h = np.array([0.3, -0.2, 0.0])
    ref = phantom.project(ell, ang, h, 20, 16, 0.5, 60.0, 0.7)
    out = ops.phantom_project(ell, ang, h, 20, 16, 0.5, 60.0, 0.7).cpu().numpy()
    assert np.abs(out - ref).max() <= 1e-9 * max(1.0, np.abs(ref).max())


# ------------------------------------------------------------------ filter
@pytest.mark.parametrize("W", [16, 17, 64, 100, 255, 256])
@pytest.mark.parametrize("ft", [0, 1, 2])
def test_filter_fp32_matches_reference_path(oracle, W, ft):
    rng = np.random.default_rng(W * 10 + ft)
    V, H = 3, 7
    imgs = rng.integers(2000, 65535, size=(V, H, W)).astype(np.uint16)
    FCD = 4.0 * W
    det, _ = ops.detector(W, H, FCD)
    raw = torch.from_numpy(imgs.astype(np.int32)).to(torch.uint16).cuda()
    out = ops.filter_projections(raw, det, ft, 1, L.FP32).cpu().numpy()
    for v in range(V):
        ref = oracle.ref_preprocess(imgs[v], 1.0, FCD, ft)
        assert rel_l2(out[v], ref) < 1e-5, (v, rel_l2(out[v], ref))


@pytest.mark.parametrize("dtype", [np.uint8, np.float32])
def test_filter_other_depths(oracle, dtype):
    rng = np.random.default_rng(5)
    V, H, W = 2, 6, 48
    if dtype == np.uint8:
        imgs = rng.integers(10, 255, size=(V, H, W)).astype(np.uint8)
        raw = torch.from_numpy(imgs).cuda()
        base = 0.95
    else:
        imgs = rng.uniform(0.05, 1.0, size=(V, H, W)).astype(np.float32)
        raw = torch.from_numpy(imgs).cuda()
        base = 1.1
    det, _ = ops.detector(W, H, 200.0, base_intensity=base)
    out = ops.filter_projections(raw, det, 1, 1, L.FP32).cpu().numpy()
    for v in range(V):
        assert rel_l2(out[v], oracle.ref_preprocess(imgs[v], base, 200.0, 1)) < 1e-5


@pytest.mark.parametrize("W", [64, 100])
def test_filter_padded_matches_fp64_oracle(oracle, W):
    rng = np.random.default_rng(7)
    V, H = 2, 5
    imgs = rng.integers(2000, 65535, size=(V, H, W)).astype(np.uint16)
    det, _ = ops.detector(W, H, 500.0)
    raw = torch.from_numpy(imgs.astype(np.int32)).to(torch.uint16).cuda()
    out = ops.filter_projections(raw, det, 2, 2, L.FP32).cpu().numpy()
    for v in range(V):
        assert rel_l2(out[v], oracle.f64_preprocess(imgs[v], 1.0, 500.0, 2, pad=2)) < 1e-5


@pytest.mark.parametrize("store", [L.FP16, L.BF16])
def test_filter_half_storage(oracle, store):
    rng = np.random.default_rng(9)
    V, H, W = 2, 8, 128
    imgs = rng.integers(2000, 65535, size=(V, H, W)).astype(np.uint16)
    det, _ = ops.detector(W, H, 600.0)
    raw = torch.from_numpy(imgs.astype(np.int32)).to(torch.uint16).cuda()
    out = ops.filter_projections(raw, det, 0, 1, store, 1.0 / W).float().cpu().numpy() * W
    tol = 2e-3 if store == L.FP16 else 1e-2
    for v in range(V):
        assert rel_l2(out[v], oracle.f64_preprocess(imgs[v], 1.0, 600.0, 0)) < tol


# ----------------------------------------------------------- backprojection
def filtered_set(oracle, V=40, H=24, W=32, FCD=100.0, ft=0, seed=0):
    imgs, geom, _ = np_phantom_images(V, H, W, FCD, 0.5, seed=seed)
    proj = np.stack([oracle.ref_preprocess(im, 1.0, FCD, ft) for im in imgs])
    return imgs, proj, geom.angles()


def gpu_bp(proj, angles, heights, det, grid, z_begin=0, z_end=None, accumulate_into=None):
    t = torch.from_numpy(proj).cuda()
    out = None if accumulate_into is None else accumulate_into
    vol = ops.backproject(t, angles, heights, det, grid, z_begin, z_end, out=out,
                          accumulate=accumulate_into is not None)
    torch.cuda.synchronize()
    return vol.cpu().numpy()  # (Zs, Y, X)


def test_backproject_fp32_matches_reference_path(oracle):
    imgs, proj, ang = filtered_set(oracle)
    V, H, W = proj.shape
    det, grid = ops.detector(W, H, 100.0)
    og = oracle.ref_geom(W, H, 100.0)
    ref = oracle.ref_backproject(proj, ang, np.zeros(V), og)  # (x, y, z)
    out = gpu_bp(proj, ang, None, det, grid)
    assert rel_l2(out.transpose(2, 1, 0), ref) < 1e-5


def test_backproject_subbox_offsets_slabs(oracle):
    imgs, proj, ang = filtered_set(oracle, V=30, H=20, W=28, FCD=90.0, ft=2, seed=3)
    V, H, W = proj.shape
    rel = (0.2, 0.8, 0.1, 0.7, 0.25, 0.9)
    det, grid = ops.detector(W, H, 90.0, u_offset=1.25, rel=rel)
    og = oracle.ref_geom(W, H, 90.0, 1.25, rel=oracle.clamp_bounds(*rel))
    heights = np.linspace(-1.5, 1.5, V)
    ref = oracle.ref_backproject(proj, ang, heights, og)
    X, Y, Z = grid.box
    # three uneven slabs into one buffer
    vol = torch.zeros((Z, Y, X), device="cuda")
    cuts = [0, 3, 9, Z]
    for a, b in zip(cuts[:-1], cuts[1:]):
        ops.backproject(torch.from_numpy(proj).cuda(), ang, heights, det, grid, a, b, out=vol[a:b])
    out = vol.cpu().numpy()
    assert rel_l2(out.transpose(2, 1, 0), ref) < 1e-5
    # accumulate: two halves of the views add up to the whole
    half = V // 2
    acc = torch.zeros((Z, Y, X), device="cuda")
    pt = torch.from_numpy(proj).cuda()
    ops.backproject(pt[:half].contiguous(), ang[:half], heights[:half], det, grid, out=acc, accumulate=True)
    ops.backproject(pt[half:].contiguous(), ang[half:], heights[half:], det, grid, out=acc, accumulate=True)
    assert rel_l2(acc.cpu().numpy().transpose(2, 1, 0), ref) < 1e-5


def test_backproject_binned_grid(oracle):
    """Voxel pitch 2 detector pixels and a z extent beyond the detector (grid extension)."""
    imgs, proj, ang = filtered_set(oracle, V=24, H=16, W=40, FCD=150.0, seed=4)
    V, H, W = proj.shape
    det, _ = ops.detector(W, H, 150.0)
    grid = ops.custom_grid(det, (20, 22, 12), 2.0)
    og = oracle.custom_geom(W, H, 150.0, (20, 22, 12), 2.0)
    ref = oracle.ref_backproject(proj, ang, np.zeros(V), og)
    out = gpu_bp(proj, ang, None, det, grid)
    assert rel_l2(out.transpose(2, 1, 0), ref) < 1e-5


# ---------------------------------------------------------------- end to end
def c1_scan(tmp_path, n_views=360, W=256, H=192, seed=11):
    """360 views over 360 deg, 256x192 at 1.0 mm pitch, SOD 500, SDD 1000, 10 ellipsoids."""
    geom = synth.ScanGeometry(n_views, W, H, pitch_mm=1.0, sod_mm=500.0, sdd_mm=1000.0)
    scan = synth.make_scan(geom, 10, seed)
    imgs = scan.images.cpu().numpy()
    csv = synth.write_scan(str(tmp_path), imgs, geom)
    return csv, imgs, geom


def test_c1_end_to_end_matches_reference_path(oracle, tmp_path):
    csv, imgs, geom = c1_scan(tmp_path)
    v = CtVolume(csv)
    assert (v.getXSize(), v.getYSize(), v.getZSize()) == (252, 252, 192)
    v.reconstructVolume()
    out = v.volume(L.Z_FASTEST)
    og = oracle.ref_geom(geom.width, geom.height, v.getFCD())
    ref, secs = oracle.ref_reconstruct(imgs, geom.angles(), np.zeros(geom.n_views), 1.0, oracle.RAMLAK, og)
    err = rel_l2(out, ref)
    print(f"360 x 256x192 scan, rel-L2 vs reference CPU path: {err:.3e} (CPU {secs:.2f} s)")
    assert err <= 1e-4


def test_save_formats(oracle, tmp_path):
    csv, imgs, geom = c1_scan(tmp_path, n_views=24, W=64, H=40)
    v = CtVolume(csv)
    v.setVolumeBounds(0.1, 0.9, 0.2, 0.8, 0.0, 0.5)
    v.setFrequencyFilterType("shepplogan")
    v.reconstructVolume()
    X, Y, Z = v.grid().box
    zf = v.volume(L.Z_FASTEST)
    for order, endian in [(L.Z_FASTEST, L.LITTLE_ENDIAN), (L.X_FASTEST, L.BIG_ENDIAN),
                          (L.Z_FASTEST, L.BIG_ENDIAN), (L.X_FASTEST, L.LITTLE_ENDIAN)]:
        path = tmp_path / f"vol_{order}_{endian}.raw"
        v.saveVolumeToBinaryFile(str(path), order, endian)
        data = np.fromfile(path, dtype=">f4" if endian == L.BIG_ENDIAN else "<f4")
        expect = zf.ravel() if order == L.Z_FASTEST else zf.transpose(2, 1, 0).ravel()
        assert np.array_equal(data.astype(np.float32), expect)
        info = (tmp_path / f"vol_{order}_{endian}.txt").read_text()
        assert f"X size:\t\t\t\t{X}\n" in info and "32bit IEEE 754 float" in info
        assert ("Z fastest" if order == L.Z_FASTEST else "X fastest") in info
        vgi = (tmp_path / f"vol_{order}_{endian}.vgi").read_text()
        assert f"size = {X} {Y} {Z}" in vgi and f"Name = ./vol_{order}_{endian}.raw" in vgi
    # reconstructInto gives the same bytes as the kept volume, both orders
    buf = np.empty(X * Y * Z, np.float32)
    v.reconstructInto(buf.ctypes.data, L.Z_FASTEST)
    assert np.array_equal(buf, zf.ravel())
    v.reconstructInto(buf.ctypes.data, L.X_FASTEST)
    assert np.array_equal(buf, zf.transpose(2, 1, 0).ravel())


def test_skip_projections_and_progress(oracle, tmp_path):
    csv, imgs, geom = c1_scan(tmp_path, n_views=30, W=48, H=32)
    v = CtVolume(csv)
    seen = []
    v.setProgressCallback(lambda s, p: seen.append((s, p)))
    v.setSkipProjections(2)
    v.setSlabHeight(16)
    v.reconstructVolume()
    out = v.volume(L.Z_FASTEST)
    og = oracle.ref_geom(48, 32, v.getFCD())
    ref, _ = oracle.ref_reconstruct(imgs, geom.angles(), np.zeros(30), 1.0, 0, og, step=3)
    assert rel_l2(out, ref) <= 1e-4
    assert seen and seen[-1] == (1, 100.0)


@pytest.mark.parametrize("store", ["fp16", "bf16"])
def test_mixed_precision_vs_fp64_oracle(oracle, tmp_path, store):
    csv, imgs, geom = c1_scan(tmp_path, n_views=120, W=128, H=96, seed=5)
    v = CtVolume(csv)
    v.setFrequencyFilterType("hann")
    v.setPrecision(store)
    v.reconstructVolume()
    out = v.volume(L.Z_FASTEST)
    og = oracle.ref_geom(128, 96, v.getFCD())
    ref = oracle.f64_reconstruct(imgs, geom.angles(), np.zeros(120), 1.0, oracle.HANN, og)
    err = rel_l2(out, ref)
    print(f"{store} rel-L2 vs FP64 oracle: {err:.3e}")
    assert err <= 1e-3


# ------------------------------------------------------------ adjoint pair
def adjoint_case(V=36, H=20, W=30, grid_size=None, vs=1.0, rel=None, uoff=0.0, heights=False, seed=0):
    rng = np.random.default_rng(seed)
    det, grid = ops.detector(W, H, 120.0, u_offset=uoff, rel=rel)
    if grid_size is not None:
        grid = ops.custom_grid(det, grid_size, vs)
    ang = np.sort(rng.uniform(0, 360, V))
    h = rng.uniform(-2, 2, V) if heights else np.zeros(V)
    X, Y, Z = grid.box
    x = torch.from_numpy(rng.standard_normal((Z, Y, X)).astype(np.float32)).cuda()
    y = torch.from_numpy(rng.standard_normal((V, H, W)).astype(np.float32)).cuda()
    return det, grid, ang, h, x, y


@pytest.mark.parametrize("case", [
    dict(),
    dict(rel=(0.1, 0.9, 0.2, 0.7, 0.3, 1.0), uoff=0.8, heights=True),
    dict(grid_size=(14, 16, 18), vs=2.0),
    dict(grid_size=(25, 21, 9), vs=1.3, heights=True),
    dict(V=50, H=33, W=47, seed=2),
    # tall slabs of fine slices: the forward projector's walk with the slice
    # spacing at run time (rows 0.3 apart, spacing 4) and at spacing 2 (rows
    # 0.7 apart), both with more steps per column than it preloads
    dict(V=12, H=120, W=24, grid_size=(8, 8, 320), vs=0.3, seed=3),
    dict(V=12, H=250, W=16, grid_size=(6, 6, 340), vs=0.7, heights=True, seed=4),
])
def test_dot_product_adjoint(case):
    det, grid, ang, h, x, y = adjoint_case(**case)
    Ax = ops.forward_project(x, ang, h, det, grid)
    Aty = ops.backproject(y, ang, h, det, grid)
    torch.cuda.synchronize()
    lhs = float((Ax.double() * y.double()).sum())
    rhs = float((x.double() * Aty.double()).sum())
    assert abs(lhs - rhs) <= 1e-5 * max(abs(lhs), abs(rhs)), (lhs, rhs)


def test_forward_slabs_accumulate():
    det, grid, ang, h, x, y = adjoint_case(heights=True)
    full = ops.forward_project(x, ang, h, det, grid)
    Z = grid.box[2]
    acc = torch.zeros_like(full)
    for a, b in [(0, 5), (5, 11), (11, Z)]:
        ops.forward_project(x[a:b].contiguous(), ang, h, det, grid, a, b, out=acc, accumulate=True)
    torch.cuda.synchronize()
    assert torch.allclose(acc, full, rtol=1e-5, atol=1e-5)


def test_adjoint_in_uneven_slabs():
    """Backprojection of slabs that start off a multiple of the tile height (the staged kernel
    shifts its tiles and skips the slices before the slab) against the whole-box launch,
    slice for slice, and the dot test with both operators run slab by slab."""
    det, grid, ang, h, x, y = adjoint_case(V=24, H=40, W=36, grid_size=(20, 18, 70), vs=1.0, heights=True, seed=9)
    Z = grid.box[2]
    cuts = [0, 5, 13, 37, 41, Z]
    whole = ops.backproject(y, ang, h, det, grid)
    Aty = torch.zeros_like(whole)
    Ax = torch.zeros_like(y)
    for a, b in zip(cuts[:-1], cuts[1:]):
        ops.backproject(y, ang, h, det, grid, a, b, out=Aty[a:b])
        ops.forward_project(x[a:b].contiguous(), ang, h, det, grid, a, b, out=Ax, accumulate=True)
    torch.cuda.synchronize()
    assert rel_l2(Aty.cpu().numpy(), whole.cpu().numpy()) <= 1e-6
    lhs = float((Ax.double() * y.double()).sum())
    rhs = float((x.double() * Aty.double()).sum())
    assert abs(lhs - rhs) <= 1e-5 * max(abs(lhs), abs(rhs)), (lhs, rhs)


def test_gradient_finite_differences():
    """grad ||Ax - p||^2 = 2 A^T (Ax - p), checked on 64 random voxels by central differences."""
    det, grid, ang, h, x, p = adjoint_case(V=30, H=18, W=26, seed=4)
    rng = np.random.default_rng(8)
    r = ops.forward_project(x, ang, h, det, grid) - p
    g = 2.0 * ops.backproject(r.contiguous(), ang, h, det, grid)
    Z, Y, X = x.shape
    idx = [(int(rng.integers(Z)), int(rng.integers(Y)), int(rng.integers(X))) for _ in range(64)]
    base = ops.forward_project(x, ang, h, det, grid).double()
    eps = 0.5
    for (k, j, i) in idx:
        xp = x.clone(); xp[k, j, i] += eps
        xm = x.clone(); xm[k, j, i] -= eps
        fp = ops.forward_project(xp, ang, h, det, grid).double() - p.double()
        fm = ops.forward_project(xm, ang, h, det, grid).double() - p.double()
        fd = float(((fp * fp) - (fm * fm)).sum()) / (2 * eps)
        gi = float(g[k, j, i])
        assert abs(fd - gi) <= 1e-4 * max(1.0, abs(fd)), ((k, j, i), fd, gi)
    del base


def test_save_load_round_trip_and_cross_sections(tmp_path):
    from ct_b200 import load_volume, read_volume_info
    csv, imgs, geom = c1_scan(tmp_path, n_views=20, W=48, H=36)
    v = CtVolume(csv)
    v.setVolumeBounds(0.0, 1.0, 0.1, 0.9, 0.2, 0.8)
    v.reconstructVolume()
    zyx = v.volume(L.X_FASTEST)
    for order, endian in [(L.Z_FASTEST, L.BIG_ENDIAN), (L.X_FASTEST, L.LITTLE_ENDIAN)]:
        raw = tmp_path / f"rt_{order}_{endian}.raw"
        v.saveVolumeToBinaryFile(str(raw), order, endian)
        info = read_volume_info(tmp_path / f"rt_{order}_{endian}.txt")
        assert (info["x"], info["y"], info["z"]) == v.grid().box
        assert (info["index_order"], info["byte_order"]) == (order, endian)
        back = load_volume(raw, info["x"], info["y"], info["z"], info["index_order"], info["byte_order"])
        assert np.array_equal(back, zyx)
    Z, Y, X = zyx.shape
    # left-handed cross sections (Common/Volume.h:577-648)
    assert np.array_equal(v.getVolumeCrossSection(2, Z // 2), zyx[Z // 2].T)             # rows x, cols y
    assert np.array_equal(v.getVolumeCrossSection(0, X // 3), zyx[::-1, :, X // 3])       # rows z (flipped), cols y
    assert np.array_equal(v.getVolumeCrossSection(1, Y // 2), zyx[::-1, Y // 2, ::-1])    # rows z (flipped), cols x (flipped)


def test_progress_previews(tmp_path):
    """Previews after every slab show the finished slabs and zeros elsewhere; the last one is the
    finished volume's cross section (reconstructionProgress / reconstructionFinished)."""
    csv, imgs, geom = c1_scan(tmp_path, n_views=40, W=64, H=64)
    v = CtVolume(csv)
    v.setSlabHeight(16)
    v.setCrossSectionAxis(ct_b200.AXIS_Y)
    seen = []
    v.setPreviewCallback(lambda pct, sec: seen.append((pct, sec)))
    v.reconstructVolume()
    final = v.getVolumeCrossSection(ct_b200.AXIS_Y, v.getCrossSectionIndex())
    Z = v.getZSize()
    assert len(seen) >= Z // 16
    assert seen[-1][0] == 100.0 and np.array_equal(seen[-1][1], final)
    assert all(b[0] >= a[0] for a, b in zip(seen, seen[1:]))
    # first preview (after slab 1 was issued): slab 0 finished, the rest still zero; rows run z = Z-1 .. 0
    first = seen[0][1]
    assert np.array_equal(first[Z - 16:], final[Z - 16:])
    assert not first[:Z - 32].any()


TRANSPOSE_SCRIPT = r"""
import sys, numpy as np, torch
sys.path.insert(0, %r)
from ct_b200 import ops
vs, uoff, heights, out = float(sys.argv[1]), float(sys.argv[2]), sys.argv[3] == "1", sys.argv[4]
V, H, W, n = 3, 14, 16, 6
rng = np.random.default_rng(int(vs * 10))
det, _ = ops.detector(W, H, 40.0, u_offset=uoff)
grid = ops.custom_grid(det, (n, n, n), vs)
ang = rng.uniform(0, 360, V)
h = rng.uniform(-1.5, 1.5, V) if heights else None
A = np.zeros((V * H * W, n * n * n))
for k in range(n * n * n):
    e = torch.zeros(n * n * n, device="cuda")
    e[k] = 1.0
    A[:, k] = ops.forward_project(e.view(n, n, n), ang, h, det, grid).cpu().numpy().ravel()
At = np.zeros((n * n * n, V * H * W))
for k in range(V * H * W):
    e = torch.zeros(V * H * W, device="cuda")
    e[k] = 1.0
    At[:, k] = ops.backproject(e.view(V, H, W), ang, h, det, grid).cpu().numpy().ravel()
np.save(out + "_A.npy", A)
np.save(out + "_At.npy", At)
"""


def transpose_matrices(tmp_path, variant, vs, uoff, heights):
    """A (forward projector, unit volumes) and A^T (backprojector forced to `variant`, unit pixels)."""
    import subprocess
    import sys
    out = str(tmp_path / f"{variant}_{vs}")
    env = dict(os.environ, CTB_BP_VARIANT=variant)
    r = subprocess.run([sys.executable, "-c", TRANSPOSE_SCRIPT % ROOT, str(vs), str(uoff), "1" if heights else "0",
                        out], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    return np.load(out + "_A.npy"), np.load(out + "_At.npy")


@pytest.mark.parametrize("vs,uoff,heights", [(1.0, 0.0, False), (0.6, 1.5, True), (2.5, -2.0, False)])
def test_forward_is_the_exact_transpose(tmp_path, vs, uoff, heights):
    """Every matrix element: A e_voxel (forward projector) against A^T e_pixel, with the
    backprojector forced to the global-gather kernel and to the shared-memory one (its pair loop
    and per-voxel loops): all form rows the same way and take the same decisions."""
    A, At = transpose_matrices(tmp_path, "global", vs, uoff, heights)
    assert np.count_nonzero(A) > 100
    assert np.array_equal(A != 0, At.T != 0)
    np.testing.assert_allclose(A, At.T, rtol=1e-6, atol=1e-7)
    A2, At2 = transpose_matrices(tmp_path, "tma", vs, uoff, heights)
    assert np.array_equal(A2, A)
    assert np.array_equal(A != 0, At2.T != 0)
    np.testing.assert_allclose(A, At2.T, rtol=1e-6, atol=1e-7)


def test_emit_signals_off_silences_callbacks(tmp_path):
    csv, imgs, geom = c1_scan(tmp_path, n_views=20, W=48, H=32)
    v = CtVolume(csv)
    seen = []
    v.setProgressCallback(lambda s, p: seen.append(p))
    v.setPreviewCallback(lambda p, sec: seen.append(p))
    v.setEmitSignals(False)
    v.reconstructVolume()
    assert seen == []
    v.setEmitSignals(True)
    v.reconstructVolume()
    assert seen and seen[-1] == 100.0


@pytest.mark.parametrize("V,H,W,FCD", [(24, 20, 32, 120.0), (24, 20, 64, 240.0), (36, 18, 40, 90.0)])
def test_row_bounds_decided_as_the_reference(oracle, V, H, W, FCD):
    """Geometries where voxels of the first and last slices project exactly onto the detector's
    row bounds (v == H/2 at 180 degrees): membership must follow the reference's own v test, else
    whole rows of voxels gain or lose a boundary sample (filtered noise makes that visible)."""
    rng = np.random.default_rng(V + H + W)
    imgs = rng.integers(20000, 65535, size=(V, H, W)).astype(np.uint16)
    angles = np.arange(V) * (360.0 / V)
    det, grid = ops.detector(W, H, FCD)
    raw = torch.from_numpy(imgs.astype(np.int32)).to(torch.uint16).cuda()
    filt = ops.filter_projections(raw, det, L.RAMLAK, 1, L.FP32)
    vol = ops.backproject(filt, angles, None, det, grid)
    torch.cuda.synchronize()
    og = oracle.ref_geom(W, H, FCD)
    ref, _ = oracle.ref_reconstruct(imgs, angles, np.zeros(V), 1.0, oracle.RAMLAK, og)
    assert rel_l2(vol.cpu().numpy().transpose(2, 1, 0), ref) < 1e-5


def test_smoke_entry_point():
    """The build's own smoke check (one small reconstruction against the CPU oracle)."""
    import sys
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    import __graft_entry__
    __graft_entry__.smoke()


def _random_case(k):
    rng = np.random.default_rng(1000 + k)
    W = int(rng.integers(16, 97))
    H = int(rng.integers(8, 65))
    FCD = float(rng.uniform(2.0, 6.0) * W)
    V = int(rng.integers(4, 41))
    angles = np.arange(V) * (360.0 / V) if k % 2 == 0 else np.sort(rng.uniform(0, 360, V))
    uoff = float(rng.choice([0.0, 2.5, -1.75]))
    heights = rng.uniform(-2.0, 2.0, V) if k % 3 == 0 else np.zeros(V)
    heights = heights - heights.mean()
    lo = rng.uniform(0.0, 0.4, 3)
    hi = rng.uniform(0.6, 1.0, 3)
    rel = (lo[0], hi[0], lo[1], hi[1], lo[2], hi[2]) if k % 4 == 1 else (0, 1, 0, 1, 0, 1)
    ft = int(k % 3)
    imgs = rng.integers(2000, 65535, size=(V, H, W)).astype(np.uint16)
    return W, H, FCD, angles, uoff, heights, rel, ft, imgs


@pytest.mark.parametrize("k", range(16))
def test_random_geometries_match_reference_path(oracle, k):
    """Seeded random detectors, orbits, u offsets, height offsets, sub-boxes and filters on noise
    projections (the input on which any boundary decision that differs from the reference's
    shows): the FP32 engine against the reference's CPU path restated."""
    W, H, FCD, angles, uoff, heights, rel, ft, imgs = _random_case(k)
    V = len(angles)
    rel_c = oracle.clamp_bounds(*rel)
    det, grid = ops.detector(W, H, FCD, u_offset=uoff, rel=rel)
    raw = torch.from_numpy(imgs.astype(np.int32)).to(torch.uint16).cuda()
    filt = ops.filter_projections(raw, det, ft, 1, L.FP32)
    vol = ops.backproject(filt, angles, heights, det, grid)
    torch.cuda.synchronize()
    og = oracle.ref_geom(W, H, FCD, uoff, rel=rel_c)
    ref, _ = oracle.ref_reconstruct(imgs, angles, heights, 1.0, ft, og)
    err = rel_l2(vol.cpu().numpy().transpose(2, 1, 0), ref)
    assert err < 2e-5, err


@pytest.mark.parametrize("k", range(6))
def test_random_scans_through_the_facade(oracle, tmp_path, k):
    """CSV scans with cw/ccw orbits, decreasing angles, height offsets in mm, u offsets, bounds,
    skipped projections and all filters, read and reconstructed by the facade, against the
    reference's CPU path restated (Ct/CtVolume.cpp:136-330, :543-632, :742-767, :923-1054)."""
    rng = np.random.default_rng(2000 + k)
    V, W, H = int(rng.integers(8, 40)), int(rng.integers(24, 80)), int(rng.integers(12, 48))
    geom = synth.ScanGeometry(V, W, H, pitch_mm=float(rng.uniform(0.2, 1.0)), sod_mm=float(rng.uniform(300, 600)),
                              sdd_mm=float(rng.uniform(700, 1200)), u_offset_mm=float(rng.choice([0.0, 0.7, -1.3])))
    rotation = "ccw" if k % 2 else "cw"
    angles = np.arange(V) * (360.0 / V)
    if k % 3 == 2:
        angles = angles[::-1].copy()
    heights = rng.uniform(-3, 3, V) if k % 2 == 0 else None
    imgs = rng.integers(3000, 65535, size=(V, H, W)).astype(np.uint16)
    csv = synth.write_scan(str(tmp_path), imgs, geom, rotation=rotation, heights_mm=heights, angles_deg=angles)
    rel = (0.0, 1.0, 0.1, 0.9, 0.2, 0.85) if k % 2 else (0.0, 1.0, 0.0, 1.0, 0.0, 1.0)
    ft, skip = k % 3, int(k % 4 == 3)
    v = CtVolume(csv)
    v.setVolumeBounds(*rel)
    v.setFrequencyFilterType(ft)
    v.setSkipProjections(skip)
    v.reconstructVolume()
    out = v.volume(L.Z_FASTEST)
    pix = v.getPixelSize()
    a, h = oracle.fix_sinogram(angles, np.zeros(V) if heights is None else heights, rotation == "ccw", pix)
    og = oracle.ref_geom(W, H, v.getFCD(), v.getUOffset(), rel=oracle.clamp_bounds(*rel))
    ref, _ = oracle.ref_reconstruct(imgs, a, h, 1.0, ft, og, step=skip + 1)
    assert out.shape == ref.shape
    err = rel_l2(out, ref)
    assert err < 2e-5, err


@pytest.mark.parametrize("order", [L.X_FASTEST, L.Z_FASTEST])
def test_slab_schedules_agree(tmp_path, order):
    """The facade pipeline under different slab heights: one slab; slabs of 64 (the first two
    backprojected while the views upload, three slab buffers, the last slab cut to 32 slices);
    slabs of 16. The volumes agree to rounding (the early slabs sum the views chunk by chunk)."""
    rng = np.random.default_rng(77)
    V, W, H = 40, 48, 192
    geom = synth.ScanGeometry(V, W, H, pitch_mm=0.5, sod_mm=400.0, sdd_mm=900.0)
    imgs = rng.integers(3000, 65535, size=(V, H, W)).astype(np.uint16)
    csv = synth.write_scan(str(tmp_path), imgs, geom)
    vols = {}
    for slab in (H, 64, 16):
        v = CtVolume(csv)
        v.setSlabHeight(slab)
        X, Y, Z = v.grid().box
        assert Z == H
        buf = np.empty(X * Y * Z, np.float32)   # pageable: staged through pinned buffers
        v.reconstructInto(buf.ctypes.data, order)
        vols[slab] = buf
    assert np.abs(vols[H]).max() > 0
    for slab in (64, 16):
        assert rel_l2(vols[slab], vols[H]) < 2e-6, slab


def test_row_band_of_a_z_sub_box(tmp_path):
    """A z sub-box uploads and filters only the detector rows its slices reach (the
    timings count the bytes); its slices equal the same slices of the whole box."""
    rng = np.random.default_rng(78)
    V, W, H = 36, 64, 160
    geom = synth.ScanGeometry(V, W, H, pitch_mm=0.5, sod_mm=400.0, sdd_mm=900.0)
    imgs = rng.integers(3000, 65535, size=(V, H, W)).astype(np.uint16)
    csv = synth.write_scan(str(tmp_path), imgs, geom)
    full = CtVolume(csv)
    full.reconstructVolume()
    ref = full.volume(L.X_FASTEST)                  # (Z, Y, X)
    t_full = full.timings()
    assert t_full.h2d_bytes == V * H * W * 2
    sub = CtVolume(csv)
    sub.setVolumeBounds(0.0, 1.0, 0.0, 1.0, 0.4, 0.6)
    sub.reconstructVolume()
    g = sub.grid()
    out = sub.volume(L.X_FASTEST)
    t_sub = sub.timings()
    assert 0 < t_sub.h2d_bytes < 0.5 * V * H * W * 2
    assert t_sub.d2h_bytes == out.size * 4
    # the row coordinates are rounded from another origin (box z index, band row),
    # which on noise projections moves the sums by about 1e-5 relative
    assert rel_l2(out, ref[g.z_from:g.z_to]) < 2e-5
