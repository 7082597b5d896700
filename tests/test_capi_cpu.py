"""C ABI checks that need no GPU: the library loads, exports every function
include/ctb.h declares, and the host-side logic (CSV ingest, image decoding,
grid rule, bounds) follows the reference."""
import ctypes
import os
import re

import numpy as np
import pytest

import ct_b200
from ct_b200 import CtbError, CtVolume, synth
from ct_b200 import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "ctb.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(ctb_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(L.LIB_PATH)
    names = declared_functions()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # and the Python binding declares a signature for each of them
    assert set(names) <= set(L.SIGNATURES), set(names) - set(L.SIGNATURES)


def test_reference_grid_matches_oracle(oracle):
    from ct_b200 import ops
    for W, H, D in [(256, 192, 1000.0), (1024, 1024, 2500.0), (2048, 2048, 5000.0), (300, 77, 301.5)]:
        d, g = ops.detector(W, H, D)
        og = oracle.ref_geom(W, H, D)
        assert (g.x_size, g.y_size, g.z_size) == (og.xSize, og.ySize, og.zSize)
        assert d.radius == og.radius
    d, g = ops.detector(256, 192, 1000.0, rel=(0.25, 0.75, 0.1, 0.3, 0.0, 0.2))
    og = oracle.ref_geom(256, 192, 1000.0, rel=oracle.clamp_bounds(0.25, 0.75, 0.1, 0.3, 0.0, 0.2))
    assert (g.x_from, g.x_to, g.y_from, g.y_to, g.z_from, g.z_to) == (
        og.xFrom, og.xTo, og.yFrom, og.yTo, og.zFrom, og.zTo)


def write_scan(tmp_path, V=6, H=8, W=12, rotation="ccw", heights=None, angles=None):
    geom = synth.ScanGeometry(V, W, H, pitch_mm=1.0, sod_mm=100.0, sdd_mm=200.0)
    imgs = np.random.default_rng(0).integers(1000, 60000, (V, H, W)).astype(np.uint16)
    csv = synth.write_scan(str(tmp_path), imgs, geom, rotation=rotation, heights_mm=heights, angles_deg=angles)
    return csv, imgs, geom


def test_csv_ingest_geometry(tmp_path, oracle):
    csv, imgs, geom = write_scan(tmp_path, heights=[0.0, 0.5, 1.0, 1.5, 2.0, 2.5])
    v = CtVolume(csv)
    assert v.getSinogramSize() == 6
    assert (v.getImageWidth(), v.getImageHeight()) == (12, 8)
    # FCD / pixelSize in float (Ct/CtVolume.cpp:170)
    assert v.getFCD() == np.float32(100.0) / np.float32(0.5)
    assert v.getPixelSize() == pytest.approx(0.5)
    og = oracle.ref_geom(12, 8, float(np.float32(100.0) / np.float32(0.5)))
    assert (v.getXSize(), v.getYSize(), v.getZSize()) == (og.xSize, og.ySize, og.zSize)
    v.setVolumeBounds(0.25, 0.75, 0.0, 1.0, 0.5, 1.0)
    g = v.grid()
    assert (g.x_from, g.x_to, g.z_from, g.z_to) == (int(0.25 * og.xSize + 0.5), int(0.75 * og.xSize + 0.5), 4, 8)


def test_cross_section_settings(tmp_path):
    """setCrossSectionAxis / Index and their re-centring (Ct/CtVolume.cpp:317-326, :395-429, :1411-1417)."""
    from ct_b200 import AXIS_X, AXIS_Y, AXIS_Z
    csv, imgs, geom = write_scan(tmp_path)
    v = CtVolume(csv)
    X, Y, Z = v.getXSize(), v.getYSize(), v.getZSize()
    assert (v.getCrossSectionAxis(), v.getCrossSectionIndex(), v.getCrossSectionSize()) == (AXIS_Z, Z // 2, Z)
    v.setCrossSectionAxis(AXIS_X)
    assert (v.getCrossSectionIndex(), v.getCrossSectionSize()) == (X // 2, X)
    v.setCrossSectionIndex(X - 1)
    assert v.getCrossSectionIndex() == X - 1
    v.setCrossSectionIndex(X)            # outside the box: ignored
    assert v.getCrossSectionIndex() == X - 1
    v.setVolumeBounds(0.0, 0.5, 0.0, 1.0, 0.0, 1.0)
    g = v.grid()
    assert v.getCrossSectionIndex() == (g.x_to - g.x_from) // 2   # clamped into the smaller box
    v.setCrossSectionAxis(AXIS_Y)
    assert v.getCrossSectionIndex() == Y // 2


def test_csv_tiff_and_png_decoding(tmp_path):
    """Same pixels through PGM, TIFF (II and MM) and PNG give the same detector data."""
    import zlib, struct
    from ct_b200 import ops  # noqa: F401
    H, W = 5, 7
    img = np.arange(H * W, dtype=np.uint16).reshape(H, W) * 997
    d = tmp_path / "imgs"
    d.mkdir()

    def tiff(path, a, be):
        e = ">" if be else "<"
        data = a.astype(e + "u2").tobytes()
        ntags = 8
        ifd_off = 8
        data_off = ifd_off + 2 + ntags * 12 + 4
        tags = [(256, 3, 1, W), (257, 3, 1, H), (258, 3, 1, 16), (259, 3, 1, 1), (262, 3, 1, 1),
                (273, 4, 1, data_off), (278, 3, 1, H), (279, 4, 1, len(data))]
        out = (b"MM" if be else b"II") + struct.pack(e + "HI", 42, ifd_off) + struct.pack(e + "H", ntags)
        for tag, typ, cnt, val in tags:
            if typ == 3:
                out += struct.pack(e + "HHIHH", tag, typ, cnt, val, 0)
            else:
                out += struct.pack(e + "HHII", tag, typ, cnt, val)
        out += struct.pack(e + "I", 0) + data
        open(path, "wb").write(out)

    def png(path, a):
        raw = b"".join(b"\x00" + row.astype(">u2").tobytes() for row in a)
        def chunk(t, b):
            return struct.pack(">I", len(b)) + t + b + struct.pack(">I", zlib.crc32(t + b) & 0xffffffff)
        ihdr = struct.pack(">IIBBBBB", W, H, 16, 0, 0, 0, 0)
        open(path, "wb").write(b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", ihdr) + chunk(b"IDAT", zlib.compress(raw)) +
                               chunk(b"IEND", b""))

    synth.write_pgm16(str(d / "a.pgm"), img)
    tiff(str(d / "b.tif"), img, False)
    tiff(str(d / "c.tif"), img, True)
    png(str(d / "d.png"), img)
    csv = tmp_path / "s.csv"
    csv.write_text("imgs\n0.5\nccw\n0\n100\n1\nx\na.pgm\t0\nb.tif\t90\nc.tif\t180\nd.png\t270\n")
    v = CtVolume(str(csv))
    assert v.getSinogramSize() == 4


@pytest.mark.parametrize("body,needle", [
    ("imgs\nabc\nccw\n0\n100\n1\nx\na.pgm\t0\n", "Could not read the parameters"),
    ("imgs\n0.5\nccw\n0\n100\n0\nx\na.pgm\t0\n", "base intensity"),
    ("imgs\n0.5\nccw\n0\n100\n1\nx\n", "does not contain any images"),
    ("imgs\n0.5\nccw\n0\n100\n1\nx\na.pgm\tzero\n", "image parameters"),
    ("imgs\n0.5\nccw\n0\n100\n1\nx\nmissing.pgm\t0\n", "Error loading the image"),
    ("imgs\n0.5\nccw\n0\n3\n1\nx\na.pgm\t0\n", "FCD must be greater than the image width"),
    ("imgs\n0.5\nccw\n0\n100\n1\nx\na.pgm\t0\nsmall.pgm\t1\n", "dimensions differ"),
])
def test_csv_error_branches(tmp_path, body, needle):
    d = tmp_path / "imgs"
    d.mkdir()
    synth.write_pgm16(str(d / "a.pgm"), np.full((4, 6), 1000, np.uint16))
    synth.write_pgm16(str(d / "small.pgm"), np.full((3, 6), 1000, np.uint16))
    csv = tmp_path / "s.csv"
    csv.write_text(body)
    with pytest.raises(CtbError) as e:
        CtVolume(str(csv))
    assert needle in e.value.message


def test_csv_direction_and_heights(tmp_path):
    """cw + increasing angles are negated; blank lines repeat the previous image (reference quirk)."""
    d = tmp_path / "imgs"
    d.mkdir()
    synth.write_pgm16(str(d / "a.pgm"), np.full((4, 6), 1000, np.uint16))
    csv = tmp_path / "s.csv"
    csv.write_text("imgs\n0.5\ncw\n0\n100\n1\nx\na.pgm\t0\t1\na.pgm\t10\t2\n\na.pgm\t20\n")
    v = CtVolume(str(csv))
    assert v.getSinogramSize() == 4


def test_missing_library_fails_loudly(monkeypatch):
    monkeypatch.setattr(L, "_lib", None)
    monkeypatch.setattr(L, "LIB_PATH", "/nonexistent/libctb.so")
    with pytest.raises(RuntimeError):
        L.lib()


@pytest.mark.parametrize("depth", [np.uint8, np.uint16])
def test_read_image_matches_cv2(tmp_path, depth):
    """Projection images decoded as cv::imread(IMREAD_GRAYSCALE | IMREAD_ANYDEPTH) does: gray as is,
    colour TIFF through cvtColor's 14-bit gray formula (bit-exact), colour PNG within the LSBs by which
    libpng's own conversion differs from that formula, gray + alpha PNG without its alpha."""
    cv2 = pytest.importorskip("cv2")
    from ct_b200.ctvolume import read_image
    rng = np.random.default_rng(int(np.iinfo(depth).max))
    top = np.iinfo(depth).max
    gray = rng.integers(0, top + 1, (23, 31)).astype(depth)
    color = rng.integers(0, top + 1, (23, 31, 3)).astype(depth)      # BGR for cv2
    rgba = rng.integers(0, top + 1, (23, 31, 4)).astype(depth)
    flags = cv2.IMREAD_GRAYSCALE | cv2.IMREAD_ANYDEPTH
    for name, img, ext, tol in [("g", gray, "png", 0), ("g", gray, "tif", 0), ("c", color, "tif", 0),
                                ("a", rgba, "tif", 0), ("c", color, "png", 4), ("a", rgba, "png", 4)]:
        path = str(tmp_path / f"{name}.{ext}")
        params = [cv2.IMWRITE_TIFF_COMPRESSION, 1] if ext == "tif" else []   # uncompressed
        assert cv2.imwrite(path, img, params)
        ref = cv2.imread(path, flags)
        got = read_image(path)
        assert got.dtype == ref.dtype and got.shape == ref.shape, (name, ext)
        diff = np.abs(got.astype(np.int64) - ref.astype(np.int64)).max()
        assert diff <= tol, (name, ext, diff)
    # gray + alpha PNG written by hand (cv2 writes no 2-channel PNG)
    import struct
    import zlib
    ga = np.stack([gray, rng.integers(0, top + 1, gray.shape).astype(depth)], -1)
    be = ">u2" if depth == np.uint16 else "u1"
    raw = b"".join(b"\x00" + row.astype(be).tobytes() for row in ga)

    def chunk(t, b):
        return struct.pack(">I", len(b)) + t + b + struct.pack(">I", zlib.crc32(t + b) & 0xffffffff)
    ihdr = struct.pack(">IIBBBBB", gray.shape[1], gray.shape[0], 8 * np.dtype(depth).itemsize, 4, 0, 0, 0)
    path = str(tmp_path / "ga.png")
    open(path, "wb").write(b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", ihdr) + chunk(b"IDAT", zlib.compress(raw)) +
                           chunk(b"IEND", b""))
    assert np.array_equal(read_image(path), cv2.imread(path, flags))
    assert np.array_equal(read_image(path), gray)


@pytest.mark.parametrize("depth", [np.uint8, np.uint16])
@pytest.mark.parametrize("compression", [1, 5, 8, 32946, 32773])
def test_read_compressed_tiff_matches_cv2(tmp_path, depth, compression):
    """TIFF strips without compression, LZW, Deflate and PackBits, with the horizontal predictor OpenCV
    writes by default, gray and colour: identical to cv2.imread(IMREAD_GRAYSCALE | IMREAD_ANYDEPTH)."""
    cv2 = pytest.importorskip("cv2")
    from ct_b200.ctvolume import read_image
    rng = np.random.default_rng(compression)
    top = np.iinfo(depth).max
    yy, xx = np.mgrid[0:181, 0:263]
    smooth = (np.sin(xx / 17.0) * np.cos(yy / 11.0) * 0.5 + 0.5) * top * 0.8
    gray = np.clip(smooth + rng.normal(0, top * 0.02, smooth.shape), 0, top).astype(depth)
    color = np.stack([gray, np.roll(gray, 5, 1), rng.integers(0, top + 1, gray.shape).astype(depth)], -1)
    flags = cv2.IMREAD_GRAYSCALE | cv2.IMREAD_ANYDEPTH
    for name, img in [("g", gray), ("c", color)]:
        path = str(tmp_path / f"{name}{compression}.tif")
        assert cv2.imwrite(path, img, [cv2.IMWRITE_TIFF_COMPRESSION, compression])
        ref = cv2.imread(path, flags)
        got = read_image(path)
        assert got.dtype == ref.dtype and np.array_equal(got, ref), (name, compression)


def test_remaining_facade_getters_and_setters(tmp_path):
    """getProjectionAt, getSkipProjections, getUseCuda, getEmitSignals, getActiveCudaDevices,
    getGpuSpareMemory, the GPU coefficients and getRequiredMemoryUpperBound (Ct/CtVolume.cpp:332-481)."""
    csv, imgs, geom = write_scan(tmp_path, heights=[0.0, 0.5, 1.0, 1.5, 2.0, 2.5])
    v = CtVolume(csv)
    # getProjectionAt: convertTo32bit then (p - min) / (max - min) with min, max = raw extremes / 2^16
    img, angle, height = v.getProjectionAt(2)
    lo, hi = np.float32(imgs.min() / 65536.0), np.float32(imgs.max() / 65536.0)
    alpha, beta = np.float32(1.0 / 65535.0), np.float32(0.000001 * 1.0)
    p = imgs[2].astype(np.float32) * alpha + beta
    np.testing.assert_array_equal(img, (p - lo) / (hi - lo))
    assert angle == pytest.approx(geom.angles()[2])
    pix = v.getPixelSize()
    assert height == pytest.approx((1.0 - 1.25) / pix)        # relative to the mean, in pixels
    with pytest.raises(CtbError):
        v.getProjectionAt(6)
    # settings
    assert v.getSkipProjections() == 0 and v.getUseCuda() and v.getEmitSignals()
    assert not v.getUseCpuPreprocessing() and v.getGpuSpareMemory() == 200
    assert (v.getMultiprocessorCoefficient(), v.getMemoryBandwidthCoefficient()) == (1.0, 1.0)
    assert v.getActiveCudaDevices() == [0]
    v.setSkipProjections(3)
    v.setGpuSpareMemory(512)
    v.setGpuCoefficients(2.0, 0.5)
    v.setUseCpuPreprocessing(True)
    v.setEmitSignals(False)
    assert v.getSkipProjections() == 3 and v.getGpuSpareMemory() == 512
    assert (v.getMultiprocessorCoefficient(), v.getMemoryBandwidthCoefficient()) == (2.0, 0.5)
    assert v.getUseCpuPreprocessing() and not v.getEmitSignals()
    with pytest.raises(CtbError):
        v.setUseCuda(False)
    v.setUseCuda(True)
    X, Y, Z = v.getXSize(), v.getYSize(), v.getZSize()
    assert v.getRequiredMemoryUpperBound() == X * Y * Z * 4 + 12 * 8 * 4 * 1 * 3
    assert isinstance(CtVolume.cudaAvailable(), bool)


def _rows_reached(det, grid, z0, z1, heights, rng, n_cols=6000, n_ang=180):
    """Brute force in float64: the detector rows (v0 and v0 + 1 of the bilinear
    sample) of voxels in the cylinder, inside the u and v bounds
    (Ct/CtVolume.cpp:923-1011), for box slices z0 and z1 - 1 (the row is
    monotone in z), over random columns and angles."""
    W, H, D, uoff, r2 = det.width, det.height, det.fcd, det.u_offset, det.radius ** 2
    vs = grid.voxel_pitch
    xpre = grid.x_size / 2 - grid.x_from
    ypre = grid.y_size / 2 - grid.y_from
    zpre = grid.z_size / 2 - grid.z_from
    X, Y = grid.x_to - grid.x_from, grid.y_to - grid.y_from
    ix = rng.integers(0, X, n_cols)
    iy = rng.integers(0, Y, n_cols)
    # the cylinder's rim, where the magnification is largest
    phi = rng.uniform(0, 2 * np.pi, n_cols)
    rim = np.sqrt(r2) * 0.999
    ix = np.concatenate([ix, np.clip(np.round(rim * np.cos(phi) / vs + xpre), 0, X - 1)]).astype(int)
    iy = np.concatenate([iy, np.clip(np.round(rim * np.sin(phi) / vs + ypre), 0, Y - 1)]).astype(int)
    x, y = (ix - xpre) * vs, (iy - ypre) * vs
    keep = x * x + y * y < r2
    x, y = x[keep], y[keep]
    rows = []
    hs = np.zeros(1) if heights is None else np.asarray(heights)
    for th in rng.uniform(0, 2 * np.pi, n_ang):
        sn, cs = np.sin(th), np.cos(th)
        s = x * cs + y * sn
        t = -x * sn + y * cs + uoff
        U = D / (D - s)
        u = t * U
        ok = (u >= -W / 2) & (u <= W - 1.1 - W / 2)
        for zi in (z0, z1 - 1):
            zw = (zi - zpre) * vs
            for h in hs:
                v = (zw + h) * U[ok]
                vok = (v >= -(H - 1 - 0.1) + H / 2) & (v <= H / 2)
                vi = -v[vok] + H / 2
                r = np.floor(vi).astype(int)
                rows.append(r)
                rows.append(r + 1)
    return np.concatenate(rows) if rows else np.zeros(0, int)


def test_row_band_covers_every_row_reached():
    from ct_b200 import ops
    rng = np.random.default_rng(11)
    shrunk = 0
    for k in range(24):
        W, H = int(rng.integers(24, 400)), int(rng.integers(16, 400))
        fcd = float(rng.uniform(1.5 * W, 10 * W))
        det, grid = ops.detector(W, H, fcd, u_offset=float(rng.choice([0.0, 2.5, -4.0])))
        Z = grid.z_to - grid.z_from
        z0 = int(rng.integers(0, Z))
        z1 = int(rng.integers(z0 + 1, Z + 1))
        heights = rng.uniform(-4, 4, 16) if k % 2 else None
        r_lo, n = ops.row_band(det, grid, z0, z1, heights)
        assert 0 <= r_lo and n >= 1 and r_lo + n <= H
        r = _rows_reached(det, grid, z0, z1, heights, rng)
        if r.size:
            assert r.min() >= r_lo and r.max() <= r_lo + n - 1, (k, r.min(), r.max(), r_lo, n)
        shrunk += n < H
    assert shrunk >= 8   # thin slabs really do get a narrower band
    # the whole box reaches the whole detector (rows clipped to it)
    det, grid = ops.detector(256, 192, 1000.0)
    assert ops.row_band(det, grid, 0, grid.z_to - grid.z_from) == (0, 192)


@pytest.mark.parametrize("pattern", ["constant", "ramp", "repeat", "noise", "sparse"])
def test_lzw_tiff_patterns_match_cv2(tmp_path, pattern):
    """LZW strings of every kind: runs that hit the code being defined (constant and
    repeating rows), full tables that force clear codes (noise over 1024^2), code widths
    9 to 12, and strips whose last code ends the strip exactly."""
    cv2 = pytest.importorskip("cv2")
    from ct_b200.ctvolume import read_image
    rng = np.random.default_rng(3)
    H, W = 1024, 1024
    if pattern == "constant":
        img = np.full((H, W), 4321, np.uint16)
    elif pattern == "ramp":
        img = (np.arange(H * W, dtype=np.uint32) % 65536).astype(np.uint16).reshape(H, W)
    elif pattern == "repeat":
        img = np.tile(rng.integers(0, 65536, 37, dtype=np.uint16), H * W // 37 + 1)[:H * W].reshape(H, W)
    elif pattern == "noise":
        img = rng.integers(0, 65536, (H, W), dtype=np.uint16)
    else:
        img = np.zeros((H, W), np.uint16)
        img[rng.integers(0, H, 500), rng.integers(0, W, 500)] = rng.integers(1, 65536, 500)
    for depth_img in (img, (img >> 8).astype(np.uint8)):
        path = str(tmp_path / f"{pattern}_{depth_img.dtype}.tif")
        assert cv2.imwrite(path, depth_img, [cv2.IMWRITE_TIFF_COMPRESSION, 5])
        ref = cv2.imread(path, cv2.IMREAD_GRAYSCALE | cv2.IMREAD_ANYDEPTH)
        got = read_image(path)
        assert got.dtype == ref.dtype and np.array_equal(got, ref), (pattern, depth_img.dtype)
