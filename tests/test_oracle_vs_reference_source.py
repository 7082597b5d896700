"""The oracle against the reference's own CPU reconstruction code.

oracle/_ref/libct_ref.so is built from the reference's lines of
Ct/CtVolume.cpp (grid rule :306-327, cylinder radius :370-373, bounds
:487-500, relative heights and angle direction :742-767, preprocessing and
windows :787-885, reconstructionCore and bilinearInterpolation :923-1054,
updateBoundaries and coordinate transforms :1399-1466), compiled unchanged
with stand-ins for the OpenCV/Qt names they use (oracle/ref_shim.h). The
oracle's restatement (orc_ref_*), which every GPU parity test is scored
against, must give the same bits.

The second build (libct_ref_gcc.so) compiles the same lines with <cmath>
alone under libstdc++, where sqrt of a float is the double square root: the
Feldkamp weight W() then differs in the last bit for some pixels, so those
results agree to rounding (rel-L2 <= 3e-7 per projection, <= 2e-6 per
volume after the ramp filter), not bit for bit.
"""
import numpy as np
import pytest

from oracle import oracle as orc


@pytest.fixture(scope="module", autouse=True)
def _ref_built():
    if not orc.ref_source_available():
        pytest.skip("the reference sources are absent and oracle/_ref is not built")
    orc.build()
    orc.build_ref()


def images(V, H, W, seed, bits=16):
    rng = np.random.default_rng(seed)
    if bits == 8:
        return rng.integers(20, 255, (V, H, W)).astype(np.uint8)
    if bits == 32:
        return rng.uniform(0.05, 1.0, (V, H, W)).astype(np.float32)
    return rng.integers(2000, 65535, (V, H, W)).astype(np.uint16)


@pytest.mark.parametrize("rotation", ["cw", "ccw"])
@pytest.mark.parametrize("increasing", [True, False])
def test_sinogram_fix_is_identical(rotation, increasing):
    rng = np.random.default_rng(3)
    ang = np.sort(rng.uniform(0, 360, 17))
    if not increasing:
        ang = ang[::-1].copy()
    h = rng.uniform(-3, 3, 17)
    a_ref, h_ref = orc.refsrc_fix_sinogram(ang, h, 0.37, rotation)
    a_orc, h_orc = orc.fix_sinogram(ang, h, rotation == "ccw", 0.37)
    assert np.array_equal(a_ref, a_orc)
    assert np.array_equal(h_ref, h_orc)


@pytest.mark.parametrize("W,H,fcd_mm,pix", [(256, 192, 500.0, 0.5), (101, 40, 90.0, 0.25), (64, 64, 33.0, 0.5)])
@pytest.mark.parametrize("rel", [None, (0.1, 0.9, 0.2, 0.7, 0.25, 0.95), (0.6, 0.9, 0.0, 0.3, 0.1, 0.4)])
def test_grid_and_bounds_are_identical(W, H, fcd_mm, pix, rel):
    """Including the clamp of yTo and zTo against xFrom (:496, :498): the last
    bounds have yTo, zTo below xFrom."""
    imgs = images(2, H, W, 0)
    dims = orc.refsrc_reconstruct(imgs, [0.0, 180.0], None, pix, fcd_mm, rel=rel, dims_only=True)
    cl = orc.clamp_bounds(*rel) if rel else (0, 1, 0, 1, 0, 1)
    g = orc.ref_geom(W, H, np.float32(fcd_mm) / np.float32(pix), rel=cl)
    assert dims == g.box


@pytest.mark.parametrize("W", [64, 100, 256])
@pytest.mark.parametrize("ft", [orc.RAMLAK, orc.SHEPPLOGAN, orc.HANN])
@pytest.mark.parametrize("bits", [8, 16, 32])
def test_preprocessing_is_identical(W, ft, bits):
    H = 12
    imgs = images(3, H, W, W + ft + bits, bits)
    base = 1.0 if bits != 32 else 1.1
    fcd_mm, pix = 3.0 * W * 0.5, 0.5
    FCD = float(np.float32(fcd_mm) / np.float32(pix))
    for i in range(3):
        a = orc.refsrc_prepare_projection(imgs, i, pix, fcd_mm, base, ft)
        b = orc.ref_preprocess(imgs[i], base, FCD, ft)
        assert np.array_equal(a, b), (i, np.abs(a - b).max())
        g = orc.refsrc_prepare_projection(imgs, i, pix, fcd_mm, base, ft, variant="gcc")
        assert np.linalg.norm(g - b) / np.linalg.norm(b) <= 3e-7


CASES = [
    # V, H, W, fcd_mm, pixel size, u offset mm, heights, rotation, bounds, filter, skip
    dict(V=48, H=40, W=64, fcd=100.0, pix=0.5, uoff=0.0, heights=False, rot="ccw", rel=None, ft=0, skip=0),
    dict(V=40, H=36, W=72, fcd=80.0, pix=0.4, uoff=0.6, heights=True, rot="cw", rel=(0.1, 0.9, 0.2, 0.7, 0.25, 0.95),
         ft=1, skip=0),
    dict(V=45, H=30, W=50, fcd=60.0, pix=0.5, uoff=-0.4, heights=True, rot="ccw", rel=(0.0, 1.0, 0.0, 1.0, 0.3, 0.6),
         ft=2, skip=2),
]


@pytest.mark.parametrize("c", CASES, ids=["plain", "subbox_cw_offsets", "thin_slab_skip"])
def test_backprojection_loops_are_identical(c):
    """The reference's filtered projections through the oracle's restated
    reconstructionCore give the reference's own volume, bit for bit; and the
    whole oracle path gives it too."""
    rng = np.random.default_rng(11)
    V, H, W = c["V"], c["H"], c["W"]
    imgs = images(V, H, W, 5)
    ang = np.sort(rng.uniform(0, 360, V))
    hmm = rng.uniform(-1.0, 1.0, V) if c["heights"] else None
    vol_ref, _ = orc.refsrc_reconstruct(imgs, ang, hmm, c["pix"], c["fcd"], c["uoff"], 1.0, c["rot"], c["rel"], c["ft"],
                                        c["skip"])
    a, h = orc.refsrc_fix_sinogram(ang, np.zeros(V) if hmm is None else hmm, c["pix"], c["rot"])
    FCD = float(np.float32(c["fcd"]) / np.float32(c["pix"]))
    uoff = float(np.float32(c["uoff"]) / np.float32(c["pix"]))
    cl = orc.clamp_bounds(*c["rel"]) if c["rel"] else (0, 1, 0, 1, 0, 1)
    g = orc.ref_geom(W, H, FCD, uoff, rel=cl)
    pf = np.stack([orc.refsrc_prepare_projection(imgs, i, c["pix"], c["fcd"], 1.0, c["ft"]) for i in range(V)])
    vol_bp = orc.ref_backproject(pf, a, h, g, step=c["skip"] + 1)
    assert np.array_equal(vol_bp, vol_ref)
    vol_orc, _ = orc.ref_reconstruct(imgs, a, h, 1.0, c["ft"], g, step=c["skip"] + 1)
    assert np.array_equal(vol_orc, vol_ref)


def test_full_size_360_view_scan_is_identical():
    """360 views of 256 x 192 into the 252^2 x 192 reference grid (SOD 500 mm,
    CSV pixel size 0.5 mm): the oracle's whole path against the reference's."""
    rng = np.random.default_rng(2)
    V, H, W = 360, 192, 256
    u = np.linspace(-1, 1, W)[None, None, :]
    imgs = np.clip(60000 * np.exp(-1.2 * np.clip(1 - u ** 2, 0, None)) + rng.normal(0, 500, (V, H, W)), 100,
                   65535).astype(np.uint16)
    ang = np.arange(V) * 1.0
    vol_ref, secs = orc.refsrc_reconstruct(imgs, ang, None, 0.5, 500.0, filter_type=orc.RAMLAK)
    assert vol_ref.shape == (252, 252, 192)
    g = orc.ref_geom(W, H, 1000.0)
    a, h = orc.refsrc_fix_sinogram(ang, np.zeros(V), 0.5, "ccw")
    vol_orc, _ = orc.ref_reconstruct(imgs, a, h, 1.0, orc.RAMLAK, g)
    assert np.array_equal(vol_orc, vol_ref)
    vol_gcc, _ = orc.refsrc_reconstruct(imgs, ang, None, 0.5, 500.0, filter_type=orc.RAMLAK, variant="gcc")
    assert np.linalg.norm(vol_gcc - vol_ref) / np.linalg.norm(vol_ref) <= 2e-6
