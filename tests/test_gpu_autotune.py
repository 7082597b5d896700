"""The autotuner of the backprojection: on the facade (block tile height,
views in flight and slab height, tuned on the context's own scan and kept per
shape) and on batches (tile height and views in flight of the persistent
kernel). A tuned reconstruction must give the volume of an untuned one (the
launch shape changes only the order of the sums: within 1e-6)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from ct_b200 import CtVolume, ops, synth  # noqa: E402
from ct_b200 import _lib as L  # noqa: E402


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.init()


def context(geom, imgs, grid, store):
    v = CtVolume()
    v.setProjections(imgs, geom.angles(), None, pixel_size=geom.pixel_eff, fcd_mm=geom.sod_mm)
    v.setGrid(*grid)
    v.setPrecision(store)
    return v


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


@pytest.mark.parametrize("store", ["fp16", "fp32"])
def test_facade_autotune_keeps_the_volume(store):
    geom = synth.ScanGeometry(240, 320, 256, pitch_mm=0.8, sod_mm=500.0, sdd_mm=1000.0)
    imgs = synth.make_scan(geom, 8, 31 + len(store)).images.cpu().numpy()
    grid = (192, 192, 160, 1.6)
    plain = context(geom, imgs, grid, store)
    assert plain.getTuning()["tuned"] in (0, 1)
    X, Y, Z = plain.grid().box
    ref = np.empty((Z, Y, X), np.float32)
    plain.reconstructInto(ref.ctypes.data, L.X_FASTEST)

    tuned = context(geom, imgs, grid, store)
    t = tuned.autotune()
    assert t["tuned"] == 1
    assert t["zc"] in (0, 16, 32) and t["views_in_flight"] in (0, 2, 3, 4)
    assert 16 <= t["slab_slices"] <= Z and t["backproject_ms"] > 0
    assert tuned.getTuning()["slab_slices"] == t["slab_slices"]
    out = np.empty_like(ref)
    tuned.reconstructInto(out.ctypes.data, L.X_FASTEST)
    assert rel(out, ref) <= 1e-6


def test_autotune_on_first_reconstruction():
    geom = synth.ScanGeometry(120, 256, 200, pitch_mm=1.0, sod_mm=500.0, sdd_mm=1000.0)
    imgs = synth.make_scan(geom, 6, 5).images.cpu().numpy()
    v = context(geom, imgs, (176, 176, 144, 1.25), "bf16")
    v.setAutotune(True)
    X, Y, Z = v.grid().box
    out = np.empty((Z, Y, X), np.float32)
    v.reconstructInto(out.ctypes.data, L.X_FASTEST)
    assert np.isfinite(out).all()
    assert v.getTuning()["tuned"] == 1


def test_batch_autotuner_times_every_candidate():
    rng = np.random.default_rng(12)
    scans = []
    for i in range(4):
        W, H, V = int(rng.integers(80, 200)), int(rng.integers(60, 150)), int(rng.integers(30, 90))
        det, _ = ops.detector(W, H, 4.0 * W)
        edge = int(rng.integers(40, 96))
        grid = ops.custom_grid(det, (edge, edge, edge), float(W) / edge)
        raw = torch.from_numpy(rng.integers(2000, 65535, (V, H, W)).astype(np.int32)).to(torch.uint16).cuda()
        scans.append(dict(raw=raw, angles_deg=np.sort(rng.uniform(0, 360, V)), heights_px=None, det=det, grid=grid,
                          filter=i % 3, pad=1, vol=torch.empty((edge, edge, edge), device="cuda")))
    b = ops.Batch(scans, L.FP16)
    detail = b.tuning_detail()
    assert len(detail) == 7
    ok = [d for d in detail if d[2] >= 0]
    assert ok
    best = min(ok, key=lambda d: d[2])
    assert b.tuning()["zc"] == best[0]
