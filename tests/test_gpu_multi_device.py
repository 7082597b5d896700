"""Multi-device reconstruction through the facade (setActiveCudaDevices).

Each listed device reconstructs its own run of z slices from all views in its
own host thread (launchCudaThreads, Ct/CtVolume.cpp:1322-1351). With one GPU
the same device is listed twice: two workers with their own streams and
buffers, none waiting on the other. The volume must match the one-device
volume up to the rounding of where slab boundaries fall, for both output
orders, and the weighted progress must end at 100 %.
"""
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from ct_b200 import CtVolume, CtbError, synth  # noqa: E402
from ct_b200 import _lib as L  # noqa: E402


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.init()


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


@pytest.fixture(scope="module")
def scan_csv(tmp_path_factory):
    tmp = tmp_path_factory.mktemp("md")
    geom = synth.ScanGeometry(90, 128, 96, pitch_mm=1.0, sod_mm=500.0, sdd_mm=1000.0)
    scan = synth.make_scan(geom, 8, 21)
    return synth.write_scan(str(tmp), scan.images.cpu().numpy(), geom)


@pytest.mark.parametrize("store", ["fp32", "fp16"])
def test_two_workers_match_one(scan_csv, store):
    one = CtVolume(scan_csv)
    one.setPrecision(store)
    one.setVolumeBounds(0.0, 1.0, 0.0, 1.0, 0.1, 0.95)
    one.reconstructVolume()
    ref_x = one.volume(L.X_FASTEST)

    two = CtVolume(scan_csv)
    two.setPrecision(store)
    two.setVolumeBounds(0.0, 1.0, 0.0, 1.0, 0.1, 0.95)
    two.setActiveCudaDevices([0, 0])
    two.setSlabHeight(16)
    seen = []
    two.setProgressCallback(lambda s, p: seen.append(p))
    two.reconstructVolume()
    out_x = two.volume(L.X_FASTEST)
    assert out_x.shape == ref_x.shape
    err = rel_l2(out_x, ref_x)
    print(f"{store}: two workers vs one, rel-L2 {err:.2e}")
    assert err <= 2e-6
    assert seen and abs(seen[-1] - 100.0) < 1e-9 and all(b >= a - 1e-12 for a, b in zip(seen, seen[1:]))

    # both orders into caller memory: pageable, and pinned (written without staging)
    X, Y, Z = two.grid().box
    buf = np.empty(X * Y * Z, np.float32)
    two.reconstructInto(buf.ctypes.data, L.Z_FASTEST)
    assert rel_l2(buf, ref_x.transpose(2, 1, 0).ravel()) <= 2e-6
    pinned = torch.empty(X * Y * Z, dtype=torch.float32).pin_memory()
    two.reconstructInto(pinned.data_ptr(), L.X_FASTEST)
    assert rel_l2(pinned.numpy(), ref_x.ravel()) <= 2e-6
    pinned_z = torch.empty(X * Y * Z, dtype=torch.float32).pin_memory()
    two.reconstructInto(pinned_z.data_ptr(), L.Z_FASTEST)
    assert np.array_equal(pinned_z.numpy(), buf)


def test_uneven_weights_and_device_selection(scan_csv):
    v = CtVolume(scan_csv)
    # one device: the whole weight
    assert v.getGpuWeights([0]) == {0: 1.0}
    w = v.getGpuWeights([0, 0])
    assert w[0] == pytest.approx(0.5)
    # invalid IDs are dropped; none valid keeps the previous selection
    with pytest.raises(CtbError):
        v.setActiveCudaDevices([torch.cuda.device_count() + 5])
    v.setActiveCudaDevices([0, torch.cuda.device_count() + 5])
    # three workers on one device: 3 x round(z/3) slices, the last takes the rest
    v.setActiveCudaDevices([0, 0, 0])
    v.setGpuCoefficients(1.0, 1.0)
    v.reconstructVolume()
    a = v.volume(L.X_FASTEST)
    ref = CtVolume(scan_csv)
    ref.reconstructVolume()
    assert rel_l2(a, ref.volume(L.X_FASTEST)) <= 2e-6
