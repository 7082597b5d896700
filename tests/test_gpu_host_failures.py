"""Failure paths of the reconstruction facade, made on the host (no GPU
fault), and the determinism of its results.

Reference mechanisms: stop() sets stopActiveProcess, polled once per view by
the reconstruction loops (Ct/CtVolume.cpp:723-726, :946, :1179); a failing
CUDA worker sets stopCudaThreads so its siblings end (:1184-1188); an
allocation that fails ends the reconstruction with an error message
(:554-557, :1133-1147). Here ctb_stop is polled per upload chunk and slab,
a failing worker sets the shared stop flag, and ctb_diag_fail_allocation
makes the n-th facade allocation fail as if memory were exhausted.
"""
import threading
import time

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from ct_b200 import CtVolume, synth  # noqa: E402
from ct_b200 import _lib as L  # noqa: E402
from ct_b200._lib import CtbError, lib  # noqa: E402


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.init()
    yield
    lib().ctb_diag_fail_allocation(0)


@pytest.fixture(scope="module")
def scan():
    geom = synth.ScanGeometry(180, 192, 160, pitch_mm=1.0, sod_mm=500.0, sdd_mm=1000.0)
    s = synth.make_scan(geom, 8, 21)
    return geom, s.images.cpu().numpy()


def context(geom, imgs, devices=None, slab=0):
    v = CtVolume()
    v.setProjections(imgs, geom.angles(), None, pixel_size=geom.pixel_eff, fcd_mm=geom.sod_mm)
    v.setPrecision("fp16")
    if slab:
        v.setSlabHeight(slab)
    if devices:
        v.setActiveCudaDevices(devices)
    return v


def reconstruct_into(v, out):
    v.reconstructInto(out.ctypes.data, L.X_FASTEST)


def empty_volume(v):
    X, Y, Z = v.grid().box
    return np.full((Z, Y, X), np.nan, np.float32)


def test_stop_from_another_thread_then_reuse(scan):
    geom, imgs = scan
    ref_ctx = context(geom, imgs, slab=8)
    ref = empty_volume(ref_ctx)
    reconstruct_into(ref_ctx, ref)

    v = context(geom, imgs, slab=8)
    started = threading.Event()
    stopped = threading.Event()

    def on_progress(stage, pct):
        if stage == 1 and not started.is_set():
            started.set()
            # hold the reconstructing thread until the other thread has called stop
            stopped.wait(10.0)

    def stopper():
        started.wait(30.0)
        lib().ctb_stop(v._ctx)
        stopped.set()

    v.setProgressCallback(on_progress)
    t = threading.Thread(target=stopper)
    t.start()
    out = empty_volume(v)
    with pytest.raises(CtbError) as e:
        reconstruct_into(v, out)
    t.join()
    assert e.value.status == L.CTB_INTERRUPTED
    assert started.is_set() and stopped.is_set()
    # the same context reconstructs normally afterwards, with the same bits
    v.setProgressCallback(None)
    out2 = empty_volume(v)
    reconstruct_into(v, out2)
    assert np.array_equal(out2, ref)


@pytest.mark.parametrize("nth", [1, 2, 4, 7])
def test_allocation_failure_leaves_the_caller_buffer_untouched(scan, nth):
    geom, imgs = scan
    v = context(geom, imgs, slab=16)
    out = empty_volume(v)
    lib().ctb_diag_fail_allocation(nth)
    try:
        with pytest.raises(CtbError) as e:
            reconstruct_into(v, out)
    finally:
        lib().ctb_diag_fail_allocation(0)
    assert e.value.status == L.CTB_ERR_ALLOC
    assert np.isnan(out).all()
    # no allocation fails any more: the same context completes
    reconstruct_into(v, out)
    assert np.isfinite(out).all()


def test_failing_worker_stops_its_siblings(scan):
    """Three workers (device 0 listed three times); one allocation fails in
    whichever worker reaches it first, the status is the allocation error,
    not a hang or an interruption, and the context works afterwards."""
    geom, imgs = scan
    v = context(geom, imgs, devices=[0, 0, 0], slab=8)
    one = context(geom, imgs, slab=8)
    ref = empty_volume(one)
    reconstruct_into(one, ref)
    out = empty_volume(v)
    lib().ctb_diag_fail_allocation(3)
    t0 = time.perf_counter()
    try:
        with pytest.raises(CtbError) as e:
            reconstruct_into(v, out)
    finally:
        lib().ctb_diag_fail_allocation(0)
    assert time.perf_counter() - t0 < 60.0
    assert e.value.status == L.CTB_ERR_ALLOC
    assert "injected" in e.value.message
    out[:] = np.nan
    reconstruct_into(v, out)
    # each worker filters only the detector rows its slices reach, so its row
    # coordinates are rounded from another first row: a few ulps of every
    # sample position from one device (the parity bar, FP16 storage)
    err = np.linalg.norm((out - ref).ravel().astype(np.float64)) / np.linalg.norm(ref.ravel().astype(np.float64))
    assert err <= 1e-5, err


@pytest.mark.parametrize("store", ["fp32", "fp16", "bf16"])
def test_reconstructions_are_bitwise_repeatable(scan, store):
    """Every voxel's sum is taken in a fixed order (the view order of its tile
    depends on the tile's launch position only), so two reconstructions, and
    a second context, give identical bits."""
    geom, imgs = scan
    a = context(geom, imgs, slab=24)
    a.setPrecision(store)
    b = context(geom, imgs, slab=24)
    b.setPrecision(store)
    x1, x2, x3 = empty_volume(a), empty_volume(a), empty_volume(b)
    reconstruct_into(a, x1)
    reconstruct_into(a, x2)
    reconstruct_into(b, x3)
    assert np.isfinite(x1).all()
    assert np.array_equal(x1, x2)
    assert np.array_equal(x1, x3)
