"""Failure detection on the device without a fault: every wait in the
backprojection kernels is bounded and reports giving up to the host.

The probe waits on a barrier that can never complete (two arrivals expected,
one given) with a short try limit; the wait must give up, be counted, and
leave the context usable for the next reconstruction."""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from ct_b200 import CtVolume, synth  # noqa: E402
from ct_b200 import _lib as L  # noqa: E402
from ct_b200._lib import lib  # noqa: E402


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.init()


def timeouts(reset):
    n = ctypes.c_uint()
    assert lib().ctb_device_wait_timeouts(0, ctypes.byref(n), reset) == L.CTB_OK
    return n.value


def test_bounded_wait_gives_up_and_context_stays_usable(tmp_path):
    timeouts(1)
    assert lib().ctb_diag_bounded_wait(0, 2000) == L.CTB_ERR_TIMEOUT
    assert b"gave up" in lib().ctb_last_error_global()
    assert timeouts(1) == 1
    assert timeouts(0) == 0
    # the device is still usable: a reconstruction runs and reports no give-up
    geom = synth.ScanGeometry(24, 64, 48, pitch_mm=1.0, sod_mm=500.0, sdd_mm=1000.0)
    scan = synth.make_scan(geom, 4, 3)
    csv = synth.write_scan(str(tmp_path), scan.images.cpu().numpy(), geom)
    v = CtVolume(csv)
    v.reconstructVolume()
    assert np.isfinite(v.volume(L.X_FASTEST)).all()
    assert timeouts(0) == 0
