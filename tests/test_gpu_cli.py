"""The ctb tool end to end (Ct/main.cpp:53-234 order: load, bounds, filter,
reconstruct, save) against the facade with the same settings."""
import os
import subprocess

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from ct_b200 import CtVolume, build, synth  # noqa: E402
from ct_b200 import _lib as L  # noqa: E402


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    if not os.path.exists(build.CLI):
        pytest.skip("ctb tool not built")


def test_cli_matches_facade(tmp_path):
    geom = synth.ScanGeometry(60, 96, 64, pitch_mm=1.0, sod_mm=500.0, sdd_mm=1000.0)
    scan = synth.make_scan(geom, 6, 17)
    csv = synth.write_scan(str(tmp_path), scan.images.cpu().numpy(), geom)
    out = str(tmp_path / "cli.raw")
    r = subprocess.run([build.CLI, "-i", csv, "-o", out, "-f", "shepplogan", "-j", "zfastest", "-e", "bigendian",
                        "--zmin", "0.25", "--zmax", "0.75", "-d", "0"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "The resulting volume dimensions will be:" in r.stdout
    v = CtVolume(csv)
    v.setVolumeBounds(0, 1, 0, 1, 0.25, 0.75)
    v.setFrequencyFilterType("shepplogan")
    v.reconstructVolume()
    X, Y, Z = v.grid().box
    ref = v.volume(L.Z_FASTEST).ravel()
    got = np.fromfile(out, dtype=">f4")
    assert got.size == X * Y * Z
    assert np.array_equal(got.astype(np.float32), ref)
    info = (tmp_path / "cli.txt").read_text()
    assert "Big endian" in info and "Z fastest" in info
    assert (tmp_path / "cli.vgi").exists()
