"""The bounds-checked build (libctb_checked.so, kernels compiled with
CTB_BOUNDS_CHECK) on geometries that stress the footprint bounds: every texel
fetch of the shared-memory and global-gather backprojectors is checked
against the buffer it reads, and none may fall outside. The checked kernels
must give the same volumes as the normal library.

The checked library is loaded in a child process (CTB_LIBRARY=checked), so
it never shares a process with libctb.so."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r"""
import sys, json, ctypes, numpy as np, torch
sys.path.insert(0, %r)
from ct_b200 import ops
from ct_b200 import _lib as L
cases = json.loads(sys.argv[1])
prefix = sys.argv[2]
lib = L.lib()
chk, n, first = ctypes.c_int(), ctypes.c_uint(), ctypes.c_ulonglong()
assert lib.ctb_diag_bounds_status(0, ctypes.byref(chk), ctypes.byref(n), ctypes.byref(first), 1) == 0
report = {"checked_build": chk.value, "cases": {}}
for name, c in cases.items():
    rng = np.random.default_rng(c["seed"])
    V, H, W = c["V"], c["H"], c["W"]
    det, grid = ops.detector(W, H, c["D"], u_offset=c.get("uoff", 0.0), rel=c.get("rel"))
    if "grid" in c:
        grid = ops.custom_grid(det, tuple(c["grid"]), c["vs"])
    ang = np.sort(rng.uniform(0, 360, V))
    h = rng.uniform(-c.get("hmax", 0.0), c.get("hmax", 0.0), V)
    dt = {"fp32": torch.float32, "fp16": torch.float16, "bf16": torch.bfloat16}[c["store"]]
    proj = torch.from_numpy(rng.standard_normal((V, H, W)).astype(np.float32)).to(dt).cuda()
    lib.ctb_diag_force_overflow(c.get("overflow_every", 0))
    vol = ops.backproject(proj, ang, h, det, grid, c.get("z0", 0), c.get("z1"))
    torch.cuda.synchronize()
    lib.ctb_diag_force_overflow(0)
    assert lib.ctb_diag_bounds_status(0, ctypes.byref(chk), ctypes.byref(n), ctypes.byref(first), 1) == 0
    report["cases"][name] = {"violations": n.value, "first": first.value}
    np.save(prefix + "_" + name + ".npy", vol.cpu().numpy())
print(json.dumps(report))
"""

CASES = {
    "reference_fp32": dict(seed=1, V=40, H=64, W=64, D=200.0, store="fp32"),
    "reference_fp16_offsets": dict(seed=2, V=40, H=64, W=96, D=260.0, store="fp16", uoff=3.5, hmax=4.0),
    "binned_bf16": dict(seed=3, V=50, H=96, W=128, D=400.0, grid=[64, 60, 70], vs=2.0, store="bf16"),
    "far_slab": dict(seed=4, V=30, H=128, W=96, D=250.0, grid=[48, 48, 120], vs=1.5, z0=90, z1=120, store="fp32",
                     hmax=4.0),
    "subbox": dict(seed=5, V=36, H=40, W=56, D=150.0, uoff=2.5, hmax=3.0, rel=[0.1, 0.9, 0.2, 0.8, 0.25, 1.0],
                   store="fp16"),
    "forced_overflow": dict(seed=6, V=45, H=64, W=128, D=500.0, store="fp16", hmax=2.0, overflow_every=2),
    "coarse_voxels_global_gather": dict(seed=7, V=20, H=48, W=64, D=300.0, grid=[24, 24, 20], vs=9.0, store="fp32"),
}


def run(tmp_path, library):
    env = dict(os.environ)
    if library == "checked":
        env["CTB_LIBRARY"] = "checked"
    else:
        env.pop("CTB_LIBRARY", None)
    prefix = str(tmp_path / library)
    r = subprocess.run([sys.executable, "-c", SCRIPT % ROOT, json.dumps(CASES), prefix], env=env,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    report = json.loads(r.stdout.strip().splitlines()[-1])
    return report, {k: np.load(prefix + "_" + k + ".npy") for k in CASES}


def test_no_fetch_leaves_its_buffer(tmp_path):
    if not os.path.exists(os.path.join(ROOT, "ct_b200", "libctb_checked.so")):
        pytest.fail("libctb_checked.so is not built (python -m ct_b200.build)")
    rep_c, vol_c = run(tmp_path, "checked")
    rep_n, vol_n = run(tmp_path, "normal")
    assert rep_c["checked_build"] == 1 and rep_n["checked_build"] == 0
    for k in CASES:
        assert rep_c["cases"][k]["violations"] == 0, (k, rep_c["cases"][k])
        assert np.isfinite(vol_c[k]).all()
        err = np.linalg.norm((vol_c[k] - vol_n[k]).ravel()) / np.linalg.norm(vol_n[k].ravel())
        assert err <= 1e-6, (k, err)
