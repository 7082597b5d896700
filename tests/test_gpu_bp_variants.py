"""The shared-memory (TMA) backprojector against the global-gather one, and
the global one against the oracle, over geometries that stress the footprint
bound (binned voxels, far z slabs, height offsets, u offset, sub-boxes)."""
import os
import subprocess
import sys

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r"""
import sys, json, numpy as np, torch
sys.path.insert(0, %r)
from ct_b200 import ops
from ct_b200 import _lib as L
cases = json.loads(sys.argv[1])
out = {}
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
    vol = ops.backproject(proj, ang, h, det, grid, c.get("z0", 0), c.get("z1"))
    torch.cuda.synchronize()
    np.save(sys.argv[2] + "_" + name + ".npy", vol.cpu().numpy())
print("ok")
"""

CASES = {
    "ref_fp32": dict(seed=1, V=40, H=64, W=64, D=200.0, store="fp32"),
    "ref_fp16": dict(seed=2, V=40, H=64, W=64, D=200.0, store="fp16"),
    "ref_bf16": dict(seed=3, V=33, H=48, W=80, D=300.0, store="bf16"),
    "binned": dict(seed=4, V=50, H=96, W=128, D=400.0, grid=[64, 60, 70], vs=2.0, store="fp16"),
    "far_slab": dict(seed=5, V=30, H=128, W=96, D=250.0, grid=[48, 48, 120], vs=1.5, z0=90, z1=120,
                     store="fp32", hmax=4.0),
    "offsets": dict(seed=6, V=36, H=40, W=56, D=150.0, uoff=2.5, hmax=3.0,
                    rel=[0.1, 0.9, 0.2, 0.8, 0.25, 1.0], store="fp32"),
}


def run_variant(tmp_path, variant):
    env = dict(os.environ, CTB_BP_VARIANT=variant)
    import json
    prefix = str(tmp_path / variant)
    r = subprocess.run([sys.executable, "-c", SCRIPT % ROOT, json.dumps(CASES), prefix], env=env,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    return {k: np.load(prefix + "_" + k + ".npy") for k in CASES}


def test_tma_matches_global(tmp_path):
    a = run_variant(tmp_path, "tma")
    b = run_variant(tmp_path, "global")
    for k in CASES:
        err = np.linalg.norm((a[k] - b[k]).ravel()) / max(np.linalg.norm(b[k].ravel()), 1e-30)
        assert err < 2e-6, (k, err)
