"""The shared-memory backprojector's global-memory path for views whose
footprint does not fit the staged box, forced on every k-th view with
ctb_diag_force_overflow, against the oracle's restatement of the reference's
reconstructionCore (Ct/CtVolume.cpp:1006-1038).

Each tile visits the views in a rotated order (the CTAs resident together
start at different views), so the path must read the texels of the view
whose box and geometry the producer staged, not the tile's loop index. The
grids here have hundreds of tiles, so almost every tile runs rotated.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from ct_b200 import _lib as L  # noqa: E402
from ct_b200 import ops  # noqa: E402


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.init()
    yield
    L.lib().ctb_diag_force_overflow(0)


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-30))


DT = {L.FP32: torch.float32, L.FP16: torch.float16, L.BF16: torch.bfloat16}


@pytest.mark.parametrize("store", [L.FP32, L.FP16])
@pytest.mark.parametrize("every", [1, 3])
@pytest.mark.parametrize("zr", [None, (10, 30)])
def test_forced_overflow_matches_oracle(oracle, store, every, zr):
    rng = np.random.default_rng(100 + store * 10 + every)
    V, H, W, D = 90, 64, 192, 600.0
    det, grid = ops.detector(W, H, D, u_offset=0.5)
    og = oracle.ref_geom(W, H, D, 0.5)
    ang = np.sort(rng.uniform(0, 360, V))
    h = rng.uniform(-1.5, 1.5, V)
    proj = torch.from_numpy(rng.standard_normal((V, H, W)).astype(np.float32)).to(DT[store]).cuda()
    # the oracle sees exactly the stored values
    pf = proj.float().cpu().numpy()
    ref = oracle.ref_backproject(pf, ang, h, og)  # (x, y, z)
    X, Y, Z = grid.box
    z0, z1 = zr if zr else (0, Z)
    L.lib().ctb_diag_force_overflow(every)
    try:
        vol = ops.backproject(proj, ang, h, det, grid, z0, z1)
        torch.cuda.synchronize()
    finally:
        L.lib().ctb_diag_force_overflow(0)
    out = vol.cpu().numpy().transpose(2, 1, 0)
    assert rel_l2(out, ref[:, :, z0:z1]) <= 1e-5
    # the same launch without the forced path gives the same sums to rounding
    vol2 = ops.backproject(proj, ang, h, det, grid, z0, z1)
    torch.cuda.synchronize()
    assert rel_l2(vol.cpu().numpy(), vol2.cpu().numpy()) <= 2e-6


@pytest.mark.parametrize("store", [L.FP32, L.FP16])
def test_forced_overflow_in_the_batch_kernel(oracle, store):
    rng = np.random.default_rng(40 + store)
    scans, refs = [], []
    for i in range(4):
        W = int(rng.integers(96, 160))
        H = int(rng.integers(32, 64))
        V = int(rng.integers(40, 80))
        D = float(rng.uniform(3.0, 5.0) * W)
        det, grid = ops.detector(W, H, D)
        og = oracle.ref_geom(W, H, D)
        raw = torch.from_numpy(rng.integers(2000, 65535, (V, H, W)).astype(np.int32)).to(torch.uint16).cuda()
        ang = np.sort(rng.uniform(0, 360, V))
        hh = rng.uniform(-1, 1, V) if i % 2 else None
        X, Y, Z = grid.box
        scans.append(dict(raw=raw, angles_deg=ang, heights_px=hh, det=det, grid=grid, filter=i % 3, pad=1,
                          vol=torch.full((Z, Y, X), np.nan, device="cuda")))
        # the batch's own filtered values, backprojected by the oracle
        scale = 1.0 if store == L.FP32 else 1.0 / W
        f = ops.filter_projections(raw, det, i % 3, 1, store, scale)
        torch.cuda.synchronize()
        pf = f.float().cpu().numpy() / scale
        refs.append(oracle.ref_backproject(pf, ang, np.zeros(V) if hh is None else hh, og))
    L.lib().ctb_diag_force_overflow(2)
    try:
        b = ops.Batch(scans, store)
        b.run()
        torch.cuda.synchronize()
    finally:
        L.lib().ctb_diag_force_overflow(0)
    for s, ref in zip(scans, refs):
        out = s["vol"].cpu().numpy().transpose(2, 1, 0)
        assert np.isfinite(out).all()
        # FP16 storage: the oracle gets the stored values divided by the store
        # scale in FP32, the kernel multiplies by the load scale; a few ulp apart
        assert rel_l2(out, ref) <= 1e-5
