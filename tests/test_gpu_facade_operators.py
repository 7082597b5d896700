"""The context-level matched projector pair and least-squares gradient
(ctb_forward, ctb_backward, ctb_gradient) and the one-shot batch
(ctb_batch_reconstruct), through the C ABI.

ctb_forward / ctb_backward must equal the operator-level forward projector
and backprojector (load scale 1) on the same geometry, and be each other's
transpose (<A x, y> = <x, A^T y> to 1e-5); ctb_gradient must return
||A x - p||^2 and 2 A^T (A x - p) as computed from the pair, and agree with
central differences of the loss. Volumes larger than one device slab are
moved through in several slabs."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from ct_b200 import CtVolume, ops  # noqa: E402
from ct_b200 import _lib as L  # noqa: E402


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.init()


def context(V=48, H=40, W=56, grid=(40, 36, 30), vs=1.25, heights=True, seed=0):
    rng = np.random.default_rng(seed)
    imgs = rng.integers(2000, 65535, (V, H, W)).astype(np.uint16)
    ang = np.sort(rng.uniform(0, 360, V))
    hmm = rng.uniform(-0.4, 0.4, V) if heights else None
    v = CtVolume()
    v.setProjections(imgs, ang, hmm, pixel_size=0.5, fcd_mm=0.5 * 4 * W, u_offset_mm=0.3)
    v.setGrid(*grid, vs)
    return v


def operator_geometry(v):
    det, grid = v.detector(), v.grid()
    n = v.getSinogramSize()
    ang = np.empty(n)
    hp = np.empty(n)
    for i in range(n):
        _, a, h = v.getProjectionAt(i)
        ang[i], hp[i] = a, h
    return det, grid, ang, hp


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-30))


def test_forward_and_backward_match_the_operator_layer():
    v = context()
    det, grid, ang, hp = operator_geometry(v)
    rng = np.random.default_rng(1)
    X, Y, Z = grid.box
    x = rng.standard_normal((Z, Y, X)).astype(np.float32)
    y = rng.standard_normal((v.getSinogramSize(), det.height, det.width)).astype(np.float32)
    Ax = v.forwardProject(x)
    Aty = v.backProject(y)
    Ax_op = ops.forward_project(torch.from_numpy(x).cuda(), ang, hp, det, grid).cpu().numpy()
    Aty_op = ops.backproject(torch.from_numpy(y).cuda(), ang, hp, det, grid).cpu().numpy()
    assert rel(Ax, Ax_op) <= 1e-6
    assert rel(Aty, Aty_op) <= 1e-6
    lhs = float(np.dot(Ax.ravel().astype(np.float64), y.ravel()))
    rhs = float(np.dot(x.ravel().astype(np.float64), Aty.ravel()))
    assert abs(lhs - rhs) / max(abs(lhs), abs(rhs)) <= 1e-5


def test_gradient_matches_the_pair_and_finite_differences():
    v = context(seed=2)
    det, grid, ang, hp = operator_geometry(v)
    rng = np.random.default_rng(3)
    X, Y, Z = grid.box
    x = rng.standard_normal((Z, Y, X)).astype(np.float32)
    p = rng.standard_normal((v.getSinogramSize(), det.height, det.width)).astype(np.float32)
    f, g = v.gradient(x, p)
    r = v.forwardProject(x).astype(np.float64) - p
    assert abs(f - float((r * r).sum())) <= 1e-5 * f
    g_ref = 2.0 * v.backProject(r.astype(np.float32))
    assert rel(g, g_ref) <= 1e-5
    # central differences of f along a few voxels (f is quadratic: exact up to rounding)
    for k in range(6):
        z, yy, xx = (int(rng.integers(2, s - 2)) for s in (Z, Y, X))
        e = np.zeros_like(x)
        e[z, yy, xx] = 1.0
        eps = 0.5
        fp, _ = v.gradient(x + eps * e, p)
        fm, _ = v.gradient(x - eps * e, p)
        fd = (fp - fm) / (2 * eps)
        assert abs(fd - g[z, yy, xx]) <= 1e-3 * max(1.0, abs(fd)), (k, fd, g[z, yy, xx])


def test_volume_in_several_slabs():
    """A box whose planes exceed a quarter of the 512 MB slab buffer: the pair
    moves it through in several slabs and still equals the operator layer."""
    v = context(V=6, H=24, W=40, grid=(6000, 6000, 5), vs=0.006, heights=False, seed=4)
    det, grid, ang, hp = operator_geometry(v)
    X, Y, Z = grid.box
    assert X * Y * 4 * Z > (512 << 20)
    rng = np.random.default_rng(5)
    y = rng.standard_normal((v.getSinogramSize(), det.height, det.width)).astype(np.float32)
    Aty = v.backProject(y)
    Aty_op = ops.backproject(torch.from_numpy(y).cuda(), ang, hp, det, grid).cpu().numpy()
    assert rel(Aty, Aty_op) <= 1e-6


def test_one_shot_batch_matches_the_batch_object():
    rng = np.random.default_rng(9)
    scans_a, scans_b = [], []
    for i in range(3):
        W, H, V = int(rng.integers(60, 130)), int(rng.integers(30, 70)), int(rng.integers(20, 50))
        det, _ = ops.detector(W, H, 4.0 * W)
        grid = ops.custom_grid(det, (40, 42, 30), 1.5)
        raw = torch.from_numpy(rng.integers(2000, 65535, (V, H, W)).astype(np.int32)).to(torch.uint16).cuda()
        ang = np.sort(rng.uniform(0, 360, V))
        for lst in (scans_a, scans_b):
            lst.append(dict(raw=raw, angles_deg=ang, heights_px=None, det=det, grid=grid, filter=i % 3, pad=1,
                            vol=torch.full((30, 42, 40), np.nan, device="cuda")))
    ops.batch_reconstruct(scans_a, L.FP16)
    b = ops.Batch(scans_b, L.FP16)
    b.run()
    torch.cuda.synchronize()
    for a, c in zip(scans_a, scans_b):
        assert torch.equal(a["vol"], c["vol"])
