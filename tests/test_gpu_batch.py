"""Batches of scans with different detector, view and volume sizes: the
persistent graph-captured launch, the scan-by-scan path and the plain
operator path give the same volumes."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from ct_b200 import ops  # noqa: E402
from ct_b200 import _lib as L  # noqa: E402


def make_scans(n, seed, store):
    rng = np.random.default_rng(seed)
    scans = []
    for i in range(n):
        W = int(rng.integers(40, 130))
        H = int(rng.integers(24, 100))
        V = int(rng.integers(12, 60))
        D = float(rng.uniform(3.0, 5.0) * W)
        det, _ = ops.detector(W, H, D)
        edge = int(rng.integers(16, 48))
        vs = float(rng.choice([1.0, 1.5, 2.0])) if i != 5 else 9.0  # scan 5: footprint beyond the box limit
        grid = ops.custom_grid(det, (edge, edge + 3, edge - 2), vs)
        raw = torch.from_numpy(rng.integers(2000, 65535, (V, H, W)).astype(np.int32)).to(torch.uint16).cuda()
        ang = np.sort(rng.uniform(0, 360, V))
        X, Y, Z = grid.box
        scans.append(dict(raw=raw, angles_deg=ang, heights_px=rng.uniform(-1, 1, V) if i % 2 else None, det=det,
                          grid=grid, filter=i % 3, pad=1 + (i % 4 == 3), vol=torch.full((Z, Y, X), np.nan,
                                                                                         device="cuda")))
    return scans


@pytest.mark.parametrize("store", [L.FP32, L.FP16])
def test_batch_matches_operator_path(store):
    scans = make_scans(7, 3 + store, store)
    b = ops.Batch(scans, store)
    b.run()
    torch.cuda.synchronize()
    graph = [s["vol"].clone() for s in scans]
    for s in scans:
        s["vol"].fill_(np.nan)
    b.run_sequential()
    torch.cuda.synchronize()
    seq = [s["vol"].clone() for s in scans]
    for i, s in enumerate(scans):
        scale = 1.0 if store == L.FP32 else 1.0 / s["det"].width
        f = ops.filter_projections(s["raw"], s["det"], s["filter"], s["pad"], store, scale)
        ref = ops.backproject(f, s["angles_deg"], s["heights_px"], s["det"], s["grid"], load_scale=1.0 / scale)
        torch.cuda.synchronize()
        r = ref.double().cpu().numpy()
        for v in (graph[i], seq[i]):
            o = v.double().cpu().numpy()
            assert np.isfinite(o).all(), i
            err = np.linalg.norm((o - r).ravel()) / max(np.linalg.norm(r.ravel()), 1e-30)
            assert err < 2e-6, (i, err)
    t = b.tuning()
    assert t["zc"] in (8, 16, 32)
    assert 1 <= t["persistent_scans"] <= len(scans) - 1  # scan 5 always runs on its own
    # replaying the graph again gives the same result
    b.run()
    torch.cuda.synchronize()
    for i, s in enumerate(scans):
        assert torch.equal(s["vol"], graph[i])


def test_batch_matches_the_oracle_on_c5_shaped_scans(oracle):
    """Scans shaped like the 32-scan batch (non-power-of-two detector widths,
    coarse voxels spanning the field of view, different magnifications and
    view counts) against the oracle's restatement of the reference CPU path
    (Ct/CtVolume.cpp:802-1054) on the same raw projections, FP32 storage."""
    rng = np.random.default_rng(77)
    scans, geoms, imgs = [], [], []
    for i, (W, H, V, edge) in enumerate([(300, 220, 90, 96), (517, 333, 120, 128), (701, 409, 100, 160)]):
        D = float(rng.uniform(1.5, 2.5) * rng.uniform(300, 700) / 0.2 * 0.2)  # focus distance in pixels
        D = max(D, 2.0 * W)
        det, _ = ops.detector(W, H, D)
        vs = float(W) / edge
        grid = ops.custom_grid(det, (edge, edge, edge), vs)
        im = rng.integers(3000, 65535, (V, H, W)).astype(np.uint16)
        raw = torch.from_numpy(im.astype(np.int32)).to(torch.uint16).cuda()
        ang = np.sort(rng.uniform(0, 360, V))
        scans.append(dict(raw=raw, angles_deg=ang, heights_px=None, det=det, grid=grid, filter=i % 3, pad=1,
                          vol=torch.full((edge, edge, edge), np.nan, device="cuda")))
        geoms.append(oracle.custom_geom(W, H, D, (edge, edge, edge), vs))
        imgs.append(im)
    b = ops.Batch(scans, L.FP32)
    b.run()
    torch.cuda.synchronize()
    for s, g, im in zip(scans, geoms, imgs):
        ref, _ = oracle.ref_reconstruct(im, s["angles_deg"], np.zeros(len(s["angles_deg"])), 1.0, s["filter"], g)
        out = s["vol"].double().cpu().numpy().transpose(2, 1, 0)
        err = np.linalg.norm((out - ref).ravel()) / np.linalg.norm(ref.ravel())
        assert err <= 1e-4, err
