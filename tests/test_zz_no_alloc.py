"""ctb_backproject_noalloc, the entry point for callers that cannot allocate
device memory (an application that reserves all of its GPU memory up front,
or whose device memory belongs to another framework's allocator).

It must give the same volume as ctb_backproject, called through the C ABI on
the same inputs, on two calls in a row (the second call reuses the shared
device array the first one filled, with a different view count and geometry),
and reject a call with more views than its array holds. This file is
collected last so that a run stopping at the first failure has already run
every other test; it also passes on its own in a fresh process.
"""
import ctypes

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


def call(name, proj, store, ang, h, det, grid, out, z0, z1, load_scale=1.0, accumulate=0):
    a = np.ascontiguousarray(ang, np.float64)
    hh = None if h is None else np.ascontiguousarray(h, np.float64)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    return getattr(L.lib(), name)(ctypes.c_void_p(proj.data_ptr()), store, len(a), a.ctypes.data,
                                  None if hh is None else hh.ctypes.data, ctypes.byref(det), ctypes.byref(grid),
                                  z0, z1, load_scale, ctypes.c_void_p(out.data_ptr()), accumulate, stream)


CASES = [
    # V, H, W, D, storage, torch dtype, height offsets, voxel grid override
    dict(V=60, H=48, W=64, D=220.0, store=L.FP32, dt=torch.float32, heights=True, grid=None),
    dict(V=25, H=40, W=96, D=300.0, store=L.FP16, dt=torch.float16, heights=False, grid=((40, 36, 30), 2.0)),
]


def test_noalloc_matches_allocating_entry_point():
    rng = np.random.default_rng(2026)
    for c in CASES:  # two calls in a row on the shared device array
        det, grid = ops.detector(c["W"], c["H"], c["D"], u_offset=0.5)
        if c["grid"] is not None:
            grid = ops.custom_grid(det, *c["grid"])
        X, Y, Z = grid.box
        ang = np.sort(rng.uniform(0, 360, c["V"]))
        h = rng.uniform(-1.5, 1.5, c["V"]) if c["heights"] else None
        proj = torch.from_numpy(rng.standard_normal((c["V"], c["H"], c["W"])).astype(np.float32)).to(c["dt"]).cuda()
        ref = torch.full((Z, Y, X), float("nan"), device="cuda")
        out = torch.full((Z, Y, X), float("nan"), device="cuda")
        assert call("ctb_backproject", proj, c["store"], ang, h, det, grid, ref, 0, Z) == L.CTB_OK
        assert call("ctb_backproject_noalloc", proj, c["store"], ang, h, det, grid, out, 0, Z) == L.CTB_OK
        torch.cuda.synchronize()
        r = ref.double().cpu().numpy()
        o = out.double().cpu().numpy()
        assert np.isfinite(o).all()
        err = np.linalg.norm((o - r).ravel()) / np.linalg.norm(r.ravel())
        assert err <= 1e-6, err


def test_noalloc_rejects_more_views_than_its_array():
    det, grid = ops.detector(32, 16, 100.0)
    V = 8193  # CTB_NOALLOC_MAX_VIEWS + 1
    proj = torch.zeros((1, 16, 32), device="cuda")
    out = torch.zeros(grid.box[::-1], device="cuda")
    ang = np.zeros(V)
    a = ang.ctypes.data
    st = L.lib().ctb_backproject_noalloc(ctypes.c_void_p(proj.data_ptr()), L.FP32, V, a, None, ctypes.byref(det),
                                         ctypes.byref(grid), 0, grid.box[2], 1.0, ctypes.c_void_p(out.data_ptr()),
                                         0, None)
    assert st == L.CTB_ERR_UNSUPPORTED
    assert b"8192" in L.lib().ctb_last_error_global()


def test_noalloc_split_views_accumulate_on_a_z_sub_range():
    """More views than one call should take, split into two calls with
    accumulate = 1 over a z sub-range, give the one-call ctb_backproject slab."""
    rng = np.random.default_rng(7)
    V, H, W, D = 50, 40, 72, 260.0
    det, grid = ops.detector(W, H, D, u_offset=-0.75)
    X, Y, Z = grid.box
    z0, z1 = 9, Z - 5
    ang = np.sort(rng.uniform(0, 360, V))
    h = rng.uniform(-2.0, 2.0, V)
    proj = torch.from_numpy(rng.standard_normal((V, H, W)).astype(np.float32)).cuda()
    ref = torch.full((z1 - z0, Y, X), float("nan"), device="cuda")
    assert call("ctb_backproject", proj, L.FP32, ang, h, det, grid, ref, z0, z1) == L.CTB_OK
    out = torch.zeros((z1 - z0, Y, X), device="cuda")
    cut = 23
    for a, b in ((0, cut), (cut, V)):
        part = proj[a:b].contiguous()
        assert call("ctb_backproject_noalloc", part, L.FP32, ang[a:b], h[a:b], det, grid, out, z0, z1,
                    accumulate=1) == L.CTB_OK
        torch.cuda.synchronize()  # the second call reuses the shared array
    r = ref.double().cpu().numpy()
    o = out.double().cpu().numpy()
    err = np.linalg.norm((o - r).ravel()) / np.linalg.norm(r.ravel())
    assert err <= 1e-6, err


def test_noalloc_rejects_what_the_allocating_entry_point_rejects():
    det, grid = ops.detector(32, 16, 100.0)
    proj = torch.zeros((2, 16, 32), device="cuda")
    out = torch.zeros(grid.box[::-1], device="cuda")
    bad = L.Grid.from_buffer_copy(grid)
    bad.x_from = -1
    ang = np.zeros(2)
    for name in ("ctb_backproject", "ctb_backproject_noalloc"):
        assert call(name, proj, L.FP32, ang, None, det, bad, out, 0, grid.box[2]) == L.CTB_ERR_ARG
        assert call(name, proj, L.FP32, ang, None, det, grid, out, 0, grid.box[2] + 1) == L.CTB_ERR_ARG
