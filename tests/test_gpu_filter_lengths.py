"""The fused preprocessing + ramp filter at the transform lengths the
production scans use: every length of the register four-step kernel
(M = 512 ... 4096, power-of-two widths and widths embedded in the next
length), both paddings and all three windows, FP32, FP16 and BF16 storage.

Reference: convertTo32bit, applyLogScaling, applyFeldkampWeight and
applyFourierFilter with the window functions (Ct/CtVolume.cpp:802-885).
Bars: FP32 <= 1e-5 relative per projection against the reference path
restated by the oracle (pad 1) or against the FP64 oracle (pad 2); FP16
<= 2e-3 and BF16 <= 1e-2 against the FP64 oracle.
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


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def raw_set(W, H=6, V=2, seed=0):
    rng = np.random.default_rng(seed)
    # smooth attenuation profile plus noise, like a real projection
    u = np.linspace(-1, 1, W)
    base = 60000 * np.exp(-1.5 * np.clip(1 - u ** 2, 0, None))
    imgs = base[None, None, :] + rng.normal(0, 800, (V, H, W))
    return np.clip(imgs, 1000, 65535).astype(np.uint16)


def run(imgs, ft, pad, store=L.FP32, scale=1.0):
    V, H, W = imgs.shape
    det, _ = ops.detector(W, H, 2.0 * W)
    raw = torch.from_numpy(imgs.astype(np.int32)).to(torch.uint16).cuda()
    out = ops.filter_projections(raw, det, ft, pad, store, scale)
    torch.cuda.synchronize()
    return out.float().cpu().numpy() / scale, 2.0 * W


# power-of-two widths: M = W; other widths embed the length-W circular filter
# into M = nextpow2(2W - 1): 300 -> 1024, 700 -> 2048, 1500 -> 4096
@pytest.mark.parametrize("W", [512, 1024, 2048, 4096, 300, 700, 1500])
@pytest.mark.parametrize("ft", [L.RAMLAK, L.SHEPPLOGAN, L.HANN])
def test_reference_filter_at_production_lengths(oracle, W, ft):
    imgs = raw_set(W, seed=W + ft)
    out, FCD = run(imgs, ft, 1)
    for v in range(imgs.shape[0]):
        ref = oracle.ref_preprocess(imgs[v], 1.0, FCD, ft)
        assert rel_l2(out[v], ref) <= 1e-5, (v, rel_l2(out[v], ref))


# pad 2: 1024 -> 2048, 2048 -> 4096 (four-step kernel), 4096 -> 8192 (Stockham kernel)
@pytest.mark.parametrize("W", [1024, 2048, 4096])
@pytest.mark.parametrize("ft", [L.RAMLAK, L.HANN])
def test_padded_filter_at_production_lengths(oracle, W, ft):
    imgs = raw_set(W, seed=3 * W + ft)
    out, FCD = run(imgs, ft, 2)
    for v in range(imgs.shape[0]):
        ref = oracle.f64_preprocess(imgs[v], 1.0, FCD, ft, pad=2)
        assert rel_l2(out[v], ref) <= 1e-5, (v, rel_l2(out[v], ref))


@pytest.mark.parametrize("store", [L.FP16, L.BF16])
@pytest.mark.parametrize("W,pad", [(2048, 1), (1024, 2), (2048, 2)])
def test_half_storage_at_production_lengths(oracle, store, W, pad):
    imgs = raw_set(W, seed=7 * W + pad + store)
    out, FCD = run(imgs, L.HANN, pad, store, 1.0 / W)
    tol = 2e-3 if store == L.FP16 else 1e-2
    for v in range(imgs.shape[0]):
        ref = oracle.f64_preprocess(imgs[v], 1.0, FCD, L.HANN, pad=pad)
        assert rel_l2(out[v], ref) <= tol, (v, rel_l2(out[v], ref))
