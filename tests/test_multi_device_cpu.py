"""Host logic of multi-device reconstruction (no GPU).

* getGpuWeights (Ct/CtVolume.cpp:1353-1381) through ctb_gpu_weights_from,
  against the formula restated here;
* the z split of launchCudaThreads (Ct/CtVolume.cpp:1339-1344) through
  ctb_split_slices: consecutive, covering, round(weight * z) slices each;
* the replica plumbing bench.py uses under torchrun (world size 2, gloo):
  max over ranks, per-rank scans, whole-job aggregation.
"""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from ct_b200.ctvolume import gpu_weights_from, split_slices  # noqa: E402


def weights_formula(sm, bw, mp_coef, bw_coef):
    sm = np.asarray(sm, np.float64)
    bw = np.asarray(bw, np.float64)
    w = (sm / sm.sum()) ** mp_coef * (bw / bw.sum()) ** bw_coef
    return w / w.sum()


def test_equal_devices_get_equal_weights():
    w = gpu_weights_from([148] * 8, [8192.0 * 3996000] * 8)
    np.testing.assert_allclose(w, np.full(8, 1 / 8), rtol=0, atol=1e-15)


@pytest.mark.parametrize("coef", [(1.0, 1.0), (1.0, 0.0), (0.0, 1.0), (2.0, 0.5), (0.0, 0.0)])
def test_weights_follow_the_formula(coef):
    sm = [148, 132, 80]
    bw = [8192.0 * 3996000, 5120.0 * 2619000, 4096.0 * 1593000]
    w = gpu_weights_from(sm, bw, *coef)
    np.testing.assert_allclose(w, weights_formula(sm, bw, *coef), rtol=1e-13)
    assert abs(w.sum() - 1) < 1e-12


def test_split_matches_reference_rounding():
    # round(weight * z) slices per device, consecutive from slice 0
    b = split_slices([0.5, 0.3, 0.2], 100)
    assert b.tolist() == [0, 50, 80, 100]
    b = split_slices([0.5, 0.5], 101)   # std::round(50.5) == 51
    assert b.tolist() == [0, 51, 101]


def test_split_covers_every_slice_once():
    # the reference leaves the last slice unassigned for 3 equal devices and
    # z = 100 (3 x 33); here the last device takes it
    b = split_slices([1 / 3] * 3, 100)
    assert b.tolist() == [0, 33, 66, 100]
    rng = np.random.default_rng(3)
    for _ in range(200):
        n = int(rng.integers(1, 9))
        w = rng.random(n)
        w /= w.sum()
        z = int(rng.integers(0, 2000))
        b = split_slices(w, z)
        assert b[0] == 0 and b[-1] == z
        assert np.all(np.diff(b) >= 0)
        for i in range(n - 1):   # every device but the last gets its rounded share, clamped
            assert b[i + 1] - b[i] == min(int(np.floor(w[i] * z + 0.5)), z - b[i])


def test_split_with_tiny_weights_gives_empty_ranges():
    b = split_slices([0.5, 0.25, 0.25], 2)
    assert b.tolist() == [0, 1, 2, 2]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    import torch.distributed as dist

    import bench
    w, r, local = bench.dist_setup()
    assert (w, r, local) == (world, rank, rank)
    bench.barrier(w)
    step_ms = 100.0 + 50.0 * rank          # rank 1 is the slow one
    m = bench.max_over_ranks(step_ms, w)
    out.put((rank, m, bench.scan_seed(rank), bench.whole_job_gups(1e9, w, m)))
    dist.destroy_process_group()


def test_replica_plumbing_gloo_world2():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [150.0, 150.0]     # both ranks see the max
    assert res[0][2] != res[1][2]                      # independent objects per rank
    assert res[0][3] == pytest.approx(2 * 1e9 / 0.150 / 1e9)
