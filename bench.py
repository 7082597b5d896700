"""FDK throughput on one B200 per rank: GUPS = voxels x views / s.

Workload (default, "c3"): 1440 views over 360 deg of a 2048 x 2048 detector
(0.2 mm pitch, SOD 500 mm, SDD 1000 mm, effective pitch 0.1 mm), reconstructed
into a 1024^3 float32 volume of 0.2 mm voxels (2 detector pixels), hann
filter, projections and filtered projections stored in FP16, FP32 arithmetic.
Synthetic input: 50 seeded ellipsoids (10 small high-contrast ones), analytic
line integrals, I = 65535 exp(-0.02 p) as uint16.

One step = preprocess + ramp-filter every view and backproject the whole
volume, inputs resident in HBM (`value`); `e2e` is the same reconstruction
through the C ABI facade from pinned host uint16 projections to a pinned host
float volume (H2D and D2H inside the timed region). Inputs (12 GB) are larger
than L2, so no flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--config c3|c2|c1]
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CONFIGS = {
    # name: views, W, H, pitch, SOD, SDD, grid edge, voxel pitch (detector px), ellipsoids, small, filter, photons
    "c3": dict(views=1440, W=2048, H=2048, pitch=0.2, sod=500.0, sdd=1000.0, edge=1024, vs=2.0, n_ell=40,
               n_small=10, filter="hann", photons=None),
    "c2": dict(views=720, W=1024, H=1024, pitch=0.4, sod=500.0, sdd=1000.0, edge=512, vs=2.0, n_ell=30,
               n_small=0, filter="shepplogan", photons=1e5),
    "c1": dict(views=360, W=256, H=192, pitch=1.0, sod=500.0, sdd=1000.0, edge=256, vs=1.0, n_ell=10,
               n_small=0, filter="ramlak", photons=None),
}
FILTERS = {"ramlak": 0, "shepplogan": 1, "hann": 2}

# DRAM bytes (read + write) of one backprojection launch per voxel-view update, from
# ncu captures (dram__bytes_read.sum + dram__bytes_write.sum, one pass) of the C3 bench's
# two 512-slice launches (1024 x 1024 x 512 voxels x 1440 views of 2048^2, FP16 storage):
# 620.2 + 2.29 GB and 658.5 + 2.29 GB over 7.73e11 updates each
BP_DRAM_BYTES_PER_UPDATE = {("c3", 512): ((620.229e9 + 2.292e9) + (658.527e9 + 2.288e9)) / 2
                            / (1024 * 1024 * 512 * 1440)}


# --------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi samples during the timed region (SM clock, throttle reasons)."""
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.device)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[0]))
                mx.append(float(f[1]))
            except ValueError:
                continue
            for n, v in zip(names, f[4:8]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ----------------------------------------------------------------- helpers
def geometry(cfg):
    from ct_b200 import synth
    return synth.ScanGeometry(cfg["views"], cfg["W"], cfg["H"], cfg["pitch"], cfg["sod"], cfg["sdd"])


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d, "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "sm_max_mhz": 1965.0}, "fallback"


# ------------------------------------------------------ reference CPU path
# The reference's own CPU reconstruction (its Ct/CtVolume.cpp lines compiled
# unchanged into oracle/_ref/libct_ref.so) on the host cores; the oracle's
# restatement of it (bit-identical) when that library is absent.
REF_SAMPLE_VIEWS = 4
REF_SAMPLE_Z = (0.4375, 0.5625)   # central eighth of the reference grid's slices (its own zmin/zmax)


def reference_cpu_available() -> bool:
    from oracle import oracle as orc
    try:
        orc.ref_lib()
        return True
    except (FileNotFoundError, OSError, subprocess.CalledProcessError):
        return False


def cpu_phantom_views(cfg, geom, seed, sel):
    """uint16 projections of the seeded phantom (the GPU arm's scan of rank 0) for the views `sel`, projected
    on the CPU (numpy), so the reference arm runs none of the engine."""
    import concurrent.futures as cf
    import multiprocessing as mp
    from oracle import phantom
    from ct_b200 import synth
    rng = np.random.default_rng(seed)
    r_mm, hz_mm = synth.fov(geom)
    ell = synth.random_ellipsoids(rng, cfg["n_ell"], r_mm, hz_mm, n_small=cfg["n_small"])
    ang = geom.angles()[sel]
    parts = np.array_split(np.arange(len(ang)), min(len(ang), os.cpu_count() or 1))
    # one process per group of views (spawned: no CUDA state is inherited)
    with cf.ProcessPoolExecutor(len(parts), mp_context=mp.get_context("spawn")) as ex:
        futs = [ex.submit(phantom.project, ell, ang[idx], None, geom.width, geom.height, geom.pixel_eff,
                          geom.sod_mm) for idx in parts]
        p = np.concatenate([f.result() for f in futs])
    return synth.intensities_from_line_integrals(p)


def reference_cpu_step(cfg, geom, imgs, angles, zrel=REF_SAMPLE_Z, full=False):
    """One timed run of the reference's CPU path: load the views, set the bounds (x, y whole, z the central
    slices zrel of the reference grid; `full`: the whole grid), reconstructionCore. Returns the measured
    wall time and voxel-views of the box it reconstructed."""
    from oracle import oracle as orc
    use_ref = reference_cpu_available()
    rel = None if full else (0.0, 1.0, 0.0, 1.0, zrel[0], zrel[1])
    ft = FILTERS[cfg["filter"]]
    t0 = time.perf_counter()
    if use_ref:
        # timed inside: the zeroed volume and reconstructionCore, what the reference's
        # reconstructVolume does for its CPU path (Ct/CtVolume.cpp:553-573)
        dims, secs = orc.refsrc_reconstruct(imgs, angles, None, geom.pixel_eff, geom.sod_mm, rel=rel,
                                            filter_type=ft, keep_volume=False)
    else:
        FCD = float(np.float32(geom.sod_mm) / np.float32(geom.pixel_eff))
        g = orc.ref_geom(geom.width, geom.height, FCD, rel=orc.clamp_bounds(*rel) if rel else (0, 1, 0, 1, 0, 1))
        a, h = orc.fix_sinogram(angles, np.zeros(len(angles)), True, geom.pixel_eff)
        vol, secs = orc.ref_reconstruct(imgs, a, h, 1.0, ft, g)
        dims = vol.shape
        del vol
    wall = time.perf_counter() - t0
    units = float(np.prod(dims)) * len(angles)
    return {"seconds": secs, "call_seconds": wall, "voxel_views": units, "box": list(dims),
            "kind": "reference" if use_ref else "port", "cores": orc.num_threads()}


def reference_c1_full(seed=1000):
    """The reference's CPU path on the whole 360-view scan of 256 x 192 into its 252^2 x 192 grid, measured."""
    cfg = CONFIGS["c1"]
    geom = geometry(cfg)
    imgs = cpu_phantom_views(cfg, geom, seed, np.arange(geom.n_views))
    r = reference_cpu_step(cfg, geom, imgs, geom.angles(), full=True)
    return {"workload": "360 views x 256x192 u16 -> 252x252x192 f32 (reference grid), ramlak", "seconds": r["seconds"],
            "gups": r["voxel_views"] / r["seconds"] / 1e9, "kind": r["kind"], "cores": r["cores"]}


def cpu_baseline(cfg, geom, imgs_sel, angles_sel, units_full):
    """The reference's CPU path on a bounded sample of the workload, measured: REF_SAMPLE_VIEWS evenly spaced
    views of this scan reconstructed by the reference's own code into the central slices of its own grid
    (voxel = 1 detector pixel; it has no coarser voxels). value = voxel-views per second of that run."""
    r = reference_cpu_step(cfg, geom, imgs_sel, angles_sel)
    gups = r["voxel_views"] / r["seconds"] / 1e9
    X, Y, Z = r["box"]
    return {"value": gups, "unit": "GUPS", "cores": r["cores"], "kind": r["kind"],
            "sample": (f"{len(angles_sel)} of {geom.n_views} views, reference grid box {X}x{Y}x{Z} (z "
                       f"{REF_SAMPLE_Z[0]}..{REF_SAMPLE_Z[1]}): {r['seconds']:.2f} s for the zeroed volume and "
                       f"reconstructionCore ({r['call_seconds']:.2f} s with loading) on {r['cores']} threads"),
            "seconds": r["seconds"],
            "seconds_full_workload_at_this_rate": units_full / (gups * 1e9)}


def log(*a):
    print("[bench]", *a, file=sys.stderr, flush=True)


def oracle_rows(raw, geom, det, grid, z0, z1):
    """The detector rows that box slices [z0, z1) touch in any view, copied to the host."""
    import torch
    V, H, W = raw.shape
    vs = grid.voxel_pitch
    zpre = grid.z_size / 2.0 - grid.z_from
    zw = np.array([(z0 - zpre) * vs, (z1 - 1 - zpre) * vs])
    R, D = float(det.radius), float(det.fcd)
    v = np.outer(zw, np.array([D / (D + R), D / (D - R)])).ravel()
    r0 = max(0, int(math.floor(H / 2.0 - v.max())) - 2)
    r1 = min(H, int(math.floor(H / 2.0 - v.min())) + 3)
    return r0, raw[:, r0:r1, :].to(torch.int32).cpu().numpy().astype(np.uint16)


def fp64_reference_slices(rows, cfg, geom, det, grid, z0, z1):
    """FP64 oracle reconstruction of box slices [z0, z1) from only the detector rows they touch."""
    from oracle import oracle as orc
    orc.build()
    r0, rows = rows
    V, _, W = rows.shape
    H = det.height
    vs = grid.voxel_pitch
    g = orc.custom_geom(W, H, float(det.fcd), (grid.x_size, grid.y_size, grid.z_size), vs,
                        box=(grid.x_from, grid.x_to, grid.y_from, grid.y_to, grid.z_from, grid.z_to))
    ref = orc.f64_slices(rows, r0, H, geom.angles(), np.zeros(V), 1.0, FILTERS[cfg["filter"]], g, z0, z1)
    return ref  # (x, y, z1 - z0)


def accuracy_slices(Z):
    """Slices scored against the FP64 oracle: both ends (largest cone angle), the octiles and the centre."""
    return sorted({0, Z // 8, Z // 4, Z // 2 - 1, Z // 2, 3 * Z // 4, 7 * Z // 8, Z - 1})


def fp64_slice_set(raw, cfg, geom, det, grid, zs):
    """FP64 oracle values of the box slices zs, each from only the detector rows it touches: (x, y, len(zs))."""
    return np.concatenate([fp64_reference_slices(oracle_rows(raw, geom, det, grid, z, z + 1), cfg, geom, det, grid,
                                                 z, z + 1) for z in zs], axis=2)


def accuracy(vol_slices_zyx, ref_xyz):
    a = np.asarray(vol_slices_zyx, np.float64).transpose(2, 1, 0)
    d = a - ref_xyz
    return {"rel_l2": float(np.linalg.norm(d.ravel()) / np.linalg.norm(ref_xyz.ravel())),
            "max_abs": float(np.abs(d).max()), "ref_max_abs": float(np.abs(ref_xyz).max())}


def dist_setup():
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1 and not dist.is_initialized():
        import datetime
        if torch.cuda.is_available():
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                    device_id=torch.device("cuda", local))
        else:  # host-only runs of the rank plumbing
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    return world, rank, local


def barrier(world):
    import torch.distributed as dist
    if world > 1:
        dist.barrier()


def max_over_ranks(x: float, world: int) -> float:
    import torch
    import torch.distributed as dist
    if world == 1:
        return x
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def scan_seed(rank: int) -> int:
    """Each rank reconstructs its own object (weak scaling, no data-path collective)."""
    return 1000 + rank


def whole_job_gups(voxel_views_per_rank: float, world: int, ms_per_step: float) -> float:
    """Whole-job throughput: the units all ranks processed over the max-over-ranks step time."""
    return voxel_views_per_rank * world / (ms_per_step * 1e-3) / 1e9


# ---------------------------------------------------------------- batch (C5)
def batch_c5(n_scans=32, seed=5, store="fp16", reps=3):
    """C5: 32 independent scans, detector W and H ~ U[128, 768], views ~ U[90, 720], volume edge ~ U[96, 384]
    float32, SOD ~ U[300, 700] mm, magnification ~ U[1.5, 2.5], 5-25 seeded ellipsoids each. Aggregate GUPS of
    the persistent graph-captured batch against launching the scans one by one."""
    import torch

    from ct_b200 import ops, synth
    from ct_b200 import _lib as L
    rng = np.random.default_rng(seed)
    st = {"fp16": L.FP16, "bf16": L.BF16, "fp32": L.FP32}[store]
    scans, units = [], 0.0
    for i in range(n_scans):
        W, H = int(rng.integers(128, 769)), int(rng.integers(128, 769))
        V = int(rng.integers(90, 721))
        edge = int(rng.integers(96, 385))
        sod = float(rng.uniform(300, 700))
        mag = float(rng.uniform(1.5, 2.5))
        pitch = 0.2
        geom = synth.ScanGeometry(V, W, H, pitch, sod, sod * mag)
        sc = synth.make_scan(geom, int(rng.integers(5, 26)), seed=seed * 1000 + i)
        det, _ = ops.detector(W, H, float(np.float32(geom.fcd_px)))
        # the volume spans the detector's field of view at the detector pixel pitch scaled to the edge
        vs = float(W) / edge
        grid = ops.custom_grid(det, (edge, edge, edge), vs)
        vol = torch.empty((edge, edge, edge), device="cuda")
        scans.append(dict(raw=sc.images, angles_deg=geom.angles(), heights_px=None, det=det, grid=grid,
                          filter=int(rng.integers(0, 3)), pad=1, vol=vol))
        units += float(edge) ** 3 * V
    b = ops.Batch(scans, st)
    stream = torch.cuda.current_stream()

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    ms_graph = timed(b.run)
    ms_seq = timed(b.run_sequential)
    out = {"scans": n_scans, "voxel_views": units, "storage": store,
           "graph_persistent": {"ms": ms_graph, "gups": units / (ms_graph * 1e-3) / 1e9},
           "one_by_one": {"ms": ms_seq, "gups": units / (ms_seq * 1e-3) / 1e9},
           "speedup": ms_seq / ms_graph, "autotune": b.tuning()}
    del b, scans
    torch.cuda.empty_cache()
    return out


# ------------------------------------------------------------ C2 (FP32)
def c2_leg(reps=3, with_accuracy=True):
    """C2: 720 views of 1024 x 1024 (0.4 mm pitch, SOD 500, SDD 1000), 30 seeded ellipsoids with Poisson
    noise at 1e5 photons, shepplogan, FP32 storage, into 512^3 (voxel 2 detector pixels) and into the
    0.25..0.75 sub-box (256^3). Device time (filter + backprojection, CUDA events) and rel-L2 / max-abs of
    eight slices per box against the FP64 oracle."""
    import torch

    from ct_b200 import ops, synth
    from ct_b200 import _lib as L
    cfg = CONFIGS["c2"]
    geom = geometry(cfg)
    V, W, H, edge, vs = geom.n_views, geom.width, geom.height, cfg["edge"], cfg["vs"]
    ft = FILTERS[cfg["filter"]]
    scan = synth.make_scan(geom, cfg["n_ell"], seed=2000, photons=cfg["photons"], n_small=cfg["n_small"])
    raw, angles = scan.images, geom.angles()
    det, _ = ops.detector(W, H, geom.fcd_px)
    stream = torch.cuda.current_stream()
    out = {"workload": f"c2: {V} views x {W}x{H} u16 -> {edge}^3 f32 (voxel {vs} px), {cfg['filter']}, fp32 storage, "
                       f"Poisson 1e5"}
    filtered = torch.empty((V, H, W), dtype=torch.float32, device="cuda")
    for name, rel in (("full", (0.0, 1.0)), ("subbox_0.25_0.75", (0.25, 0.75))):
        lo, hi = int(rel[0] * edge + 0.5), int(rel[1] * edge + 0.5)
        grid = ops.custom_grid(det, (edge, edge, edge), vs, box=(lo, hi, lo, hi, lo, hi))
        X, Y, Z = grid.box
        vol = torch.empty((Z, Y, X), dtype=torch.float32, device="cuda")

        def step():
            ops.filter_projections(raw, det, ft, 1, L.FP32, 1.0, out=filtered)
            ops.backproject(filtered, angles, None, det, grid, out=vol)

        step()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        r = {"volume": [X, Y, Z], "ms": ms, "gups": float(X) * Y * Z * V / (ms * 1e-3) / 1e9}
        if with_accuracy:
            zs = accuracy_slices(Z)
            got = vol[torch.tensor(zs, device="cuda")].cpu().numpy()
            ref = fp64_slice_set(raw, cfg, geom, det, grid, zs)
            r["accuracy_vs_fp64"] = {"slices": zs, "fp32": accuracy(got, ref)}
        out[name] = r
        del vol
    del filtered, raw, scan
    torch.cuda.empty_cache()
    return out


# ------------------------------------------------------- differentiation (C4)
def voxelise_gpu(ellipsoids, edge, voxel_mm):
    """Phantom density at the voxel centres of an edge^3 grid centred on the axis, (Z, Y, X) float32."""
    import torch
    c = (torch.arange(edge, device="cuda", dtype=torch.float64) - edge / 2.0) * voxel_mm
    out = torch.zeros((edge, edge, edge), device="cuda", dtype=torch.float32)
    Z, Y = torch.meshgrid(c, c, indexing="ij")
    for E in np.asarray(ellipsoids, np.float64):
        R = torch.tensor(E[6:15].reshape(3, 3), device="cuda", dtype=torch.float64)
        for xi in range(0, edge, 64):  # chunks of x keep the temporaries small
            X = c[xi:xi + 64]
            P = torch.stack(torch.broadcast_tensors(X[None, None, :], Y[:, :, None], Z[:, :, None]), -1)
            q = ((P - torch.tensor(E[:3], device="cuda")) @ R) / torch.tensor(E[3:6], device="cuda")
            out[:, :, xi:xi + 64] += torch.where((q * q).sum(-1) <= 1.0, float(E[15]), 0.0).float()
    return out


def gradient_c4(edge=512, views=360, det=512, iters=20, seed=4):
    """C4: matched forward projector A and backprojector A^T on a 512^3 float32 volume, 360 views of
    512x512. Dot-product test <Ax, y> = <x, A^T y> with seeded Gaussian x, y; device time of A and A^T;
    central finite differences of f(x) = ||Ax - p||^2 on 64 random voxels against 2 A^T (Ax - p)
    (A(x +- eps e_i) = Ax +- eps A e_i, with A e_i projected from a one-slice slab holding the voxel);
    then 20 steepest-descent iterations with exact line search from the FDK reconstruction.
    Data as the configuration states them: the analytic projections of a 20-ellipsoid phantom with Poisson
    noise at 1e4 photons, as line integrals in voxel lengths (-ln(I / I0) / 0.02 / voxel mm; with the U^2
    weight, A of a density is its line integral in voxel lengths). The same descent on model-consistent
    data (A of the voxelised phantom + 1 % Gaussian noise) is reported beside it."""
    import torch

    from ct_b200 import ops, synth
    from ct_b200 import _lib as L
    geom = synth.ScanGeometry(views, det, det, 0.4, 500.0, 1000.0)
    d, _ = ops.detector(det, det, float(np.float32(geom.fcd_px)))
    grid = ops.custom_grid(d, (edge, edge, edge), 1.0)
    ang = geom.angles()
    units = float(edge) ** 3 * views
    out = {"volume": [edge] * 3, "views": views, "detector": [det, det], "voxel_views_per_op": units}
    t0 = time.perf_counter()
    g = torch.Generator(device="cuda").manual_seed(seed)
    x = torch.randn((edge, edge, edge), device="cuda", generator=g)
    y = torch.randn((views, det, det), device="cuda", generator=g)
    Ax = ops.forward_project(x, ang, None, d, grid)
    Aty = ops.backproject(y, ang, None, d, grid)
    lhs, rhs = float((Ax.double() * y.double()).sum()), float((x.double() * Aty.double()).sum())
    out["dot_test_rel"] = abs(lhs - rhs) / max(abs(lhs), abs(rhs))
    # device time of one A and one A^T (CUDA events around each call, after the warm-up
    # above; the median of five)
    def per_call(fn, reps=5):
        ts = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        return float(np.median(ts)), float(np.min(ts)), float(np.max(ts))

    fp_ms, fp_min, fp_max = per_call(lambda: ops.forward_project(x, ang, None, d, grid, out=Ax))
    bp_ms, bp_min, bp_max = per_call(lambda: ops.backproject(y, ang, None, d, grid, out=Aty))
    out["forward_ms_min_max"] = [fp_min, fp_max]
    out["backproject_ms_min_max"] = [bp_min, bp_max]
    out.update({"forward_ms": fp_ms, "forward_gups": units / fp_ms / 1e6,
                "backproject_fp32_ms": bp_ms, "backproject_fp32_gups": units / bp_ms / 1e6})
    del Ax, Aty, y, x
    scan = synth.make_scan(geom, 20, seed=seed, photons=1e4)
    voxel_mm = geom.pixel_eff
    truth = voxelise_gpu(scan.ellipsoids, edge, voxel_mm)
    # FDK (hann, FP32) of the noisy analytic projections
    filt = ops.filter_projections(scan.images, d, L.HANN, 1, L.FP32)
    fdk = ops.backproject(filt, ang, None, d, grid)
    del filt

    def err_to_truth(v):
        vs = v.double()
        s_fit = float((vs * truth).sum() / (vs * vs).sum())
        return float((s_fit * vs - truth).norm() / truth.norm())

    def descend(p, fd_check):
        """Steepest descent on ||Ax - p||^2 from the FDK volume scaled to p by least squares."""
        x = fdk.clone()
        Ax = ops.forward_project(x, ang, None, d, grid)
        c = float((Ax.double() * p.double()).sum() / (Ax.double() * Ax.double()).sum())
        x.mul_(c)
        r = Ax.mul_(c).sub_(p)
        res = {}
        if fd_check:
            grad = 2.0 * ops.backproject(r, ang, None, d, grid)
            rng = np.random.default_rng(seed)
            eps, worst = 1.0, 0.0
            for _ in range(64):
                k, j, i = (int(rng.integers(edge // 4, 3 * edge // 4)) for _ in range(3))
                slab = torch.zeros((1, edge, edge), device="cuda")
                slab[0, j, i] = 1.0
                Ae = ops.forward_project(slab, ang, None, d, grid, k, k + 1).double()
                rd = r.double()
                fp = float(((rd + eps * Ae) ** 2).sum())
                fm = float(((rd - eps * Ae) ** 2).sum())
                fd = (fp - fm) / (2 * eps)
                gi = float(grad[k, j, i])
                worst = max(worst, abs(fd - gi) / max(abs(fd), 1e-12))
            del grad
            res["fd_max_rel_err_64_voxels"] = worst
        res0 = float(r.double().norm() / p.double().norm())
        err0 = err_to_truth(x)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        for _ in range(iters):
            gk = 2.0 * ops.backproject(r, ang, None, d, grid)
            Ag = ops.forward_project(gk, ang, None, d, grid)
            alpha = float((gk.double() ** 2).sum() / (2.0 * (Ag.double() ** 2).sum()))
            x.sub_(alpha * gk)
            r.sub_(alpha * Ag)
            del gk, Ag
        torch.cuda.synchronize()
        t_it = (time.perf_counter() - t1) / iters
        res.update({"data_residual_rel_start": res0, "data_residual_rel_after": float(r.double().norm() /
                                                                                       p.double().norm()),
                    "iterations": iters, "rel_l2_to_phantom_start": err0, "rel_l2_to_phantom_after": err_to_truth(x),
                    "seconds_per_iteration": t_it})
        del x, r
        return res

    # the configuration's data: analytic Poisson-1e4 projections as line integrals in voxel lengths
    p = (-torch.log(scan.images.float().clamp_min(1.0) / 65535.0) / 0.02 / voxel_mm).contiguous()
    a = descend(p, fd_check=True)
    out["fd_max_rel_err_64_voxels"] = a.pop("fd_max_rel_err_64_voxels")
    out["analytic_poisson_1e4"] = a
    # model-consistent data: A(truth) + 1 % Gaussian noise
    p = ops.forward_project(truth, ang, None, d, grid)
    p.add_(torch.randn(p.shape, device="cuda", generator=g), alpha=0.01 * float(p.double().pow(2).mean().sqrt()))
    out["model_consistent"] = descend(p, fd_check=False)
    out["seconds_total"] = time.perf_counter() - t0
    del p, truth, scan, fdk
    torch.cuda.empty_cache()
    return out


def facade_split(v, host_out, n, V, W, H, Z, Y, X, units, edge, vs, det, geom, reps=2):
    """One scan through the facade with the active device list [0] * n (the reference's launchCudaThreads
    z split, Ct/CtVolume.cpp:1322-1351): per-worker slices and detector row bands, bytes copied, seconds,
    and the largest difference from the one-device volume already in host_out."""
    import torch

    from ct_b200 import ops
    from ct_b200 import _lib as L
    one = host_out.clone()
    v.setActiveCudaDevices([0] * n)   # one-process leg, run at world size 1 only
    weights = np.full(n, 1.0 / n)
    begin = np.zeros(n + 1, np.int32)
    L.lib().ctb_split_slices(weights.ctypes.data, n, Z, begin.ctypes.data)
    grid = v.grid()
    workers = []
    for i in range(n):
        r_lo, rows = ops.row_band(v.detector(), grid, int(begin[i]), int(begin[i + 1]))
        workers.append({"slices": [int(begin[i]), int(begin[i + 1])], "detector_rows": [r_lo, r_lo + rows]})
    v.reconstructInto(host_out.data_ptr(), L.X_FASTEST)  # warm-up of the new workers
    ts = []
    for _ in range(reps):
        t0 = time.perf_counter()
        v.reconstructInto(host_out.data_ptr(), L.X_FASTEST)
        ts.append(time.perf_counter() - t0)
    tm = v.timings()
    diff = float((host_out - one).abs().max())
    scale = float(one.abs().max())
    v.setActiveCudaDevices([0])
    del one
    return {"devices": [0] * n, "workers": workers, "seconds": float(np.mean(ts)),
            "gups": units / float(np.mean(ts)) / 1e9, "h2d_bytes": int(tm.h2d_bytes),
            "d2h_bytes": int(tm.d2h_bytes), "max_abs_diff_vs_one_device": diff, "volume_max_abs": scale,
            "note": "workers share one GPU here (device 0 listed twice): no speed-up is expected; on n GPUs each "
                    "moves only its detector row band"}


L2_BYTES = 126 << 20


def working_set_bytes(args):
    """Bytes the device pass touches: raw and filtered projections, the volume."""
    cfg = CONFIGS[args.config]
    V, W, H, edge = cfg["views"], cfg["W"], cfg["H"], cfg["edge"]
    store_bytes = 4 if args.store == "fp32" else 2
    return V * H * W * (2 + store_bytes) + edge ** 3 * 4


def needs_l2_flush(args):
    """Whether that working set is small enough for L2 to keep much of it between timed steps
    (C1): then L2 is flushed between steps."""
    return working_set_bytes(args) < 4 * L2_BYTES


def workload_config(args, world):
    """The `config` object of the bench line (both arms print the same one)."""
    cfg = CONFIGS[args.config]
    V, W, H, edge, vs = cfg["views"], cfg["W"], cfg["H"], cfg["edge"], cfg["vs"]
    rel = (0.25, 0.75) if args.subbox else (0.0, 1.0)
    n = int(rel[1] * edge + 0.5) - int(rel[0] * edge + 0.5)
    return {"workload": f"{args.config}: {V} views x {W}x{H} u16 -> {n}x{n}x{n} f32 (voxel {vs} px), "
                        f"{cfg['filter']}, {args.store} storage"
                        + (f", sub-box 0.25..0.75 of {edge}^3" if args.subbox else ""),
            "storage": args.store, "views": V, "detector": [W, H], "volume": [n, n, n], "voxel_pitch_px": vs,
            "slab": args.slab,
            "l2": (f"inputs ({V * H * W * 2 / 1e9:.1f} GB raw) larger than L2 (126 MB); no flush"
                   if not needs_l2_flush(args) else
                   f"working set ({working_set_bytes(args) / 1e6:.0f} MB of projections and volume) within 4x L2 "
                   f"(126 MB): a 256 MB buffer is written between timed steps, outside the step events"),
            "parallelism": f"replicas{world}"}


# ------------------------------------------------------------------ our arm
def run_ours(args):
    import torch

    from ct_b200 import CtVolume, ops, synth
    from ct_b200 import _lib as L

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    cfg = CONFIGS[args.config]
    geom = geometry(cfg)
    V, W, H = geom.n_views, geom.width, geom.height
    edge, vs = cfg["edge"], cfg["vs"]
    ft = FILTERS[cfg["filter"]]
    store = {"fp16": L.FP16, "bf16": L.BF16, "fp32": L.FP32}[args.store]

    # independent scan per rank (weak scaling: each rank reconstructs its own object)
    scan = synth.make_scan(geom, cfg["n_ell"], seed=scan_seed(rank), photons=cfg["photons"], n_small=cfg["n_small"])
    raw = scan.images
    angles = geom.angles()
    det, _ = ops.detector(W, H, geom.fcd_px)
    # --subbox: the reference's xmin..zmax = 0.25..0.75 bounds (from/to = floor(f * size + 0.5))
    rel = (0.25, 0.75) if args.subbox else (0.0, 1.0)
    lo, hi = int(rel[0] * edge + 0.5), int(rel[1] * edge + 0.5)
    grid = ops.custom_grid(det, (edge, edge, edge), vs, box=(lo, hi, lo, hi, lo, hi))
    X, Y, Z = grid.box
    units = float(X) * Y * Z * V
    slab = args.slab
    slabs = [(z, min(Z, z + slab)) for z in range(0, Z, slab)]
    stream = torch.cuda.current_stream()

    def device_pass(store_t, filtered, vol, ev=None):
        scale = 1.0 if store_t == L.FP32 else 1.0 / W
        if ev is not None:
            ev[0].record(stream)
        ops.filter_projections(raw, det, ft, 1, store_t, scale, out=filtered)
        if ev is not None:
            ev[1].record(stream)
        for (a, b) in slabs:
            ops.backproject(filtered, angles, None, det, grid, a, b, load_scale=1.0 / scale, out=vol[a:b])
        if ev is not None:
            ev[2].record(stream)

    def timed(store_t, steps, warmup):
        dt = {L.FP32: torch.float32, L.FP16: torch.float16, L.BF16: torch.bfloat16}[store_t]
        filtered = torch.empty((V, H, W), dtype=dt, device="cuda")
        vol = torch.empty((Z, Y, X), dtype=torch.float32, device="cuda")
        for _ in range(warmup):
            device_pass(store_t, filtered, vol)
        torch.cuda.synchronize()
        barrier(world)
        torch.cuda.synchronize()
        evs = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(steps)]
        clk = ClockSampler(local)
        clk.start()
        start = torch.cuda.Event(enable_timing=True)
        end = torch.cuda.Event(enable_timing=True)
        flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda") if needs_l2_flush(args) else None
        start.record(stream)
        for k in range(steps):
            if flush is not None:
                flush.fill_(k & 0xff)   # evicts the previous step's data from L2 (outside the step events)
            device_pass(store_t, filtered, vol, evs[k])
        end.record(stream)
        torch.cuda.synchronize()
        clocks = clk.stop()
        barrier(world)
        # with flushes the steps are timed by their own events (filter start to backprojection end)
        total_ms = (start.elapsed_time(end) if flush is None
                    else float(sum(e[0].elapsed_time(e[2]) for e in evs)))
        del flush
        f_ms = float(np.mean([e[0].elapsed_time(e[1]) for e in evs]))
        b_ms = float(np.mean([e[1].elapsed_time(e[2]) for e in evs]))
        out = {"total_ms": max_over_ranks(total_ms, world), "filter_ms": f_ms, "bp_ms": b_ms, "clocks": clocks}
        del filtered
        sel = vol[torch.tensor(acc_z, device="cuda")].cpu().numpy()
        del vol
        torch.cuda.empty_cache()
        return out, sel

    acc_z = accuracy_slices(Z)
    log(f"scan ready: {V} views {W}x{H} -> {X}x{Y}x{Z}")
    main, slices_main = timed(store, args.steps, args.warmup)
    ms_per_step = main["total_ms"] / args.steps
    value = whole_job_gups(units, world, ms_per_step)
    log(f"{args.store}: {ms_per_step:.1f} ms/step, {value:.1f} GUPS, filter {main['filter_ms']:.1f} ms, "
        f"bp {main['bp_ms']:.1f} ms, clocks {main['clocks']}")

    # plain FP32 path on the same workload (mixed vs plain ratio)
    fp32, slices32 = None, None
    if store != L.FP32 and not args.skip_fp32:
        r32, slices32 = timed(L.FP32, max(2, args.steps // 2), 1)
        ms32 = r32["total_ms"] / max(2, args.steps // 2)
        fp32 = {"value": whole_job_gups(units, world, ms32), "ms_per_step": ms32, "bp_ms": r32["bp_ms"],
                "filter_ms": r32["filter_ms"]}
        log(f"fp32: {fp32}")
    # the other 16-bit storage type on the same workload
    other = {L.FP16: ("bf16", L.BF16), L.BF16: ("fp16", L.FP16)}.get(store)
    alt, slices_alt = None, None
    if other and not args.skip_fp32:
        ra, slices_alt = timed(other[1], max(2, args.steps // 2), 1)
        msa = ra["total_ms"] / max(2, args.steps // 2)
        alt = {"value": whole_job_gups(units, world, msa), "ms_per_step": msa, "bp_ms": ra["bp_ms"],
               "filter_ms": ra["filter_ms"]}
        log(f"{other[0]}: {alt}")

    # the FP64-oracle accuracy of these slices is computed in the CPU leg below
    acc = None

    # end to end through the C ABI facade: pinned host u16 -> pinned host float volume
    e2e = None
    if not args.skip_e2e:
        host_in = torch.empty((V, H, W), dtype=torch.uint16, pin_memory=True)
        host_in.copy_(raw)
        host_out = torch.empty((Z, Y, X), dtype=torch.float32, pin_memory=True)
        v = CtVolume()
        v.setActiveCudaDevices([local])   # this rank's GPU (the facade's default is device 0)
        v.setProjectionsPointer(host_in.data_ptr(), L.U16, V, W, H, angles, None, pixel_size=geom.pixel_eff,
                                rotation="ccw", fcd_mm=geom.sod_mm, keep=host_in)
        v.setGrid(edge, edge, edge, vs)
        v.setVolumeBounds(rel[0], rel[1], rel[0], rel[1], rel[0], rel[1])
        v.setFrequencyFilterType(cfg["filter"])
        v.setPrecision(args.store)
        if args.e2e_slab > 0:
            v.setSlabHeight(args.e2e_slab)   # else the facade's own (or the autotuner's) choice
        else:
            v.setAutotune(True)              # the first warm-up reconstruction tunes the backprojection
        for _ in range(args.warmup):
            v.reconstructInto(host_out.data_ptr(), L.X_FASTEST)
        barrier(world)
        ts = []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            v.reconstructInto(host_out.data_ptr(), L.X_FASTEST)
            ts.append(time.perf_counter() - t0)
        barrier(world)
        tm = v.timings()
        sec = max_over_ranks(float(np.mean(ts)), world)
        e2e = {"value": whole_job_gups(units, world, sec * 1e3), "unit": "GUPS", "seconds": sec,
               "h2d_bytes_per_step": int(tm.h2d_bytes), "d2h_bytes_per_step": int(tm.d2h_bytes),
               "stages_s": {"upload_exposed": tm.upload_s, "filter": tm.filter_s, "backproject": tm.backproject_s,
                            "download_exposed": tm.download_s},
               "autotune": v.getTuning()}
        # the facade's z split across devices (setActiveCudaDevices): device 0 listed
        # args.split times, each worker reconstructing its run of slices from the
        # detector rows those slices reach; compared with the one-device volume
        if args.split > 1 and rank == 0 and world == 1:
            e2e["split"] = facade_split(v, host_out, args.split, V, W, H, Z, Y, X, units, edge, vs, det, geom)
            log(f"split: {e2e['split']}")
        del v, host_in, host_out
        log(f"e2e: {e2e}")

    c2 = None
    if not args.skip_c2 and args.config == "c3":
        c2 = c2_leg(with_accuracy=rank == 0 and world == 1 and not args.skip_accuracy)
        log(f"c2: {c2}")
    batch = None
    if not args.skip_batch and args.config == "c3":
        batch = batch_c5(store=args.store)
        log(f"batch c5: {batch}")
    grad = None
    if not args.skip_gradient and args.config == "c3":
        grad = gradient_c4()
        log(f"gradient c4: {grad}")

    peaks, peak_kind = measured_peaks()
    clock_mhz = main["clocks"].get("sm_mhz") or peaks.get("sm_max_mhz", 1965.0)
    sm_count = torch.cuda.get_device_properties(local).multi_processor_count
    # fetch roofline: one bilinear sample = 4 texel loads; the L1/shared load path serves one
    # warp-wide (32-lane) load instruction per SM per clock
    peak_gups = sm_count * clock_mhz * 1e6 * 32 / 4 / 1e9
    bp_gups = units / (main["bp_ms"] * 1e-3) / 1e9
    bytes_px_in, bytes_px_out = 2, (2 if store != L.FP32 else 4)
    filt_gbs = V * H * W * (bytes_px_in + bytes_px_out) / (main["filter_ms"] * 1e-3) / 1e9
    roofline = {"bound": "fetch", "kernel": "bp_tma_kernel", "achieved": bp_gups, "peak": peak_gups, "unit": "GUPS",
                "frac": bp_gups / peak_gups,
                "traffic": (BP_DRAM_BYTES_PER_UPDATE[(args.config, slab)] * X * Y * slab * V
                            if (args.config, slab) in BP_DRAM_BYTES_PER_UPDATE and args.store == "fp16" else None),
                "traffic_unit": "DRAM bytes per backprojection launch (one slab)",
                "algorithmic_bytes_per_launch": 8.0 * X * Y * slab * V,
                "peak_basis": f"{sm_count} SMs x {clock_mhz:.0f} MHz (median sampled) x 32 lanes / 4 texel loads"}
    fft_len = W if W & (W - 1) == 0 else 1 << (2 * W - 2).bit_length()   # transform length of the row filter
    filt_kernel = "filter_rf_kernel" if 512 <= fft_len <= 4096 else "filter_kernel"
    roofline_filter = {"bound": "hbm", "kernel": filt_kernel, "achieved": filt_gbs, "peak": peaks["hbm_gbs"],
                       "unit": "GB/s", "frac": filt_gbs / peaks["hbm_gbs"], "peak_kind": peak_kind,
                       "algorithmic_bytes_per_launch": V * H * W * (bytes_px_in + bytes_px_out)}
    launches_per_step = 1 + 2 * len(slabs)   # filter + (view table + backprojection) per slab

    line = {
        "metric": "FDK GUPS (voxels x views / s)", "value": value, "unit": "GUPS", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(args, world),
        "recon_seconds": ms_per_step * 1e-3,
        "stage_ms": {"filter": main["filter_ms"], "backproject": main["bp_ms"]},
        "fp32": fp32,
        "mixed_over_fp32": (value / fp32["value"]) if fp32 else None,
        (other[0] if other else "other_storage"): alt,
        "accuracy_vs_fp64": acc,
        "c2_fp32": c2,
        "batch_c5": batch,
        "gradient_c4": grad,
        "e2e": e2e,
        "roofline": roofline,
        "roofline_filter": roofline_filter,
        "gpu_launches": launches_per_step * args.steps,
        "clocks": main["clocks"],
    }
    if rank == 0 and world == 1 and not args.skip_cpu:
        # CPU leg: the reference's CPU path on a bounded sample (baseline) and the FP64
        # oracle on the central slices (accuracy of this run's volumes)
        sel = np.linspace(0, V - 1, REF_SAMPLE_VIEWS).astype(int)
        imgs_sel = torch.stack([raw[int(i)] for i in sel]).to(torch.int32).cpu().numpy().astype(np.uint16)
        line["cpu_baseline"] = cpu_baseline(cfg, geom, imgs_sel, angles[sel], units)
        line["cpu_baseline"]["c1_full"] = reference_c1_full()
        log(f"cpu baseline: {line['cpu_baseline']}")
        if not args.skip_accuracy:
            t0 = time.perf_counter()
            ref = fp64_slice_set(raw, cfg, geom, det, grid, acc_z)
            acc = {"slices": acc_z, args.store: accuracy(slices_main, ref)}
            if slices_alt is not None:
                acc[other[0]] = accuracy(slices_alt, ref)
            if slices32 is not None:
                acc["fp32"] = accuracy(slices32, ref)
            # per slice, the mixed-precision storage
            acc["per_slice_rel_l2_" + args.store] = [accuracy(slices_main[i:i + 1], ref[:, :, i:i + 1])["rel_l2"]
                                                     for i in range(len(acc_z))]
            acc["oracle_seconds"] = time.perf_counter() - t0
            line["accuracy_vs_fp64"] = acc
            log(f"accuracy: {acc}")
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


# ----------------------------------------------------------- reference arm
def run_reference(args):
    """The reference's own CPU reconstruction code (oracle/_ref: its Ct/CtVolume.cpp lines compiled unchanged;
    the reference application itself needs Qt5 and the OpenCV C++ API, absent here) on all host cores. Each
    step is a measured run on a bounded sample of the same workload: REF_SAMPLE_VIEWS views of the same seeded
    phantom reconstructed into the central slices of the reference's own grid. ms_per_step is that run's wall
    time and value its voxel-views per second; the full workload's time at that rate is a separate field."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    cfg = CONFIGS[args.config]
    geom = geometry(cfg)
    V = geom.n_views
    sel = np.linspace(0, V - 1, REF_SAMPLE_VIEWS).astype(int)
    imgs = cpu_phantom_views(cfg, geom, scan_seed(0), sel)
    angles = geom.angles()[sel]
    runs = []
    for k in range(args.warmup + args.steps):
        r = reference_cpu_step(cfg, geom, imgs, angles)
        if k >= args.warmup:
            runs.append(r)
    secs = float(np.mean([r["seconds"] for r in runs]))
    value = runs[0]["voxel_views"] / secs / 1e9
    conf = workload_config(args, world)
    n = conf["volume"][0]
    units_full = float(n) ** 3 * V
    X, Y, Z = runs[0]["box"]
    sample = (f"{REF_SAMPLE_VIEWS} of {V} views of the seeded phantom (CPU-projected), reference grid box "
              f"{X}x{Y}x{Z} (z {REF_SAMPLE_Z[0]}..{REF_SAMPLE_Z[1]}; voxel = 1 detector pixel, the reference has "
              f"no coarser voxels), {runs[0]['cores']} threads, {cfg['filter']}")
    line = {"metric": "FDK GUPS (voxels x views / s)", "value": value, "unit": "GUPS", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": secs * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "impl": "reference", "config": conf,
            "cpu_baseline": {"value": value, "unit": "GUPS", "cores": runs[0]["cores"], "kind": runs[0]["kind"],
                             "sample": sample},
            "e2e": {"value": value, "unit": "GUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "extrapolated": {"seconds_full_workload_at_measured_rate": units_full / (value * 1e9),
                             "note": f"{n}^3 x {V} voxel-views at this run's rate"},
            "c1_full": reference_c1_full()}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c3", choices=sorted(CONFIGS))
    ap.add_argument("--store", default="fp16", choices=["fp16", "bf16", "fp32"])
    ap.add_argument("--slab", type=int, default=512, help="z slices per backprojection launch (device-resident leg)")
    ap.add_argument("--e2e-slab", type=int, default=0, help="slab height of the end-to-end leg (0: the facade's own)")
    ap.add_argument("--subbox", action="store_true", help="reconstruct the 0.25..0.75 sub-box in x, y and z")
    ap.add_argument("--skip-fp32", action="store_true")
    ap.add_argument("--skip-e2e", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--skip-accuracy", action="store_true")
    ap.add_argument("--skip-batch", action="store_true")
    ap.add_argument("--skip-c2", action="store_true")
    ap.add_argument("--split", type=int, default=2,
                    help="end-to-end leg: also run the facade's z split over device 0 listed this many times (0: off)")
    ap.add_argument("--skip-gradient", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        print("warning: fewer than 3 warm-up steps", file=sys.stderr)
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
