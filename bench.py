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


def cpu_baseline(cfg, imgs_sel: np.ndarray, angles_sel, n_views_total, z_slices=16, nthreads=0):
    """Reference CPU path (oracle restatement) on a bounded sample of the workload.

    Sample: `n_views_sample` views, preprocessed one at a time on one thread (the
    reference's prefetch thread, Ct/CtVolume.cpp:963-965), and backprojected with
    all host threads into the full x-y extent of the box over `z_slices` central
    slices. Scaled to the full workload with the reference's overlap of
    preprocessing and backprojection: T = V * max(t_pre, t_bp * Z / z_slices)."""
    from oracle import oracle as orc
    orc.build()
    n_views_sample, H, W = imgs_sel.shape
    V = n_views_total
    fcd = float(np.float32(cfg["sod"]) / np.float32(cfg["pitch"] * cfg["sod"] / cfg["sdd"]))
    edge, vs = cfg["edge"], cfg["vs"]
    z0 = edge // 2 - z_slices // 2
    g = orc.custom_geom(W, H, fcd, (edge, edge, edge), vs, box=(0, edge, 0, edge, z0, z0 + z_slices))
    t0 = time.perf_counter()
    proj = np.stack([orc.ref_preprocess(im, 1.0, fcd, FILTERS[cfg["filter"]]) for im in imgs_sel])
    t_pre = (time.perf_counter() - t0) / n_views_sample
    t0 = time.perf_counter()
    orc.ref_backproject(proj, np.asarray(angles_sel), np.zeros(n_views_sample), g, nthreads=nthreads)
    t_bp = (time.perf_counter() - t0) / n_views_sample
    per_view = max(t_pre, t_bp * edge / z_slices)
    gups = edge ** 3 / per_view / 1e9
    cores = orc.num_threads() if nthreads <= 0 else nthreads
    return {"value": gups, "unit": "GUPS", "cores": cores, "kind": "port",
            "sample": (f"{n_views_sample} views: preprocessing {t_pre:.3f} s/view on 1 thread, backprojection of "
                       f"{edge}x{edge}x{z_slices} central slices {t_bp:.3f} s/view on {cores} threads; scaled to "
                       f"{edge}^3 x {V} views as V*max(t_pre, t_bp*{edge}/{z_slices}) (prefetch overlap)"),
            "seconds_full_workload_est": per_view * V}


def log(*a):
    print("[bench]", *a, file=sys.stderr, flush=True)


def fp64_reference_slices(raw, cfg, geom, det, grid, z0, z1):
    """FP64 oracle reconstruction of box slices [z0, z1) from only the detector rows they touch."""
    import torch

    from oracle import oracle as orc
    orc.build()
    V, H, W = raw.shape
    vs = grid.voxel_pitch
    zpre = grid.z_size / 2.0 - grid.z_from
    zw = np.array([(z0 - zpre) * vs, (z1 - 1 - zpre) * vs])
    R = float(det.radius)
    D = float(det.fcd)
    U = np.array([D / (D + R), D / (D - R)])
    v = np.outer(zw, U).ravel()
    vpre = H / 2.0
    r0 = max(0, int(math.floor(vpre - v.max())) - 2)
    r1 = min(H, int(math.floor(vpre - v.min())) + 3)
    rows = raw[:, r0:r1, :].to(torch.int32).cpu().numpy().astype(np.uint16)
    g = orc.custom_geom(W, H, float(det.fcd), (grid.x_size, grid.y_size, grid.z_size), vs)
    ref = orc.f64_slices(rows, r0, H, geom.angles(), np.zeros(V), 1.0, FILTERS[cfg["filter"]], g, z0, z1)
    return ref  # (x, y, z1 - z0)


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
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
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
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


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
    scan = synth.make_scan(geom, cfg["n_ell"], seed=1000 + rank, photons=cfg["photons"], n_small=cfg["n_small"])
    raw = scan.images
    angles = geom.angles()
    det, _ = ops.detector(W, H, geom.fcd_px)
    grid = ops.custom_grid(det, (edge, edge, edge), vs)
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
        start.record(stream)
        for k in range(steps):
            device_pass(store_t, filtered, vol, evs[k])
        end.record(stream)
        torch.cuda.synchronize()
        clocks = clk.stop()
        barrier(world)
        total_ms = start.elapsed_time(end)
        f_ms = float(np.mean([e[0].elapsed_time(e[1]) for e in evs]))
        b_ms = float(np.mean([e[1].elapsed_time(e[2]) for e in evs]))
        out = {"total_ms": max_over_ranks(total_ms, world), "filter_ms": f_ms, "bp_ms": b_ms, "clocks": clocks}
        del filtered
        zc = Z // 2
        centre = vol[zc - 1:zc + 1].cpu().numpy()
        del vol
        torch.cuda.empty_cache()
        return out, centre

    log(f"scan ready: {V} views {W}x{H} -> {X}x{Y}x{Z}")
    main, centre = timed(store, args.steps, args.warmup)
    ms_per_step = main["total_ms"] / args.steps
    value = units * world / (ms_per_step * 1e-3) / 1e9
    log(f"{args.store}: {ms_per_step:.1f} ms/step, {value:.1f} GUPS, filter {main['filter_ms']:.1f} ms, "
        f"bp {main['bp_ms']:.1f} ms, clocks {main['clocks']}")

    # plain FP32 path on the same workload (mixed vs plain ratio)
    fp32, centre32 = None, None
    if store != L.FP32 and not args.skip_fp32:
        r32, centre32 = timed(L.FP32, max(2, args.steps // 2), 1)
        ms32 = r32["total_ms"] / max(2, args.steps // 2)
        fp32 = {"value": units * world / (ms32 * 1e-3) / 1e9, "ms_per_step": ms32, "bp_ms": r32["bp_ms"],
                "filter_ms": r32["filter_ms"]}
        log(f"fp32: {fp32}")

    # accuracy of the volumes on the two central slices vs the FP64 oracle
    acc = None
    if rank == 0 and not args.skip_accuracy:
        zc = Z // 2
        ref = fp64_reference_slices(raw, cfg, geom, det, grid, zc - 1, zc + 1)
        acc = {"slices": [zc - 1, zc + 1], args.store: accuracy(centre, ref)}
        if centre32 is not None:
            acc["fp32"] = accuracy(centre32, ref)
        log(f"accuracy: {acc}")

    # end to end through the C ABI facade: pinned host u16 -> pinned host float volume
    e2e = None
    if not args.skip_e2e:
        host_in = torch.empty((V, H, W), dtype=torch.uint16, pin_memory=True)
        host_in.copy_(raw)
        host_out = torch.empty((Z, Y, X), dtype=torch.float32, pin_memory=True)
        v = CtVolume()
        v.setProjectionsPointer(host_in.data_ptr(), L.U16, V, W, H, angles, None, pixel_size=geom.pixel_eff,
                                rotation="ccw", fcd_mm=geom.sod_mm, keep=host_in)
        v.setGrid(edge, edge, edge, vs)
        v.setFrequencyFilterType(cfg["filter"])
        v.setPrecision(args.store)
        v.setSlabHeight(slab)
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
        e2e = {"value": units * world / sec / 1e9, "unit": "GUPS", "seconds": sec,
               "h2d_bytes_per_step": int(V * H * W * 2), "d2h_bytes_per_step": int(X * Y * Z * 4),
               "stages_s": {"upload_exposed": tm.upload_s, "filter": tm.filter_s, "backproject": tm.backproject_s,
                            "download_exposed": tm.download_s}}
        del v, host_in, host_out
        log(f"e2e: {e2e}")

    peaks, peak_kind = measured_peaks()
    clock_mhz = main["clocks"].get("sm_mhz") or peaks.get("sm_max_mhz", 1965.0)
    sm_count = torch.cuda.get_device_properties(local).multi_processor_count
    # fetch roofline: one bilinear sample = 4 texel loads; the L1/shared load path serves one
    # warp-wide (32-lane) load instruction per SM per clock
    peak_gups = sm_count * clock_mhz * 1e6 * 32 / 4 / 1e9
    bp_gups = units / (main["bp_ms"] * 1e-3) / 1e9
    bytes_px_in, bytes_px_out = 2, (2 if store != L.FP32 else 4)
    filt_gbs = V * H * W * (bytes_px_in + bytes_px_out) / (main["filter_ms"] * 1e-3) / 1e9
    roofline = {"bound": "fetch", "kernel": "bp_kernel", "achieved": bp_gups, "peak": peak_gups, "unit": "GUPS",
                "frac": bp_gups / peak_gups, "traffic": None,
                "peak_basis": f"{sm_count} SMs x {clock_mhz:.0f} MHz (median sampled) x 32 lanes / 4 texel loads"}
    roofline_filter = {"bound": "hbm", "kernel": "filter_kernel", "achieved": filt_gbs, "peak": peaks["hbm_gbs"],
                       "unit": "GB/s", "frac": filt_gbs / peaks["hbm_gbs"], "peak_kind": peak_kind,
                       "algorithmic_bytes_per_launch": V * H * W * (bytes_px_in + bytes_px_out)}
    launches_per_step = 1 + 2 * len(slabs)   # filter + (view table + backprojection) per slab

    line = {
        "metric": "FDK GUPS (voxels x views / s)", "value": value, "unit": "GUPS", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"{args.config}: {V} views x {W}x{H} u16 -> {X}x{Y}x{Z} f32 (voxel {vs} px), "
                               f"{cfg['filter']}, {args.store} storage", "storage": args.store,
                   "views": V, "detector": [W, H], "volume": [X, Y, Z], "voxel_pitch_px": vs,
                   "slab": slab, "l2": "inputs (12 GB) larger than L2; no flush", "parallelism": f"replicas{world}"},
        "recon_seconds": ms_per_step * 1e-3,
        "stage_ms": {"filter": main["filter_ms"], "backproject": main["bp_ms"]},
        "fp32": fp32,
        "mixed_over_fp32": (value / fp32["value"]) if fp32 else None,
        "accuracy_vs_fp64": acc,
        "e2e": e2e,
        "roofline": roofline,
        "roofline_filter": roofline_filter,
        "gpu_launches": launches_per_step * args.steps,
        "clocks": main["clocks"],
    }
    if rank == 0 and world == 1 and not args.skip_cpu:
        sel = np.linspace(0, V - 1, 8).astype(int)
        imgs_sel = torch.stack([raw[int(i)] for i in sel]).to(torch.int32).cpu().numpy().astype(np.uint16)
        line["cpu_baseline"] = cpu_baseline(cfg, imgs_sel, angles[sel], V)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


# ----------------------------------------------------------- reference arm
def run_reference(args):
    """The reference's CPU reconstruction path (oracle restatement; the reference
    itself needs Qt5 + OpenCV C++ and is not buildable here) on the host cores,
    each step a bounded sample of the same workload."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    cfg = CONFIGS[args.config]
    geom = geometry(cfg)
    V, W, H = geom.n_views, geom.width, geom.height
    # the same phantom family, projected on the CPU for the sampled views only
    from oracle import phantom
    from ct_b200 import synth
    rng = np.random.default_rng(1000)
    r_mm, hz_mm = synth.fov(geom)
    ell = synth.random_ellipsoids(rng, cfg["n_ell"], r_mm, hz_mm, n_small=cfg["n_small"])
    angles = geom.angles()
    n_s = 8
    sel = np.linspace(0, V - 1, n_s).astype(int)
    p = phantom.project(ell, angles[sel], None, W, H, geom.pixel_eff, geom.sod_mm)
    imgs = synth.intensities_from_line_integrals(p)
    vals = []
    for k in range(args.warmup + args.steps):
        r = cpu_baseline(cfg, imgs, angles[sel], V)
        if k >= args.warmup:
            vals.append(r)
    value = float(np.mean([r["value"] for r in vals]))
    last = vals[-1]
    line = {"metric": "FDK GUPS (voxels x views / s)", "value": value, "unit": "GUPS", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": last["seconds_full_workload_est"] * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": f"{args.config}: {V} views x {W}x{H} u16 -> {cfg['edge']}^3 f32, "
                                   f"{cfg['filter']}, reference CPU path"},
            "cpu_baseline": {"value": value, "unit": "GUPS", "cores": last["cores"], "kind": "port",
                             "sample": last["sample"]},
            "e2e": {"value": value, "unit": "GUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c3", choices=sorted(CONFIGS))
    ap.add_argument("--store", default="fp16", choices=["fp16", "bf16", "fp32"])
    ap.add_argument("--slab", type=int, default=128)
    ap.add_argument("--skip-fp32", action="store_true")
    ap.add_argument("--skip-e2e", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--skip-accuracy", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        print("warning: fewer than 3 warm-up steps", file=sys.stderr)
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
