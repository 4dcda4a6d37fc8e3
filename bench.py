#!/usr/bin/env python
"""Benchmark of the 2D-Gaussian-surfel training step on B200.

One step = forward over every view (projection, binning, tile raster), fused
L1+SSIM loss, backward raster, projection backward and Adam over all surfel
parameters, on a resident seeded synthetic scene (default: 1,000,000 surfels
and 8 ring views from 640x480 to 1920x1080, 9.0 Mpx). The headline `value` is
the batched mixed-precision form ("chosen"); the plain FP32 one-view-at-a-time
form is timed on the same inputs in the same run.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs N independent replicas (one process per GPU under torchrun; the
path has no exchange step at this scope), timed as the max over ranks.
`--impl reference` times the reference algorithm's CPU implementation (the
C++ restatement of the reference's CPU renderer; the reference itself is Rust
+ WGSL on wgpu/Vulkan and cannot be built or run on this machine).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "fwd+bwd+Adam steps/s, 1M surfels 1080p: chosen vs plain form; HBM roofline frac"
# dram__bytes_read.sum + dram__bytes_write.sum per launch of the dominant kernel,
# from one ncu capture of the same workload
# (python profile_step.py --workload ring8_1m --shapes 64,4,32,8, the
# autotuned shapes).
TRAFFIC = {("ring8_1m", "raster_bwd"): 1_606_542_848}
# Launch shapes (fwd batch, fwd pixels/thread, bwd batch, bwd pixels/thread)
# tried for the plain form at 16-pixel tiles before it is timed.
PLAIN_SHAPES = [(128, 2, 128, 2), (128, 2, 64, 4), (128, 1, 128, 2), (64, 4, 64, 8)]
FALLBACK_HBM_GBS = 6650.0
L2_BYTES = 126 * 2 ** 20  # B200 L2


def working_set_bytes(n: int, nv: int, P: int) -> int:
    """Bytes one training step touches, roughly: parameters, optimizer state
    and SH copies (~1.2 KB per surfel), records and item buffers (~96 B per
    surfel and view), per-pixel buffers (~100 B per pixel)."""
    return 1200 * n + 96 * n * nv + 100 * P


def workload_config(name: str, wl) -> dict:
    """The workload description both arms print as `config`."""
    n, nv, P = wl.surfels.n, len(wl.cameras), wl.pixels
    ws_bytes = working_set_bytes(n, nv, P)
    return {"workload": name, "surfels": n, "views": nv,
            "resolutions": [f"{c.width}x{c.height}" for c in wl.cameras], "pixels_per_step": P,
            "l2": (f"inputs larger than L2 (about {ws_bytes / 1e9:.1f} GB touched per step)" if ws_bytes >= 2 * L2_BYTES
                   else f"L2 flushed before every timed step (256 MB written; about {ws_bytes / 1e6:.0f} MB touched "
                        f"per step)")}
# FP32 arithmetic of the raster kernels (an FMA counts 2), counted from
# splattar_b200/csrc/gs_raster.cuh, as (per hit evaluation, per contributing
# pair, MUFU ops per hit evaluation, MUFU ops per contributing pair):
#   hit test eval_hit / eval_hit2: det 1 FMA, u.det and v.det 2 FMA, u and v
#     2 MUL, t 1 MUL, u^2+v^2 1 MUL + 1 FMA, q_ray 1 MUL, dy 1 ADD, q_screen
#     1 FMA, exp 1 MUL + 1 EX2, 1/det 1 RCP (17 flops, 2 MUFU), alpha 1 MUL,
#     plus the column partial sums (1 FMA, 1 ADD, 3 MUL = 6 flops per entry
#     and thread, over 4 forward / 8 backward pixels per thread);
#   forward composite: w 1 MUL, colour 3 FMA, alpha sum 1 ADD, T 1 ADD + 1 MUL;
#   backward per contributor: 1 - alpha 1 ADD + 1 RCP, T_before 1 MUL, w 1 MUL,
#     dL/dcolour.colour 1 MUL + 2 FMA, dL/dalpha 1 MUL + 1 FMA, suffix 1 FMA,
#     colour gradient 3 FMA, dL/dghat, opacity sum, K 3 MUL/ADD, ray-branch
#     record moments 1 + 2 + 1 MUL and 6 FMA (38 flops, 1 MUFU).
RASTER_OPS = {"raster_fwd": (20, 10, 2, 0), "raster_bwd": (19, 38, 2, 1)}
# Nominal B200 rates per SM per clock: 128 FP32 lanes (FMA = 2 flops), 16 MUFU.
SM_COUNT, FP32_PER_SM_CLK, MUFU_PER_SM_CLK = 148, 256, 16
# Issue-slot activity of the raster kernels measured by ncu on ring2_200k
# (profiles/raster_fwd_bwd_ring2_200k.md).
ISSUE_ACTIVE_NCU = {"raster_fwd": 0.864, "raster_bwd": 0.802}


def parse(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--workload", default="ring8_1m")
    p.add_argument("--precision", default="f16", choices=["f32", "f16", "bf16"])
    p.add_argument("--no-plain", action="store_true")
    p.add_argument("--no-full-lists", action="store_true",
                   help="skip timing the chosen form without the occlusion cut")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--cpu-seconds", type=float, default=20.0, help="target CPU-baseline sample time")
    p.add_argument("--densify-every", type=int, default=0,
                   help="densify/prune cycle: clone/prune every K timed steps (grad 2e-4, opacity 0.005)")
    p.add_argument("--deterministic", action="store_true", help="ordered gradient reduction (densify cycle)")
    p.add_argument("--stored-state", action="store_true",
                   help="stored-state backward: the forward records per-pixel contributor masks")
    p.add_argument("--entries-budget", type=float, default=96.0, help="tile-entry capacity per item")
    p.add_argument("--tile", default="auto", choices=["auto", "8", "16", "32"],
                   help="tile edge of the chosen form: autotuned over 8/16/32, or fixed (the plain form uses 16)")
    p.add_argument("--capacity-factor", type=float, default=1.25, help="densify cycle: capacity / initial surfels")
    p.add_argument("--entries-per-item", type=float, default=12.0, help="densify cycle: tile-entry budget per item")
    return p.parse_args(argv)


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def max_over_ranks(ms: float, ws: int, device: str = "cuda") -> float:
    """The slowest rank's time: every rank calls this at the same point."""
    if ws <= 1:
        return ms
    import torch
    import torch.distributed as dist
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_steps_per_s(ms_per_step: float, ws: int) -> float:
    """Whole-job throughput of ws replicas that each ran one step per ms_per_step
    (ms_per_step is already the max over ranks)."""
    return 1000.0 / ms_per_step * ws


# ----------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device, self.proc, self.lines = device, None, []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.device)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if f[5 + k].lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_hbm_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


# ------------------------------------------------------ CPU (oracle) timing
def cpu_step_estimate(wl, seconds_target: float, threads: int = 0, view_ids=None, stride: int = 0):
    """Seconds per full training step of the C++ restatement of the
    reference's CPU renderer (crates/gs-cpu-ref) on this workload, measured on
    a bounded sample: every view's projection, tile lists, L1+SSIM and
    parameter chain in full, the per-pixel forward and backward walks on every
    `stride`-th tile only, scaled by `stride`; Adam over all parameters once.
    stride 0 chooses: every 64th tile, or every tile (no sampling, nothing
    extrapolated) when the whole step is estimated at no more than half of
    `seconds_target`."""
    if stride == 0:
        est, _, detail = cpu_step_estimate(wl, seconds_target, threads, view_ids, 64)
        if seconds_target <= 0 or est > 0.5 * seconds_target:
            return est, 64, detail
        stride = 1
    import oracle
    s = wl.surfels
    scene = oracle.Scene(s.positions.astype(np.float64), s.scales.astype(np.float64), s.quats.astype(np.float64),
                         s.opacities.astype(np.float64), s.sh48().astype(np.float64), s.sh_degree)
    views = range(len(wl.cameras)) if view_ids is None else view_ids
    total, detail = 0.0, []
    adam = 0.0
    for v in views:
        c = wl.cameras[v]
        cam = oracle.Camera(np.array(c.center), np.array(c.quat), c.focal, c.width, c.height)
        tgt = np.zeros((c.width * c.height, 4))
        t = oracle.cpu_step_timed(scene, cam, tgt, tile_stride=stride, threads=threads)
        per_view = t[0] + (t[1] + t[3]) * stride + t[2] + t[4]
        adam = t[5]
        total += per_view
        detail.append([round(x, 4) for x in t])
    scale = len(wl.cameras) / len(list(views))
    step = total * scale + adam
    return step, stride, detail


# ---------------------------------------------------------------- our arm
def algorithmic_bytes(stage: str, n: int, views, E: int, P: int) -> float:
    """Algorithmic HBM bytes of a stage per step (FP32 plain form)."""
    nv = len(views)
    if stage == "raster_fwd":
        return E * (4 + 72) + 40 * P
    if stage == "raster_bwd":
        return E * (4 + 68) + 40 * P + 64 * n * nv
    if stage == "project":
        return 332.0 * n * nv
    if stage == "project_bwd_adam":
        return 600.0 * n * nv + 58 * 32.0 * n
    if stage == "l1_ssim":
        return 36.0 * P
    if stage in ("tile_sort",):
        return 2 * 2 * 8.0 * E
    if stage == "expand":
        return 8.0 * E
    if stage == "ranges":
        return 4.0 * E
    if stage == "depth_sort_scan":
        return 4 * 2 * 8.0 * n * nv
    return 0.0


def raster_compute(stage: str, work: dict, kernel_ms: float, sm_mhz) -> dict:
    """Compute side of a raster kernel's roofline: FP32 flops and MUFU ops
    from the device-counted hit evaluations and contributing pairs, over the
    kernel's measured time, against the nominal rates at the sampled SM
    clock."""
    f_eval, f_contrib, m_eval, m_contrib = RASTER_OPS[stage]
    evals = work["fwd_evals"] if stage == "raster_fwd" else work["bwd_evals"]
    flops = f_eval * evals + f_contrib * work["contrib_pairs"]
    mufu = m_eval * evals + m_contrib * work["contrib_pairs"]
    hz = (sm_mhz or 1965.0) * 1e6
    peak_tf = SM_COUNT * FP32_PER_SM_CLK * hz / 1e12
    peak_mufu = SM_COUNT * MUFU_PER_SM_CLK * hz / 1e12
    sec = kernel_ms * 1e-3
    return {"bound": "issue", "hit_evaluations": evals, "contributing_pairs": work["contrib_pairs"],
            "fp32_flops": flops, "achieved_tflops": round(flops / sec / 1e12, 3),
            "peak_tflops": round(peak_tf, 2), "frac": round(flops / sec / 1e12 / peak_tf, 4),
            "mufu_ops": mufu, "mufu_frac": round(mufu / sec / 1e12 / peak_mufu, 4),
            "issue_active_ncu": ISSUE_ACTIVE_NCU.get(stage),
            "peak_source": f"nominal B200: {SM_COUNT} SMs x {FP32_PER_SM_CLK} FP32 flops and {MUFU_PER_SM_CLK} MUFU "
                           f"ops per clock at the sampled {hz / 1e6:.0f} MHz",
            "ops_per_unit": {"flops_per_hit": f_eval, "flops_per_contributor": f_contrib, "mufu_per_hit": m_eval,
                             "mufu_per_contributor": m_contrib}}


def literal_baselines() -> dict:
    """The reference CPU renderer's own O(P·N) per-pixel walk
    (crates/gs-cpu-ref/src/forward.rs:207-246: every sorted surfel tested
    against every pixel's tile), single-threaded, at the 16,384-surfel 256x256
    scene and the 1,024-surfel 128x128 scene, and the binned step at the
    16,384-surfel scene in full (no sampling), all host threads."""
    import oracle
    from splattar_b200.synthetic import look_at, make_surfels, workload
    f64 = lambda a: np.asarray(a, np.float64)  # noqa: E731
    out = {}
    wl0 = workload("small_1view_256")
    s0, c0 = wl0.surfels, wl0.cameras[0]
    sc0 = oracle.Scene(f64(s0.positions), f64(s0.scales), f64(s0.quats), f64(s0.opacities), f64(s0.sh48()), 0)
    cam0 = oracle.Camera(f64(c0.center), f64(c0.quat), float(c0.focal), c0.width, c0.height)
    t = time.time()
    oracle.render(sc0, cam0, literal=True)
    out["literal_forward_16k_256px_s"] = round(time.time() - t, 3)
    s1 = make_surfels(1024, 0, False, 0, 0.3)
    c1 = look_at((0, 0, -3), (0, 0, 0), 128, 128, focal=128.0)
    sc1 = oracle.Scene(f64(s1.positions), f64(s1.scales), f64(s1.quats), f64(s1.opacities), f64(s1.sh48()), 0)
    cam1 = oracle.Camera(f64(c1.center), f64(c1.quat), float(c1.focal), 128, 128)
    t = time.time()
    oracle.render(sc1, cam1, literal=True)
    out["literal_forward_1k_128px_s"] = round(time.time() - t, 3)
    tgt = np.zeros((c0.width * c0.height, 4))
    t = time.time()
    oracle.cpu_step_timed(sc0, cam0, tgt, tile_stride=1, threads=oracle.max_threads())
    out["binned_step_16k_256px_s"] = round(time.time() - t, 3)
    out["threads"] = {"literal": 1, "binned": oracle.max_threads()}
    return out


def launches_per_step(n_tiles: int, nv: int, form: str) -> int:
    """Kernel launches of one step: projection; depth sort (4 radix passes of
    upsweep + 3-kernel histogram scan + downsweep); entry scan (3) and entry
    guard; expansion; tile sort (same passes over the tile-id bits); ranges;
    forward raster; L1+SSIM (2); backward raster; projection backward + Adam
    (chosen form, which also orders its tiles heaviest first before each
    raster pass: two more launches, and runs the occlusion cut's completion
    pass: gate, flagged counts, entry scan (3), guard, range reset,
    expansion, tile sort, range fix and forward raster, each finding zero work
    when no tile needs it)."""
    bits = max(1, math.ceil(math.log2(max(n_tiles, 2))))
    tile_passes = math.ceil(bits / 8)
    per_pass = 5
    fwd = 1 + 4 * per_pass + 3 + 1 + 1 + tile_passes * per_pass + 1 + 1
    if form == "chosen":
        completion = 1 + 1 + 3 + 1 + 1 + 1 + tile_passes * per_pass + 1 + 1
        return fwd + 1 + 2 + 1 + 1 + 1 + completion
    return nv * (fwd + 2 + 1 + 1) + 5


def run_ours(args, ws, rank, local):
    import torch
    torch.cuda.set_device(local)
    from splattar_b200 import Rasterizer, StepSettings
    from splattar_b200.rasterizer import AdamSettings
    from splattar_b200.synthetic import workload

    wl = workload(args.workload)
    cams = wl.cameras
    n, nv, P = wl.surfels.n, len(cams), wl.pixels
    max_entries = int(min(4.2e9, args.entries_budget * n * nv))
    free0, _ = torch.cuda.mem_get_info()
    rast = Rasterizer(n, 0, 0, max_entries, max_views=nv, max_pixels=P, precision=args.precision, color_only=True,
                      stored_state=args.stored_state)
    free1, _ = torch.cuda.mem_get_info()
    # Target images: the seed-1 scene rendered through the same cameras.
    rast.upload_scene(wl.target_surfels.scene_input())
    rast.forward(cams, n)
    rast.check()
    target = rast.read("out_color", 4 * P)
    rast.write("target", target)
    rast.upload_scene(wl.surfels.scene_input())
    rast.optimizer_init(n)
    if args.tile == "auto":
        tuned = rast.autotune_tiles(cams, n)
    else:
        rast.tile = int(args.tile)
        tuned = dict(tile=int(args.tile), **rast.autotune(cams, n))
    tile = rast.tile
    adam = AdamSettings(eps=1e-15)
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream
    chosen = StepSettings(0.8, 0.2, adam, "chosen")
    plain = StepSettings(0.8, 0.2, adam, "plain")

    # A working set smaller than L2 is timed step by step with 256 MB written
    # between the steps, outside the timed regions.
    flush = working_set_bytes(n, nv, P) < 2 * L2_BYTES
    scratch = torch.empty(256 << 20, dtype=torch.uint8, device="cuda") if flush else None

    def timed(step_cfg, steps, warmup, h=None):
        h = rast if h is None else h
        for _ in range(warmup):
            h.train_step(cams, n, step_cfg, sp)
        h.check(sp)
        if ws > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        if flush:
            evs = []
            for _ in range(steps):
                scratch.fill_(1)
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(stream)
                h.train_step(cams, n, step_cfg, sp)
                b.record(stream)
                evs.append((a, b))
            torch.cuda.synchronize()
            h.check(sp)
            return max_over_ranks(sum(a.elapsed_time(b) for a, b in evs) / steps, ws)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            h.train_step(cams, n, step_cfg, sp)
        e1.record(stream)
        torch.cuda.synchronize()
        h.check(sp)
        return max_over_ranks(e0.elapsed_time(e1) / steps, ws)

    clocks = ClockSampler(local)
    clocks.start()
    ms_chosen = timed(chosen, args.steps, args.warmup)
    clk = clocks.stop()
    E = rast.entry_count()
    redone = None if args.stored_state else int(rast.read("incomplete_tiles", 1)[0])
    ms_plain = None
    plain_shapes = None
    if not args.no_plain:
        # The plain form at the reference's 16-pixel tiles, with the launch
        # shapes that suit it best (its kernels are the non-persistent,
        # per-view variants, whose best shapes differ from the chosen form's).
        rast.tile = 16
        best = None
        for shp in PLAIN_SHAPES:
            rast.set_launch_shapes(*shp)
            ms = timed(plain, 2, 1)
            if best is None or ms < best[0]:
                best = (ms, shp)
        plain_shapes = best[1]
        rast.set_launch_shapes(*plain_shapes)
        ms_plain = timed(plain, max(2, args.steps // 2), args.warmup)
        rast.tile = tile
        rast.set_launch_shapes(tuned["fwd_batch"], tuned["fwd_pixels_per_thread"], tuned["bwd_batch"],
                               tuned["bwd_pixels_per_thread"])

    # End to end through the public API: every step's target comes from pinned
    # host memory and its loss goes back to pinned host memory. The target of
    # step k+1 is copied host-to-device on a side stream into one of two device
    # staging buffers while step k runs, then moved into the handle's target
    # buffer with a device-to-device write_async at the start of step k+1 (how
    # a trainer prefetches its next batch). All copies lie inside the timed
    # region.
    tgt_host = torch.from_numpy(target.view(np.float32)).pin_memory()
    loss_host = torch.zeros(2 * nv, dtype=torch.float64).pin_memory()
    tgt_bytes = tgt_host.numel() * 4
    staging = [torch.empty_like(tgt_host, device="cuda") for _ in range(2)]
    feed_stream = torch.cuda.Stream()
    copied = [torch.cuda.Event() for _ in range(2)]
    consumed = [torch.cuda.Event() for _ in range(2)]

    def feed(k):
        b = k % 2
        feed_stream.wait_event(consumed[b])  # step k-2 has moved this buffer into the handle
        with torch.cuda.stream(feed_stream):
            staging[b].copy_(tgt_host, non_blocking=True)
        copied[b].record(feed_stream)

    def e2e_step(k):
        b = k % 2
        stream.wait_event(copied[b])
        rast.write_async("target", staging[b].data_ptr(), tgt_bytes, 0, sp)
        consumed[b].record(stream)
        rast.train_step(cams, n, chosen, sp)
        rast.read_async("loss", loss_host.data_ptr(), loss_host.numel() * 8, 0, sp)

    def e2e_run(steps, start_event=None, evs=None):
        if start_event is not None:
            feed_stream.wait_event(start_event)
        feed(0)
        for k in range(steps):
            if k + 1 < steps:
                feed(k + 1)
            if evs is not None:  # small working set: flush L2, then time the step alone
                scratch.fill_(1)
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(stream)
                e2e_step(k)
                b.record(stream)
                evs.append((a, b))
            else:
                e2e_step(k)

    e2e_run(args.warmup)
    torch.cuda.synchronize()
    if ws > 1:
        torch.distributed.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    evs = [] if flush else None
    e2e_run(args.steps, e0, evs)
    e1.record(stream)
    torch.cuda.synchronize()
    ms_e2e = max_over_ranks((sum(a.elapsed_time(b) for a, b in evs) if flush else e0.elapsed_time(e1)) / args.steps,
                            ws)
    loss_vals = loss_host.numpy().copy()

    # Stage timing (CUDA events between stages on the launch stream), then
    # the raster kernels' work on the last of those steps (counted on the
    # device, outside every timed region).
    prof = [rast.train_step_profiled(cams, n, chosen, sp) for _ in range(3)]
    stages = {k: statistics.median(p[k] for p in prof) for k in prof[0]}
    work = rast.raster_work(sp)
    n_tiles = sum(((c.width + tile - 1) // tile) * ((c.height + tile - 1) // tile) for c in cams)
    rast.check(sp)
    handle_bytes = int(free0 - free1)
    rast.close()

    # The chosen form without the occlusion cut (full tile lists every step):
    # its speed does not depend on the views repeating from step to step.
    ms_full = None
    if not args.no_full_lists and not args.stored_state:
        rf = Rasterizer(n, 0, 0, max_entries, max_views=nv, max_pixels=P, precision=args.precision, color_only=True,
                        full_lists=True)
        rf.upload_scene(wl.surfels.scene_input())
        rf.write("target", target)
        rf.optimizer_init(n)
        rf.tile = tile
        rf.set_launch_shapes(tuned["fwd_batch"], tuned["fwd_pixels_per_thread"], tuned["bwd_batch"],
                             tuned["bwd_pixels_per_thread"])
        ms_full = timed(chosen, args.steps, args.warmup, rf)
        rf.close()
    result = dict(tuned=tuned, wl=wl, n=n, nv=nv, P=P, E=E, redone=redone, ms_chosen=ms_chosen, ms_plain=ms_plain,
                  ms_e2e=ms_e2e, ms_full=ms_full, clk=clk, plain_shapes=plain_shapes, handle_bytes=handle_bytes,
                  stages=stages, work=work, n_tiles=n_tiles, loss=loss_vals, h2d=tgt_host.numel() * 4,
                  d2h=loss_host.numel() * 8)
    return result


def run_densify_cycle(args, ws, rank, local):
    """Training with the densify/prune cycle: `steps` chosen-form steps, a
    densify/prune compaction after every `densify_every` of them (clone where
    the mean |dL/dpos| exceeds 2e-4, prune activated opacity below 0.005),
    all inside the timed region (the compaction synchronises with the host to
    learn the new surfel count)."""
    import torch
    torch.cuda.set_device(local)
    from splattar_b200 import Rasterizer, StepSettings
    from splattar_b200.rasterizer import AdamSettings
    from splattar_b200.synthetic import workload

    wl = workload(args.workload)
    cams = wl.cameras
    n, nv, P = wl.surfels.n, len(cams), wl.pixels
    cap = int(n * args.capacity_factor)
    max_entries = int(min(4.2e9, args.entries_per_item * cap * nv))
    free0, total = torch.cuda.mem_get_info()
    rast = Rasterizer(cap, 0, 0, max_entries, max_views=nv, max_pixels=P, precision=args.precision, color_only=True,
                      deterministic=args.deterministic, tight=True)
    free1, _ = torch.cuda.mem_get_info()
    rast.upload_scene(wl.target_surfels.scene_input())
    rast.forward(cams, n)
    rast.check()
    rast.write("target", rast.read("out_color", 4 * P))
    rast.upload_scene(wl.surfels.scene_input())
    rast.optimizer_init(n)
    tuned = rast.autotune(cams, n)  # raster launch shapes for this workload (tile 16)
    step = StepSettings(0.8, 0.2, AdamSettings(eps=1e-15), "chosen")
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream
    for _ in range(args.warmup):
        rast.train_step(cams, n, step, sp)
    rast.check(sp)
    counts = [n]
    entries = []
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for k in range(args.steps):
        rast.train_step(cams, n, step, sp)
        if args.densify_every and (k + 1) % args.densify_every == 0:
            entries.append(rast.entry_count())
            n = rast.densify_prune(2e-4, 0.005, n, sp)
            counts.append(n)
    e1.record(stream)
    torch.cuda.synchronize()
    rast.check(sp)
    ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, ws)
    rast.close()
    if rank != 0:
        return
    print(json.dumps({
        "metric": METRIC, "value": round(aggregate_steps_per_s(ms, ws), 4), "unit": "steps/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f32" if args.precision == "f32" else f"f32 compute, {args.precision} storage", "data": "synthetic",
        "config": {"workload": args.workload, "views": nv, "pixels_per_step": P, "capacity": cap, "autotuned": tuned,
                   "densify_every": args.densify_every, "mode": "deterministic" if args.deterministic else "atomic",
                   "surfels_after_each_densify": counts, "tile_entries_before_each_densify": entries,
                   "device_bytes_of_handle": int(free0 - free1), "device_bytes_total": int(total),
                   "note": "densify/prune cycle inside the timed region"},
    }))


def main():
    args = parse()
    ws, rank, local = dist_env()
    if args.impl == "reference":
        return main_reference(args, ws, rank)
    if ws > 1:
        import torch
        import torch.distributed as dist
        import datetime
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    if args.densify_every or args.deterministic:
        run_densify_cycle(args, ws, rank, local)
        if ws > 1:
            import torch.distributed as dist
            dist.barrier()
            dist.destroy_process_group()
        return
    r = run_ours(args, ws, rank, local)
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    n, nv, P, E = r["n"], r["nv"], r["P"], r["E"]
    steps_s = 1000.0 / r["ms_chosen"]
    job_steps_s = aggregate_steps_per_s(r["ms_chosen"], ws)
    peak, peak_kind = measured_hbm_peak()
    stages = r["stages"]
    dom = max(stages, key=stages.get)
    alg = algorithmic_bytes(dom, n, r["wl"].cameras, E, P)
    achieved = alg / (stages[dom] * 1e-3) / 1e9 if stages[dom] > 0 else 0.0
    sm_mhz = r["clk"].get("sm_mhz")
    compute = {k: raster_compute(k, r["work"], stages[k], sm_mhz) for k in ("raster_fwd", "raster_bwd")}
    line = {
        "metric": METRIC,
        "value": round(job_steps_s, 4),
        "unit": "steps/s",
        "n_gpus": ws,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(r["ms_chosen"], 4),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32" if args.precision == "f32" else f"f32 compute, {args.precision} storage",
        "storage": None if args.precision == "f32" else
        f"{args.precision}: SH coefficients and the projected record's normal and depth; geometry, colour, opacity, "
        "compositing, gradients and Adam moments f32",
        "data": "synthetic",
        "config": workload_config(args.workload, r["wl"]),
        "setup": {
            "tile_entries_per_step": E,
            "occlusion_cut": None if r["redone"] is None else {
                "tiles_rendered_again_in_last_step": r["redone"],
                "what": "each tile binned down to the depth its pixels needed in the previous step plus a margin; "
                        "tiles whose truncated list ran out re-binned and re-rendered in full within the step; "
                        "images and gradients equal to full lists"},
            "form": "chosen: views batched per pass, persistent raster kernels, projection backward fused with Adam, "
                    f"{args.precision} storage of SH and projected colour/normal, CUDA-graph replay, "
                    f"{r['tuned']['tile']}-pixel tiles",
            "loss": "0.8*L1 + 0.2*(1-SSIM), 11x11 Gaussian sigma 1.5",
            "adam": "lr pos 1.6e-4 scales 5e-3 quat 1e-3 opacity 5e-2 sh 2.5e-3, betas 0.9/0.999, eps 1e-15",
            "parallelism": f"replicas x{ws}" if ws > 1 else "single GPU",
            "autotuned": r["tuned"],
            "backward": "stored-state (forward contributor masks)" if args.stored_state else "recompute",
            "device_bytes_of_handle": r["handle_bytes"],
        },
        "mpix_per_s": round(steps_s * P / 1e6 * ws, 2),
        "plain": None if r["ms_plain"] is None else {
            "steps_per_s": round(aggregate_steps_per_s(r["ms_plain"], ws), 4), "ms_per_step": round(r["ms_plain"], 4),
            "form": "views one at a time, FP32 records and SH, separate projection backward and Adam kernels, "
                    "16-pixel tiles",
            "launch_shapes": r["plain_shapes"]},
        "chosen_over_plain": None if r["ms_plain"] is None else round(r["ms_plain"] / r["ms_chosen"], 3),
        "full_lists": None if r["ms_full"] is None else {
            "steps_per_s": round(aggregate_steps_per_s(r["ms_full"], ws), 4), "ms_per_step": round(r["ms_full"], 4),
            "over_plain": None if r["ms_plain"] is None else round(r["ms_plain"] / r["ms_full"], 3),
            "form": "the chosen form with GS_FLAG_FULL_LISTS: no occlusion cut, full tile lists every step (its speed "
                    "does not depend on the views repeating between steps)"},
        "e2e": {"value": round(aggregate_steps_per_s(r["ms_e2e"], ws), 4), "unit": "steps/s", "h2d_bytes_per_step": r["h2d"],
                "d2h_bytes_per_step": r["d2h"], "ms_per_step": round(r["ms_e2e"], 4),
                "path": "per step: pinned host target -> device staging (side stream, prefetched one step ahead) -> "
                        "Rasterizer.write_async(target) + gs_train_step + read_async(loss -> pinned host)"},
        "gpu_launches": launches_per_step(r["n_tiles"], nv, "chosen") * args.steps,
        "roofline": {"kernel": dom, "bound": compute[dom]["bound"] if dom in compute else "hbm",
                     "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": TRAFFIC.get((args.workload, dom)),
                     "traffic_unit": "DRAM bytes read + written per launch (ncu capture of this workload)",
                     "peak_source": f"{peak_kind} MEASURED_PEAKS.json hbm_gbs" if peak_kind == "measured"
                     else "fallback 6.65 TB/s",
                     "algorithmic_bytes": alg, "kernel_ms": round(stages[dom], 4),
                     "compute": compute.get(dom)},
        "raster_compute": compute,
        "raster_work": r["work"],
        "stages_ms": {k: round(v, 4) for k, v in stages.items()},
        "clocks": r["clk"],
        "loss": [float(x) for x in r["loss"][:4]],
    }
    if not args.no_cpu_baseline:
        import oracle
        cores = oracle.max_threads()
        t0 = time.time()
        step_s, stride, detail = cpu_step_estimate(r["wl"], args.cpu_seconds, threads=cores)
        spent = time.time() - t0
        line["cpu_baseline"] = {"value": round(1.0 / step_s, 6), "unit": "steps/s", "cores": cores, "kind": "port",
                                "sample": (f"all {nv} views; projection, tile lists, L1+SSIM, parameter chain and Adam "
                                           f"in full; per-pixel forward/backward on every {stride}th tile, scaled by "
                                           f"{stride}") if stride > 1 else
                                          f"the whole step, all {nv} views, every tile (not sampled)",
                                "extrapolated": stride > 1, "sample_fraction_of_pixel_walks": round(1.0 / stride, 5),
                                "seconds_spent": round(spent, 2), "seconds_per_step": round(step_s, 3),
                                "literal": literal_baselines()}
    print(json.dumps(line))


def main_reference(args, ws, rank):
    """Reference arm: the reference's CPU algorithm (C++ restatement of
    crates/gs-cpu-ref) on this workload, all host threads, rank 0 only."""
    if rank != 0:
        return
    import oracle
    from splattar_b200.synthetic import workload
    wl = workload(args.workload)
    cores = oracle.max_threads()
    nv = len(wl.cameras)
    times = []
    t0 = time.time()
    # every tile (no sampling) when a whole step takes at most 5 s, else every 64th tile
    est, _, _ = cpu_step_estimate(wl, 0, threads=cores, view_ids=[0], stride=64)
    stride = 1 if est <= 5.0 else 64
    samples = []  # wall-clock seconds of each timed sample
    for k in range(args.warmup + args.steps):
        v = k % nv
        ts = time.time()
        step_s, stride, _ = cpu_step_estimate(wl, 0, threads=cores, view_ids=[v], stride=stride)
        if k >= args.warmup:
            times.append(step_s)
            samples.append(time.time() - ts)
    spent = time.time() - t0
    step_s = statistics.mean(times)
    val = 1.0 / step_s
    # ms_per_step is what each timed step ran (the bounded sample); value is
    # the whole workload's steps/s extrapolated from it (sampled tiles scaled
    # up, one view scaled to all views), as extrapolated_ms_per_full_step.
    line = {"metric": METRIC, "value": round(val, 6), "unit": "steps/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(statistics.mean(samples) * 1000, 1),
            "extrapolated_ms_per_full_step": round(step_s * 1000, 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": workload_config(args.workload, wl),
            "cpu_baseline": {"value": round(val, 6), "unit": "steps/s", "cores": cores, "kind": "port",
                             "sample": f"each step one view (rotating) of {nv}: projection, tile lists, L1+SSIM, "
                                       + (f"parameter chain in full, per-pixel walks on every {stride}th tile scaled by {stride}"
                                          if stride > 1 else "parameter chain and per-pixel walks in full (every tile)")
                                       + (f", extrapolated to all {nv} views" if nv > 1 else "")
                                       + "; Adam over all parameters",
                             "extrapolated": stride > 1 or nv > 1,
                             "sample_fraction_of_pixel_walks": round(1.0 / (stride * nv), 6),
                             "seconds_spent": round(spent, 2)},
            "e2e": {"value": round(val, 6), "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "the reference (Rust + WGSL on wgpu/Vulkan) cannot be built or run here; this is its CPU "
                    "renderer's algorithm restated in C++"}
    print(json.dumps(line))


if __name__ == "__main__":
    main()
