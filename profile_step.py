"""Runs training steps of a synthetic workload for a profiler to capture.

    python profile_step.py --workload ring2_200k --steps 2 --shapes 128,2,64,4

Sets up the workload exactly as the benchmark does (target images rendered
from the seed-1 scene, optimizer initialised), applies the given raster launch
shapes (or autotunes when none are given), runs ``--warmup`` steps, then
``--steps`` steps of the requested form, and prints one JSON line with the
milliseconds per step, the tile-entry count and the raster kernels' work
on the last step (gs_raster_work, counted after the timed steps). Every step
is a complete
forward + loss + backward + Adam pass; nothing is skipped. Launch order per
chosen step: projection, depth sort, entry scan, expansion, tile sort, ranges,
forward raster, the occlusion cut's completion pass (gate, flagged counts,
entry scan, guard, range reset, expansion, tile sort, range fix, forward
raster), L1+SSIM, backward raster, projection backward + Adam.
"""
from __future__ import annotations

import argparse
import json
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def main(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("--workload", default="ring2_200k")
    p.add_argument("--steps", type=int, default=2)
    p.add_argument("--warmup", type=int, default=1)
    p.add_argument("--form", choices=["chosen", "plain"], default="chosen")
    p.add_argument("--precision", default="f16")
    p.add_argument("--shapes", default="", help="fwd_batch,fwd_ppt,bwd_batch,bwd_ppt (default: autotune)")
    a = p.parse_args(argv)

    import torch

    from splattar_b200.rasterizer import AdamSettings, Rasterizer, StepSettings
    from splattar_b200.synthetic import workload

    wl = workload(a.workload)
    cams, n, nv, P = wl.cameras, wl.surfels.n, len(wl.cameras), wl.pixels
    rast = Rasterizer(n, 0, 0, int(min(4.2e9, 96 * n * nv)), max_views=nv, max_pixels=P, precision=a.precision,
                      color_only=True)
    rast.upload_scene(wl.target_surfels.scene_input())
    rast.forward(cams, n)
    rast.check()
    rast.write("target", rast.read("out_color", 4 * P))
    rast.upload_scene(wl.surfels.scene_input())
    rast.optimizer_init(n)
    if a.shapes:
        fb, fp, bb, bp = (int(x) for x in a.shapes.split(","))
        rast.set_launch_shapes(fb, fp, bb, bp)
        shapes = {"fwd_batch": fb, "fwd_pixels_per_thread": fp, "bwd_batch": bb, "bwd_pixels_per_thread": bp}
    else:
        shapes = rast.autotune(cams, n)
    step = StepSettings(0.8, 0.2, AdamSettings(eps=1e-15), a.form)
    stream = torch.cuda.current_stream()
    for _ in range(a.warmup):
        rast.train_step(cams, n, step, stream.cuda_stream)
    rast.check(stream.cuda_stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(a.steps):
        rast.train_step(cams, n, step, stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize()
    rast.check(stream.cuda_stream)
    print(json.dumps({"workload": a.workload, "form": a.form, "steps": a.steps, "shapes": shapes,
                      "ms_per_step": round(e0.elapsed_time(e1) / max(1, a.steps), 4),
                      "tile_entries": rast.entry_count(), "raster_work": rast.raster_work(stream.cuda_stream)}))
    rast.close()


if __name__ == "__main__":
    main()
