"""Writes the golden fixtures under tests/golden/ from the oracle.

    python tests/golden/make_golden.py

The reference ships no golden vectors for this path (its tests regenerate
scenes from seeds and compare against its CPU renderer), so these fixtures
freeze the oracle's f64 outputs on a few of the reference's own seeded parity
cases (crates/gs-kernels/tests/raster_parity.rs:20-290), inputs included, so a
change of the oracle or of the CUDA path shows against a fixed answer. The
binning fixture is computed independently of the oracle by the order the
reference defines (crates/gs-kernels/src/binning.rs:5-8): one stable sort of
the expanded entries by (tile, depth bits, entry index).
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

import oracle  # noqa: E402
from gpu_util import f32_cam, f32_scene  # noqa: E402
from scenes import XorShift, make_scene  # noqa: E402


def scene_arrays(scene, cam):
    return dict(pos=scene.pos, scales=scene.scales, quat=scene.quat, opacity=scene.opacity, sh=scene.sh,
                sh_degree=np.int32(scene.sh_degree), cam_center=np.asarray(cam.center, np.float64),
                cam_quat=np.asarray(cam.quat, np.float64), focal=np.float64(cam.focal),
                width=np.int32(cam.width), height=np.int32(cam.height))


def forward_case(seed, n, deg, size):
    scene, cam = make_scene(seed, n, deg, size)
    s, c = f32_scene(scene), f32_cam(cam)
    out = oracle.render(s, c)
    keys = ("color", "alpha", "depth", "normal", "trans", "ncontrib", "marginal")  # the fixture's fields
    return dict(**scene_arrays(s, c), **{"out_" + k: out[k] for k in keys})


def gradient_case(seed, n, deg, size, aux):
    scene, cam = make_scene(seed, n, deg, size)
    s, c = f32_scene(scene), f32_cam(cam)
    P = size * size
    rng = XorShift(seed ^ 0xFEED)
    w = np.array([[rng.uniform(-1, 1) for _ in range(3)] for _ in range(P)])
    wd = np.array([rng.uniform(-0.3, 0.3) if aux else 0.0 for _ in range(P)])
    wn = np.array([[rng.uniform(-0.5, 0.5) for _ in range(3)] if aux else [0.0] * 3 for _ in range(P)])
    # the values the GPU receives are float32
    w, wd, wn = (a.astype(np.float32).astype(np.float64) for a in (w, wd, wn))
    lam = 0.35 if aux else 0.0
    g = oracle.gradients(s, c, w, wd, wn, lam)
    return dict(**scene_arrays(s, c), dl_dcolor=w, dl_ddepth=wd, dl_dnormal=wn, lambda_dist=np.float64(lam),
                **{"grad_" + k: v for k, v in g.items()})


def l1_ssim_case(W, H, seed, w_l1, w_ssim):
    rng = np.random.default_rng(seed)
    img = rng.uniform(0.0, 1.0, (W * H, 4)).astype(np.float32)
    ref = np.clip(img + rng.normal(0, 0.15, (W * H, 4)), 0, 1).astype(np.float32)
    loss, dl, l1, ss = oracle.l1_ssim(img, ref, W, H, w_l1, w_ssim)
    return dict(img=img, ref=ref, width=np.int32(W), height=np.int32(H), w_l1=np.float64(w_l1),
                w_ssim=np.float64(w_ssim), loss=np.float64(loss), dl=dl, l1_sum=np.float64(l1),
                ssim_sum=np.float64(ss))


def adam_case(seed, n=257, steps=3):
    rng = np.random.default_rng(seed)
    out = {}
    for act in (0, 1, 2):
        raw0 = rng.normal(0, 1, n).astype(np.float32)
        grads = rng.normal(0, 0.1, (steps, n)).astype(np.float32)
        raw = raw0.astype(np.float64).copy()
        m = np.zeros(n)
        v = np.zeros(n)
        for t in range(steps):
            raw, m, v, activated = oracle.adam(raw, grads[t].astype(np.float64), m, v, act, 1e-2, 0.9, 0.999,
                                               1e-8, 0.0, t + 1)
        out.update({f"raw0_{act}": raw0, f"grads_{act}": grads, f"raw_{act}": raw, f"m_{act}": m, f"v_{act}": v,
                    f"act_{act}": activated})
    return out


def binning_case(seed, tiles_x=13, tiles_y=9, n=400):
    rng = np.random.default_rng(seed)
    rects = np.zeros((n, 4), np.uint32)
    x0 = rng.integers(0, tiles_x, n)
    y0 = rng.integers(0, tiles_y, n)
    w = rng.integers(0, 4, n)
    h = rng.integers(0, 4, n)
    rects[:, 0], rects[:, 1] = x0, y0
    rects[:, 2] = np.minimum(x0 + w, tiles_x - 1)
    rects[:, 3] = np.minimum(y0 + h, tiles_y - 1)
    culled = rng.random(n) < 0.1
    rects[culled] = (1, 1, 0, 0)
    depths = rng.integers(0, 64, n).astype(np.uint32)  # many ties
    # expansion: item-major, row-major within the rect
    ent_tile, ent_item = [], []
    for i in range(n):
        x0_, y0_, x1_, y1_ = (int(v) for v in rects[i])
        for ty in range(y0_, y1_ + 1):
            for tx in range(x0_, x1_ + 1):
                ent_tile.append(ty * tiles_x + tx)
                ent_item.append(i)
    ent_tile = np.array(ent_tile, np.int64)
    ent_item = np.array(ent_item, np.uint32)
    e = np.arange(ent_tile.size)
    order = np.lexsort((e, depths[ent_item], ent_tile)).astype(np.uint32)
    T = tiles_x * tiles_y
    starts = np.searchsorted(ent_tile[order], np.arange(T), side="left")
    ends = np.searchsorted(ent_tile[order], np.arange(T), side="right")
    return dict(rects=rects, depths=depths, tiles_x=np.int32(tiles_x), tiles_y=np.int32(tiles_y),
                sorted_entries=order, entry_items=ent_item,
                ranges=np.stack([starts, ends], axis=1).astype(np.uint32))


CASES = {
    "forward_s101_n20_d0_64": lambda: forward_case(101, 20, 0, 64),
    "forward_s303_n12_d3_48": lambda: forward_case(303, 12, 3, 48),
    "gradients_s222_n15_d1_48": lambda: gradient_case(222, 15, 1, 48, False),
    "gradients_aux_s444_n12_d0_40": lambda: gradient_case(444, 12, 0, 40, True),
    "l1_ssim_37x29": lambda: l1_ssim_case(37, 29, 7, 0.8, 0.2),
    "adam_3steps": lambda: adam_case(11),
    "binning_13x9": lambda: binning_case(5),
}


def main():
    oracle.build()
    for name, fn in CASES.items():
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **fn())
        print(name, os.path.getsize(os.path.join(HERE, name + ".npz")))


if __name__ == "__main__":
    main()
