"""Precision report: the CUDA forward and backward with FP32, FP16 and BF16
storage of SH and projected record fields (geometry, colour, opacity,
compositing and accumulation stay FP32; normal and depth are 16-bit), each
against the FP64 oracle (tile-binned walk) on the same f32-rounded scene:
image PSNR and, for the linear loss sum w.colour, the relative L2 error of
each parameter class's gradient. Pixels the oracle flags as marginal carry no
loss weight and are left out of the PSNR; besides the fixed bands around the
alpha, clamp, transmittance and branch thresholds, the oracle flags a pixel
where a float32 evaluation of a hit's exponent is ill-conditioned (surfels
seen nearly edge-on, where the ray-splat solve divides by det ~ 0) or a
decision lies within that error bound.

Targets: PSNR >= 60 dB and gradient relative error <= 1e-3 for every storage
precision. BF16 misses the gradient target by construction: its 8-bit
significand rounds SH coefficients of N(0, 0.1) by up to 2e-4 absolute, which
alone moves the colour gradients' chain by about 1.2e-3 relative (measured by
rounding the oracle's own SH). That miss is reported as an expected failure;
BF16 is held to 3e-3.

Default size: 1,000,000 clustered surfels (SH degree 3) and one 1920x1080 view.
With GS_PRECISION_FULL=1: 3,000,000 surfels and four 1920x1080 views."""
import json
import os

import numpy as np
import pytest

import oracle
from splattar_b200 import Rasterizer
from splattar_b200.synthetic import make_surfels, ring_cameras

pytestmark = pytest.mark.gpu

CLASSES = (("pos", 4, 3), ("scales", 2, 2), ("quat", 4, 4), ("opacity", 1, 1), ("sh", 48, 48))
MIN_PSNR = {"f32": 60.0, "f16": 60.0, "bf16": 60.0}
TARGET_GRAD_ERR = 1e-3
MAX_GRAD_ERR = {"f32": 1e-3, "f16": 1e-3, "bf16": 3e-3}
_REPORT = {}


def _setup():
    if os.environ.get("GS_PRECISION_FULL") == "1":
        n, res = 3_000_000, [(1920, 1080)] * 4
    else:
        n, res = 1_000_000, [(1920, 1080)]
    s = make_surfels(n, 0, True, 3, 0.1)
    cams = ring_cameras(res)
    return s, cams


def _gpu(s, cam, precision, w4):
    n, P = s.n, cam.width * cam.height
    r = Rasterizer(n, cam.width, cam.height, 64 * n, precision=precision)
    r.upload_scene(s.scene_input())
    r.forward(cam, n)
    r.check()
    img = r.read("out_color", 4 * P).reshape(P, 4)[:, :3].astype(np.float64)
    r.write("dl_dcolor", w4.ravel())
    r.write("dl_dnormal", np.zeros(4 * P, np.float32))
    r.backward(n)
    r.check()
    g = {}
    for name, width, used in CLASSES:
        buf = {"pos": "grad_pos", "scales": "grad_scales", "quat": "grad_quat", "opacity": "grad_opacity",
               "sh": "grad_sh"}[name]
        g[name] = r.read(buf, width * n).reshape(n, width)[:, :used].astype(np.float64)
    r.close()
    return img, g


def _report():
    if _REPORT:
        return _REPORT
    s, cams = _setup()
    scene = oracle.Scene(s.positions.astype(np.float64), s.scales.astype(np.float64), s.quats.astype(np.float64),
                         s.opacities.astype(np.float64), s.sh48().astype(np.float64), 3)
    report = {"surfels": s.n, "views": [f"{c.width}x{c.height}" for c in cams], "precisions": {}}
    acc = {p: {"se": 0.0, "cnt": 0, "gerr": {k: 0.0 for k, _, _ in CLASSES}} for p in MIN_PSNR}
    gref_norm = {k: 0.0 for k, _, _ in CLASSES}
    for v, c in enumerate(cams):
        cam = oracle.Camera(np.array(c.center, np.float64), np.array(c.quat, np.float64), float(c.focal), c.width,
                            c.height)
        P = c.width * c.height
        ref = oracle.render(scene, cam)
        keep = ~ref["marginal"].astype(bool)
        w = np.random.default_rng(100 + v).uniform(-1, 1, (P, 3)).astype(np.float32)
        w[~keep] = 0.0
        gref = oracle.gradients(scene, cam, w.astype(np.float64))
        w4 = np.concatenate([w, np.zeros((P, 1), np.float32)], axis=1)
        for name, _, used in CLASSES:
            gr = gref[name].reshape(s.n, -1)[:, :used]
            gref_norm[name] += float((gr ** 2).sum())
        for prec in MIN_PSNR:
            img, g = _gpu(s, c, prec, w4)
            d = img[keep] - ref["color"][keep]
            acc[prec]["se"] += float((d ** 2).sum())
            acc[prec]["cnt"] += int(d.size)
            for name, _, used in CLASSES:
                gr = gref[name].reshape(s.n, -1)[:, :used]
                acc[prec]["gerr"][name] += float(((g[name] - gr) ** 2).sum())
    for prec, a in acc.items():
        mse = a["se"] / max(a["cnt"], 1)
        psnr = 99.0 if mse == 0 else -10.0 * np.log10(mse)
        errs = {k: float(np.sqrt(a["gerr"][k] / max(gref_norm[k], 1e-300))) for k in a["gerr"]}
        report["precisions"][prec] = {"psnr_db": round(psnr, 2), "grad_rel_l2": {k: float(f"{e:.3e}") for k, e in
                                                                                 errs.items()}}
    print("PRECISION_REPORT " + json.dumps(report))
    _REPORT.update(report)
    return _REPORT


@pytest.mark.parametrize("prec", ["f32", "f16", "bf16"])
def test_precision_report(prec):
    rep = _report()["precisions"][prec]
    assert rep["psnr_db"] >= MIN_PSNR[prec], (prec, rep)
    for k, e in rep["grad_rel_l2"].items():
        assert e <= MAX_GRAD_ERR[prec], (prec, k, e)


def test_bf16_gradient_target():
    """The 1e-3 gradient target with BF16 storage: expected to fail (see the module docstring)."""
    rep = _report()["precisions"]["bf16"]
    worst = max(rep["grad_rel_l2"].values())
    if worst > TARGET_GRAD_ERR:
        pytest.xfail(f"bf16 storage misses the 1e-3 gradient target: worst class {worst:.2e}")
    assert worst <= TARGET_GRAD_ERR
