"""Densify/prune compaction on the GPU against its numpy restatement
(oracle.densify): surfels below the opacity threshold are removed, surfels
whose mean |dL/dpos| over the accumulated steps exceeds the gradient threshold
are cloned with zeroed Adam moments, survivors keep their order and clones
follow, clones past the capacity are dropped. Copies are exact, so the check
is bit-exact; the accumulator restarts at zero."""
import numpy as np
import pytest

import oracle
from gpu_util import raster_camera, scene_input
from splattar_b200 import Rasterizer, StepSettings
from splattar_b200.rasterizer import AdamSettings
from test_gpu_train_step import multi_view_setup

pytestmark = pytest.mark.gpu

CLASSES = (("pos", 4), ("scales", 2), ("quat", 4), ("opacity", 1), ("sh", 48))
ACT_BUF = {"pos": "positions", "scales": "scales", "quat": "quats", "opacity": "opacities", "sh": "sh"}


def _state(r, n):
    arrays, widths = {}, {}
    for name, w in CLASSES:
        for kind, buf in (("raw", f"raw_{name}"), ("act", ACT_BUF[name]), ("m", f"m_{name}"), ("v", f"v_{name}")):
            arrays[f"{kind}_{name}"] = r.read(buf, w * n).reshape(n, w)
            widths[f"{kind}_{name}"] = w
    return arrays, widths


def _run(form, capacity_extra, steps=3):
    scene, cams = multi_view_setup()
    n = scene.n
    rc = [raster_camera(c, 3) for c in cams]
    cap = n + capacity_extra
    P = sum(c.width * c.height for c in cams)
    r = Rasterizer(cap, 0, 0, 64 * cap * len(cams), max_views=len(cams), max_pixels=P, color_only=True)
    r.upload_scene(scene_input(scene))
    r.forward(rc, n)
    r.check()
    tgt = r.read("out_color", 4 * P)
    r.write("target", np.clip(tgt + 0.05, 0, 1).astype(np.float32))
    r.optimizer_init(n)
    for _ in range(steps):
        r.train_step(rc, n, StepSettings(0.8, 0.2, AdamSettings(eps=1e-15), form))
    r.check()
    arrays, widths = _state(r, n)
    gsum = r.read("grad_norm_sum", n)
    opac = r.read("opacities", n)
    othr = float(np.quantile(opac, 0.3))
    gthr = float(np.quantile(gsum / steps, 0.7))
    want, n_want = oracle.densify(arrays, widths, {k for k in arrays if k[0] in "mv"}, gsum, steps, opac, gthr,
                                  othr, cap)
    n_out = r.densify_prune(gthr, othr, n)
    assert n_out == n_want
    got, _ = _state(r, n_out)
    for k in want:
        assert np.array_equal(got[k], want[k]), k
    assert np.all(r.read("grad_norm_sum", cap) == 0)
    # training continues on the new count
    r.train_step(rc, n_out, StepSettings(0.8, 0.2, AdamSettings(eps=1e-15), form))
    r.check()
    return n, n_out


@pytest.mark.parametrize("form", ["chosen", "plain"])
def test_densify_matches_restatement(form):
    n, n_out = _run(form, capacity_extra=10_000)
    assert n_out != n


def test_densify_clones_truncated_at_capacity():
    n, n_out = _run("chosen", capacity_extra=7)
    assert n_out <= n + 7
