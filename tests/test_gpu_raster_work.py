"""gs_raster_work: the raster kernels' work on the last forward, counted on
the device (forward hit evaluations, contributing pairs, backward hit
evaluations, pixels), which the benchmark turns into the compute side of the
raster kernels' roofline.

Contributing pairs are a property of the scene (alpha >= 1/255 before the
pixel terminates), and an entry dropped by tight binning or the occlusion cut
is one whose alpha box misses the tile or that lies past every pixel's
termination, so the chosen training step must count exactly the contributing
pairs and forward evaluations of the reference-binned forward at the same
parameters; its backward evaluates fewer entries (the row-group summary)."""
import numpy as np
import pytest

import oracle
from gpu_util import f32_cam, f32_scene, forward, raster_camera, scene_input
from scenes import make_scene
from splattar_b200 import AdamSettings, Rasterizer, StepSettings

pytestmark = pytest.mark.gpu


def test_raster_work_counts_match_oracle_contributors():
    scene, cam = make_scene(18, 40, 1, 64)
    rast, out = forward(scene, cam)
    wk = rast.raster_work()
    ref = oracle.render(f32_scene(scene), f32_cam(cam))
    P = cam.width * cam.height
    assert wk["pixels"] == P
    marg = ref["marginal"]
    # a decision on a marginal pixel may flip between f32 and f64
    slack = int((ref["count"][marg] + 2).sum())
    assert abs(wk["contrib_pairs"] - int(ref["count"].sum())) <= slack, (wk, int(ref["count"].sum()), slack)
    assert wk["fwd_evals"] >= wk["bwd_evals"] >= wk["contrib_pairs"] > 0


def test_chosen_step_counts_equal_reference_binning():
    scene, cam = make_scene(19, 400, 3, 64)
    cams = []
    for k, (w, h) in enumerate([(64, 64), (80, 48), (96, 72)]):
        c = cam.copy()
        c.width, c.height = w, h
        c.quat = np.array(cam.quat) + np.array([0.02 * k, -0.01 * k, 0.0, 0.0])
        cams.append(c)
    rc = [raster_camera(c, 3) for c in cams]
    P = sum(c.width * c.height for c in cams)
    r = Rasterizer(scene.n, 0, 0, 0, max_views=3, max_pixels=P, color_only=True)
    r.upload_scene(scene_input(scene))
    r.write("target", np.random.default_rng(2).uniform(0, 1, 4 * P).astype(np.float32))
    r.optimizer_init(scene.n)
    for _ in range(3):  # the cut is recorded by the first step and used by the next
        # reference binning at the parameters the chosen step starts from
        r.forward(rc, scene.n)
        r.check()
        ref = r.raster_work()
        r.train_step(rc, scene.n, StepSettings(0.8, 0.2, AdamSettings(eps=1e-15), "chosen"))
        r.check()
        got = r.raster_work()
        assert got["pixels"] == ref["pixels"] == P
        assert got["contrib_pairs"] == ref["contrib_pairs"], (got, ref)
        assert got["fwd_evals"] == ref["fwd_evals"], (got, ref)
        assert got["contrib_pairs"] <= got["bwd_evals"] <= ref["bwd_evals"], (got, ref)
