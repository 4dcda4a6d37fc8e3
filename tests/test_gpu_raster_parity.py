"""CUDA forward/backward rasterizer vs the f64 oracle, on the reference's own
parity cases (crates/gs-kernels/tests/raster_parity.rs:20-290) and tolerances:
forward colour |Δ| < 3e-3 per pixel and < 3e-4 mean; gradients
err ≤ 1e-5 + 2e-3·max(|g|) (aux losses 6e-3, camera 3e-2). Contributor counts
must match exactly on every pixel the oracle does not flag as marginal."""
import numpy as np
import pytest

import oracle
from gpu_util import GradCheck, backward, f32_cam, f32_scene, forward
from scenes import XorShift, make_scene

pytestmark = pytest.mark.gpu


def run_parity(seed, n, deg, size, **kw):
    scene, cam = make_scene(seed, n, deg, size)
    sc32, cam32 = f32_scene(scene), f32_cam(cam)
    cpu = oracle.render(sc32, cam32)
    rast, gpu = forward(scene, cam, **kw)
    diff = np.abs(gpu["color"][:, :3] - cpu["color"])
    assert diff.max() < 3e-3, f"seed {seed}: max colour diff {diff.max():.2e}"
    assert diff.mean() < 3e-4, f"seed {seed}: mean colour diff {diff.mean():.2e}"
    assert np.abs(gpu["color"][:, 3] - cpu["alpha"]).max() < 3e-3
    assert np.abs(gpu["aux"][:, 0] - cpu["trans"]).max() < 3e-3
    assert np.abs(gpu["aux"][:, 1] - cpu["depth"]).max() < 3e-2
    assert np.abs(gpu["normal"][:, :3] - cpu["normal"]).max() < 3e-3
    ok = ~cpu["marginal"]
    mism = (gpu["ncontrib"].astype(np.int64) != cpu["ncontrib"]) & ok
    assert not mism.any(), f"seed {seed}: n_contrib differs on {int(mism.sum())} non-marginal pixels"
    return rast, diff


@pytest.mark.parametrize("seed,n,deg,size", [(101, 20, 0, 64), (202, 20, 1, 64), (303, 12, 3, 48), (404, 50, 1, 128)])
def test_forward_matches_cpu_oracle(seed, n, deg, size):
    run_parity(seed, n, deg, size)


@pytest.mark.parametrize("batch", [64, 256])
def test_forward_batch_depths_agree(batch):
    scene, cam = make_scene(404, 50, 1, 128)
    _, a = forward(scene, cam)
    _, b = forward(scene, cam, batch=batch)
    assert np.array_equal(a["color"], b["color"]) and np.array_equal(a["ncontrib"], b["ncontrib"])


@pytest.mark.parametrize("batch,ppt", [(64, 1), (128, 1), (256, 1), (64, 2), (128, 2), (64, 4)])
def test_forward_pixel_splits_agree(batch, ppt):
    scene, cam = make_scene(404, 50, 1, 128)
    _, a = forward(scene, cam, batch=128, pixels_per_thread=1)
    _, b = forward(scene, cam, batch=batch, pixels_per_thread=ppt)
    for k in ("color", "aux", "normal", "ncontrib"):
        assert np.array_equal(a[k], b[k]), k


def test_forward_persistent_equals_plain_grid():
    scene, cam = make_scene(202, 40, 3, 96)
    _, a = forward(scene, cam)
    _, b = forward(scene, cam, persistent=True)
    assert np.array_equal(a["color"], b["color"]) and np.array_equal(a["ncontrib"], b["ncontrib"])


def weights(seed, P, aux):
    rng = XorShift(seed ^ 0xFEED)
    w = np.array([[rng.uniform(-1, 1) for _ in range(3)] for _ in range(P)])
    wd = np.array([rng.uniform(-0.3, 0.3) if aux else 0.0 for _ in range(P)])
    wn = np.array([[rng.uniform(-0.5, 0.5) for _ in range(3)] if aux else [0.0] * 3 for _ in range(P)])
    return w, wd, wn


def run_grad_parity(seed, n, deg, size, aux=False, rel=2e-3, cam_rel=2e-3, **kw):
    scene, cam = make_scene(seed, n, deg, size)
    P = size * size
    w, wd, wn = weights(seed, P, aux)
    lam = 0.35 if aux else 0.0
    sc32, cam32 = f32_scene(scene), f32_cam(cam)
    cpu = oracle.gradients(sc32, cam32, w, wd, wn, lam)
    rast, _ = forward(scene, cam, **kw)
    rast.lambda_dist = lam
    dlc = np.concatenate([w, wd[:, None]], axis=1)
    dln = np.concatenate([wn, np.zeros((P, 1))], axis=1)
    g = backward(rast, scene, dlc, dln)
    ck = GradCheck(rel)
    ncoef = (deg + 1) ** 2
    ck.check("pos", g["pos"], cpu["pos"])
    ck.check("scales", g["scales"], cpu["scales"])
    ck.check("quat", g["quat"], cpu["quat"])
    ck.check("opacity", g["opacity"], cpu["opacity"])
    ck.check("sh", g["sh"][:, :3 * ncoef], cpu["sh"][:, :3 * ncoef])
    assert np.all(g["sh"][:, 3 * ncoef:] == 0)
    cc = GradCheck(cam_rel)
    cc.check("dl_dR_cam", g["cam"][:9], cpu["dl_dr_cam"])
    cc.check("cam_center", g["cam"][9:12], cpu["cam_center"])
    cc.check("focal", g["cam"][12:13], [cpu["focal"]])
    return ck, cc


@pytest.mark.parametrize("seed,n,deg,size", [(111, 15, 0, 48), (222, 15, 1, 48), (333, 10, 3, 40)])
def test_backward_matches_cpu_oracle(seed, n, deg, size):
    ck, cc = run_grad_parity(seed, n, deg, size)
    print(f"grad parity seed={seed}: worst rel {ck.worst:.2e} at {ck.label}; camera {cc.worst:.2e} at {cc.label}")


@pytest.mark.parametrize("seed,n,deg,size", [(444, 12, 0, 40), (555, 12, 1, 40)])
def test_backward_aux_losses_match_cpu_oracle(seed, n, deg, size):
    run_grad_parity(seed, n, deg, size, aux=True, rel=6e-3, cam_rel=3e-2)


def test_backward_deterministic_mode_matches_and_repeats():
    a = run_grad_parity(222, 15, 1, 48, deterministic=True)
    scene, cam = make_scene(222, 15, 1, 48)
    P = 48 * 48
    w, _, _ = weights(222, P, False)
    dlc = np.concatenate([w, np.zeros((P, 1))], axis=1)
    outs = []
    for _ in range(2):
        rast, _ = forward(scene, cam, deterministic=True)
        outs.append(backward(rast, scene, dlc))
    for k in ("pos", "scales", "quat", "opacity", "sh", "cam"):
        assert np.array_equal(outs[0][k], outs[1][k]), k
    assert a[0].worst < 2e-3


def test_backward_persistent_matches():
    run_grad_parity(333, 10, 3, 40, persistent=True)
