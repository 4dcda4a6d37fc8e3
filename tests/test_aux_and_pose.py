"""Normal-consistency loss (first_attempt/crates/gs-train/src/shaders/
normal_loss.wgsl) and camera pose refinement (crates/gs-track/src/lib.rs:
289-337). CPU: the normal-loss restatement against central differences of its
own loss (α and orientation detached), the pose step's sign conventions by
descent, adam6 against its formula. GPU: the CUDA normal loss against the
restatement."""
import math

import numpy as np
import pytest

import oracle
from splattar_b200.rasterizer import RasterCamera, camera_adam6, camera_apply_step, camera_rotation, camera_step_grad


def _surface(W=24, H=20, seed=0):
    rng = np.random.default_rng(seed)
    ys, xs = np.mgrid[0:H, 0:W]
    alpha = np.clip(0.6 + 0.3 * np.sin(xs * 0.3) * np.cos(ys * 0.2) + 0.05 * rng.normal(size=(H, W)), 0, 1)
    alpha[3, 4] = 0.1  # below alpha_min
    depth = 2.0 + 0.2 * np.sin(xs * 0.25 + ys * 0.15) + 0.02 * rng.normal(size=(H, W))
    normal = rng.normal(size=(H, W, 3)) * 0.3 + np.array([0.0, 0.0, 1.0])
    return alpha.ravel(), (depth * alpha).ravel(), normal.reshape(-1, 3), W, H


def test_normal_loss_gradients_match_central_differences():
    alpha, dacc, nrm, W, H = _surface()
    lam, f = 3.0, 20.0
    _, dn, dd = oracle.normal_loss(alpha, dacc, nrm, W, H, f, lam)
    rng = np.random.default_rng(1)

    def L(dacc_, nrm_):
        return lam / (W * H) * oracle.normal_loss(alpha, dacc_, nrm_, W, H, f, lam)[0]
    for _ in range(12):
        i, c = int(rng.integers(0, W * H)), int(rng.integers(0, 3))
        h = 1e-6
        a, b = nrm.copy(), nrm.copy()
        a[i, c] += h
        b[i, c] -= h
        assert abs((L(dacc, a) - L(dacc, b)) / (2 * h) - dn[i, c]) < 1e-7
        j = int(rng.integers(0, W * H))
        a, b = dacc.copy(), dacc.copy()
        a[j] += h
        b[j] -= h
        assert abs((L(a, nrm) - L(b, nrm)) / (2 * h) - dd[j]) < 1e-7


def test_pose_step_descends_a_rotation_objective():
    rng = np.random.default_rng(2)
    W = rng.normal(size=9).astype(np.float32)  # f(R) = Σ W∘R (column-major)
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    cam = RasterCamera((0.1, 0.2, 0.3), tuple(q), 100.0, 0, 64, 64)

    def f(c):
        return float((camera_rotation(c).astype(np.float64) * W).sum())
    g = camera_step_grad(np.concatenate([W, [0.5, -0.25, 0.125], np.zeros(4)]), q)
    assert np.allclose(g[3:], [0.5, -0.25, 0.125])
    h = 1e-3
    for i in range(3):
        e = np.zeros(6, np.float32)
        e[i] = h
        fd = (f(camera_apply_step(cam, -e)) - f(camera_apply_step(cam, e))) / (2 * h)
        assert abs(fd - g[i]) < 2e-3 * max(1.0, abs(g[i])), (i, fd, g[i])
    step = 1e-2 * g
    assert f(camera_apply_step(cam, step)) < f(cam)
    moved = camera_apply_step(cam, np.array([0, 0, 0, 0.5, -0.25, 0.125], np.float32))
    assert np.allclose(moved.center, [0.1 - 0.5, 0.2 + 0.25, 0.3 - 0.125], atol=1e-6)


def test_pose_step_rejects_non_finite():
    from splattar_b200 import GsError
    g = np.zeros(16, np.float32)
    g[4] = np.nan
    with pytest.raises(GsError, match="GS_ERR_NONFINITE"):
        camera_step_grad(g, [0, 0, 0, 1])


def test_adam6_formula():
    m, v = np.zeros(6, np.float32), np.zeros(6, np.float32)
    mm, vv = np.zeros(6), np.zeros(6)
    rng = np.random.default_rng(3)
    for t in range(1, 4):
        g = rng.normal(size=6).astype(np.float32)
        step = camera_adam6(m, v, t, g, 1e-3, 2e-2)
        mm = 0.9 * mm + 0.1 * g
        vv = 0.999 * vv + 0.001 * g * g
        lr = np.array([1e-3] * 3 + [2e-2] * 3)
        want = lr * (mm / (1 - 0.9 ** t)) / (np.sqrt(vv / (1 - 0.999 ** t)) + 1e-10)
        assert np.allclose(step, want, rtol=1e-4)


@pytest.mark.gpu
def test_cuda_normal_loss_matches_restatement():
    from gpu_util import raster_camera, scene_input
    from scenes import make_scene
    from splattar_b200 import Rasterizer
    alpha, dacc, nrm, W, H = _surface(40, 32, 5)
    scene, cam = make_scene(5, 10, 0, 32)
    cam.width, cam.height = W, H
    r = Rasterizer(scene.n, W, H, 64 * scene.n)
    r.upload_scene(scene_input(scene))
    r.forward(raster_camera(cam, 0), scene.n)
    r.check()
    P = W * H
    col = np.zeros((P, 4), np.float32)
    col[:, 3] = alpha
    aux = np.zeros((P, 4), np.float32)
    aux[:, 1] = dacc
    nr4 = np.zeros((P, 4), np.float32)
    nr4[:, :3] = nrm
    r.write("out_color", col.ravel())
    r.write("out_aux", aux.ravel())
    r.write("out_normal", nr4.ravel())
    rgb = np.random.default_rng(6).normal(size=(P, 4)).astype(np.float32)
    r.write("dl_dcolor", rgb.ravel())
    lam = 2.5
    r.loss_normal(lam, 0.2)
    r.check()
    f32 = lambda a: np.asarray(a, np.float32).astype(np.float64)  # noqa: E731
    total, dn, dd = oracle.normal_loss(f32(alpha), f32(dacc), f32(nrm), W, H, float(np.float32(cam.focal)), lam)
    got_dn = r.read("dl_dnormal", 4 * P).reshape(P, 4)
    got_c = r.read("dl_dcolor", 4 * P).reshape(P, 4)
    assert np.array_equal(got_c[:, :3], rgb[:, :3])  # colour channels untouched
    assert np.abs(got_dn[:, :3] - dn).max() <= 1e-4 * np.abs(dn).max() + 1e-9
    assert np.abs(got_c[:, 3] - dd).max() <= 1e-4 * np.abs(dd).max() + 1e-9
    assert abs(r.read("normal_loss", 1)[0] - total) <= 1e-4 * abs(total)
