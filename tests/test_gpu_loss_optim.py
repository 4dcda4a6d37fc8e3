"""L1+SSIM loss/gradient and the Adam optimizer on the GPU against the
oracle: first_attempt/crates/gs-train/tests/adam.rs:37-98 (5 steps × 3
activations, |Δ| < 1e-5) and the SSIM restatement of
first_attempt/crates/gs-train/src/shaders/ssim.wgsl (reference form and the
benchmark form)."""
import ctypes

import numpy as np
import pytest

import oracle
from gpu_util import forward
from scenes import make_scene
from splattar_b200 import Rasterizer, adam_flat

pytestmark = pytest.mark.gpu


def _images(seed, P, smooth=True):
    rng = np.random.default_rng(seed)
    img = rng.uniform(0.0, 1.0, (P, 4))
    ref = np.clip(img + rng.normal(0, 0.15, (P, 4)), 0, 1)
    return img, ref


@pytest.mark.parametrize("size,w_l1,w_ssim", [((64, 48), 0.8, 0.2), ((37, 53), 0.8, 0.1), ((128, 128), 0.0, 1.0),
                                              ((45, 300), 0.8, 0.2), ((300, 261), 0.8, 0.2)])
def test_l1_ssim_matches_oracle(size, w_l1, w_ssim):
    W, H = size
    scene, cam = make_scene(5, 10, 0, 32)
    cam.width, cam.height = W, H
    rast, _ = forward(scene, cam)
    P = W * H
    img, ref = _images(W * 1000 + H, P)
    rast.write("out_color", img.astype(np.float32).ravel())
    rast.write("target", ref.astype(np.float32).ravel())
    rast.loss_l1_ssim(w_l1, w_ssim)
    rast.check()
    dl = rast.read("dl_dcolor", 4 * P).reshape(P, 4)
    sums = rast.read("loss", 2)
    loss_o, dl_o, l1_o, ss_o = oracle.l1_ssim(img.astype(np.float32), ref.astype(np.float32), W, H, w_l1, w_ssim)
    assert abs(sums[0] - l1_o) <= 1e-4 * abs(l1_o) + 1e-3
    assert abs(sums[1] - ss_o) <= 1e-4 * abs(ss_o) + 1e-3
    scale = np.abs(dl_o[:, :3]).max()
    assert np.abs(dl[:, :3] - dl_o[:, :3]).max() <= 2e-4 * scale
    assert np.all(dl[:, 3] == 0)


def test_l1_ssim_two_views_batched():
    """Per-view normalisation: two views of different sizes in one pass give
    each view's own loss and gradient."""
    s, c = make_scene(6, 10, 0, 32)
    c2 = c.copy()
    c.width, c.height = 40, 24
    c2.width, c2.height = 24, 56
    from gpu_util import raster_camera, scene_input
    rast = Rasterizer(s.n, 0, 0, 0, max_views=2, max_pixels=40 * 24 + 24 * 56)
    rast.upload_scene(scene_input(s))
    rast.forward([raster_camera(c, 0), raster_camera(c2, 0)], s.n)
    rast.check()
    off1, _ = rast.view_offset(1)
    P = 40 * 24 + 24 * 56
    img, ref = _images(3, P)
    rast.write("out_color", img.astype(np.float32).ravel())
    rast.write("target", ref.astype(np.float32).ravel())
    rast.loss_l1_ssim(0.8, 0.2)
    rast.check()
    dl = rast.read("dl_dcolor", 4 * P).reshape(P, 4)
    for (a, b, W, H, v) in ((0, off1, 40, 24, 0), (off1, P, 24, 56, 1)):
        _, dl_o, l1_o, ss_o = oracle.l1_ssim(img[a:b].astype(np.float32), ref[a:b].astype(np.float32), W, H, 0.8, 0.2)
        assert np.abs(dl[a:b, :3] - dl_o[:, :3]).max() <= 2e-4 * np.abs(dl_o[:, :3]).max()


def xorshift_pm1(state):
    M = (1 << 64) - 1
    x = state
    x ^= (x << 13) & M
    x ^= x >> 7
    x ^= (x << 17) & M
    return x, ((x >> 11) / float(1 << 53)) * 2.0 - 1.0


@pytest.mark.parametrize("activation", [0, 1, 2])
def test_adam_matches_cpu_reference(activation):
    import torch
    N, STEPS, LR = 1000, 5, 0.01
    s = 0xADA ^ activation
    init = []
    for _ in range(N):
        s, u = xorshift_pm1(s)
        init.append(np.float32(u * 0.8))
    grads = []
    for _ in range(STEPS):
        g = []
        for _ in range(N):
            s, u = xorshift_pm1(s)
            g.append(np.float32(u))
        grads.append(np.array(g, np.float32))
    init = np.array(init, np.float32)
    # CPU reference in f32 exactly as adam.rs:51-65 writes it.
    p = init.copy(); m = np.zeros(N, np.float32); v = np.zeros(N, np.float32)
    for t, g in enumerate(grads, start=1):
        if activation == 1:
            da = np.exp(p)
        elif activation == 2:
            sg = 1 / (1 + np.exp(-p)); da = sg * (1 - sg)
        else:
            da = np.ones_like(p)
        gg = (g * da).astype(np.float32)
        m = (np.float32(0.9) * m + np.float32(0.1) * gg).astype(np.float32)
        v = (np.float32(0.999) * v + np.float32(0.001) * gg * gg).astype(np.float32)
        mh = m / np.float32(1 - np.float32(0.9) ** t)
        vh = v / np.float32(1 - np.float32(0.999) ** t)
        p = (p - np.float32(LR) * mh / (np.sqrt(vh) + np.float32(1e-8))).astype(np.float32)
    raw = torch.from_numpy(init.copy()).cuda()
    mm = torch.zeros(N, device="cuda"); vv = torch.zeros(N, device="cuda"); act = torch.zeros(N, device="cuda")
    for t, g in enumerate(grads, start=1):
        tg = torch.from_numpy(g).cuda()
        adam_flat(raw.data_ptr(), tg.data_ptr(), mm.data_ptr(), vv.data_ptr(), act.data_ptr(), N, activation, LR,
                  t=t)
    torch.cuda.synchronize()
    got = raw.cpu().numpy()
    assert np.abs(got - p).max() < 1e-5
    a = act.cpu().numpy()
    want_act = np.exp(got) if activation == 1 else (1 / (1 + np.exp(-got)) if activation == 2 else got)
    assert np.abs(a - want_act).max() < 1e-5


def test_optimizer_init_inverts_activations():
    from gpu_util import scene_input
    scene, cam = make_scene(8, 30, 1, 32)
    rast = Rasterizer(scene.n, 32, 32)
    rast.upload_scene(scene_input(scene))
    rast.optimizer_init(scene.n)
    n = scene.n
    raw_s = rast.read("raw_scales", 2 * n).reshape(n, 2)
    raw_o = rast.read("raw_opacity", n)
    assert np.allclose(raw_s, np.log(scene.scales), atol=1e-5)
    o = np.clip(scene.opacity, 1e-4, 1 - 1e-4)
    assert np.allclose(raw_o, np.log(o / (1 - o)), atol=1e-4)
    act_s = rast.read("scales", 2 * n).reshape(n, 2)
    assert np.allclose(act_s, scene.scales, rtol=1e-5)
