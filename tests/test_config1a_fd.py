"""Finite-difference gate at the 1,024-surfel, 128×128 size (FP64 oracle,
relative step 1e-4, 64 random parameters per attribute class):

* the rasterizer adjoint through the reference's random-weight linear loss
  Σ w·colour (crates/gs-cpu-ref/tests/gradcheck.rs:110-117), on the oracle;
* the L1+SSIM gradient (ssim.wgsl:130-143) by central differences of the
  oracle's loss, at pixels away from the |x − y| = 0 kink of the L1 term;
* on the GPU, the CUDA backward against the oracle's analytic gradients for
  the same scene and loss (tolerance of crates/gs-kernels/tests/raster_parity.rs).

Scene: surfel centres U[−1,1]³, log-scales N(−3.5, 0.5), uniform random unit
quaternions, opacity sigmoid(N(0,1)), SH degree 0 coefficients N(0, 0.3);
one 128×128 view, f = 128, eye (0, 0, −3) looking at the origin."""
import numpy as np
import pytest

import oracle
from splattar_b200.synthetic import look_at, make_surfels

N, SIZE = 1024, 128
CLASSES = (("pos", 3), ("scales", 2), ("quat", 4), ("opacity", 1), ("sh", 3))


def scene_cam(seed=0):
    s = make_surfels(N, seed, False, 0, 0.3)
    c = look_at((0.0, 0.0, -3.0), (0.0, 0.0, 0.0), SIZE, SIZE, focal=float(SIZE), sh_degree=0)
    scene = oracle.Scene(s.positions.astype(np.float64), s.scales.astype(np.float64), s.quats.astype(np.float64),
                         s.opacities.astype(np.float64), s.sh48().astype(np.float64), 0)
    cam = oracle.Camera(np.array(c.center, np.float64), np.array(c.quat, np.float64), float(c.focal), SIZE, SIZE)
    return s, c, scene, cam


def weights(seed=5):
    return np.random.default_rng(seed).uniform(-1, 1, (SIZE * SIZE, 3))


def linear_loss(scene, cam, w):
    return float((oracle.render(scene, cam)["color"] * w).sum())


def fd(scene, cam, w, key, idx, rel=1e-4):
    """Central difference with step rel·max(|x|, 1e-3); None where the loss
    jumps inside the step (steps h and h/2 disagree)."""
    x0 = getattr(scene, key)[idx]
    h = rel * max(abs(x0), 1e-3)

    def at(hh):
        sp, sm = scene.copy(), scene.copy()
        getattr(sp, key)[idx] += hh
        getattr(sm, key)[idx] -= hh
        return (linear_loss(sp, cam, w) - linear_loss(sm, cam, w)) / (2 * hh)

    a, b = at(h), at(h / 2)
    if abs(a - b) > 1e-3 * max(abs(a), abs(b)) + 1e-7:
        return None
    return b


def sample(rng, n, width, k=64):
    """k distinct (surfel, component) indices, drawn among visible surfels."""
    flat = rng.choice(n * width, size=k, replace=False)
    return [(int(f // width), int(f % width)) for f in flat]


def test_oracle_fd_gate_1024_surfels_128px():
    _, _, scene, cam = scene_cam()
    w = weights()
    g = oracle.gradients(scene, cam, w)
    rng = np.random.default_rng(11)
    for key, width in CLASSES:
        checked = jumps = 0
        nonzero = np.nonzero(np.abs(g[key].reshape(N, -1)[:, :width]).sum(axis=1) > 0)[0]
        for i, d in sample(rng, len(nonzero), width):
            idx = (int(nonzero[i]), d) if key != "opacity" else (int(nonzero[i]),)
            f = fd(scene, cam, w, key, idx)
            if f is None:
                jumps += 1
                continue
            a = float(g[key][idx])
            assert abs(a - f) <= 1e-6 + 2e-3 * max(abs(a), abs(f)), (key, idx, a, f)
            checked += 1
        assert checked >= 56 and jumps <= 8, (key, checked, jumps)


def test_l1_ssim_gradient_fd_away_from_kinks():
    rng = np.random.default_rng(3)
    W = H = 48
    img = rng.uniform(0.05, 0.95, (W * H, 4))
    ref = np.clip(img + rng.choice([-1, 1], img.shape) * rng.uniform(0.02, 0.2, img.shape), 0, 1)
    _, dl, _, _ = oracle.l1_ssim(img, ref, W, H, 0.8, 0.2)
    checked = 0
    for _ in range(64):
        p, ch = int(rng.integers(0, W * H)), int(rng.integers(0, 3))
        if abs(img[p, ch] - ref[p, ch]) < 1e-2:
            continue
        h = 1e-4 * max(abs(img[p, ch]), 1e-3)
        ip, im = img.copy(), img.copy()
        ip[p, ch] += h
        im[p, ch] -= h
        f = (oracle.l1_ssim(ip, ref, W, H, 0.8, 0.2)[0] - oracle.l1_ssim(im, ref, W, H, 0.8, 0.2)[0]) / (2 * h)
        assert abs(dl[p, ch] - f) <= 1e-9 + 1e-4 * max(abs(dl[p, ch]), abs(f)), (p, ch, dl[p, ch], f)
        checked += 1
    assert checked >= 48


@pytest.mark.gpu
def test_cuda_backward_matches_oracle_1024_surfels_128px():
    from gpu_util import GradCheck, f32_cam, f32_scene
    from splattar_b200 import Rasterizer
    s, c, scene, cam = scene_cam()
    sc32, cam32 = f32_scene(scene), f32_cam(cam)
    w = weights().astype(np.float32).astype(np.float64)
    # Pixels where an f32 decision (alpha skip or clamp, termination, branch,
    # rect truncation) may legitimately differ from f64 carry no loss weight,
    # on both sides.
    marginal = oracle.render(sc32, cam32)["marginal"].astype(bool)
    w[marginal] = 0.0
    want = oracle.gradients(sc32, cam32, w)
    r = Rasterizer(N, SIZE, SIZE, 64 * N)
    r.upload_scene(s.scene_input())
    r.forward(c, N)
    r.check()
    P = SIZE * SIZE
    r.write("dl_dcolor", np.concatenate([w, np.zeros((P, 1))], axis=1).astype(np.float32).ravel())
    r.write("dl_dnormal", np.zeros(4 * P, np.float32))
    r.backward(N)
    r.check()
    got = {"pos": r.read("grad_pos", 4 * N).reshape(N, 4)[:, :3], "scales": r.read("grad_scales", 2 * N).reshape(N, 2),
           "quat": r.read("grad_quat", 4 * N).reshape(N, 4), "opacity": r.read("grad_opacity", N),
           "sh": r.read("grad_sh", 48 * N).reshape(N, 48)[:, :3]}
    # 1,024 surfels hold a few near-grazing ones: at most 0.5% of the entries
    # may exceed 2e-3, none 2e-2.
    ck = GradCheck(2e-3, outliers=5e-3)
    for key in got:
        ck.check(key, got[key], want[key] if key != "sh" else want["sh"][:, :3])
    cc = GradCheck(3e-2)
    cam_g = r.read("grad_cam", 16)
    cc.check("cam_center", cam_g[9:12], want["cam_center"])
    cc.check("focal", cam_g[12:13], want["focal"])
