"""The training step end to end: batched multi-view passes against per-view
passes, the chosen form against the plain form, mixed-precision storage
against the f64 oracle (image PSNR, gradient relative error), and
deterministic-mode reproducibility."""
import numpy as np
import pytest

import oracle
from gpu_util import f32_cam, f32_scene, raster_camera, scene_input
from scenes import make_scene
from splattar_b200 import AdamSettings, Rasterizer, StepSettings
from splattar_b200.synthetic import look_at, make_surfels

pytestmark = pytest.mark.gpu


def multi_view_setup(seed=21, n=400):
    scene, cam = make_scene(seed, n, 3, 64)
    cams = []
    for k, (w, h) in enumerate([(64, 64), (80, 48), (40, 72)]):
        c = cam.copy()
        c.width, c.height = w, h
        c.quat = np.array(cam.quat) + np.array([0.02 * k, -0.01 * k, 0.0, 0.0])
        cams.append(c)
    return scene, cams


def psnr(a, b):
    mse = float(np.mean((np.asarray(a, np.float64) - np.asarray(b, np.float64)) ** 2))
    return 99.0 if mse == 0 else -10 * np.log10(mse)


def test_batched_forward_equals_per_view_forward():
    scene, cams = multi_view_setup()
    P = sum(c.width * c.height for c in cams)
    rc = [raster_camera(c, 3) for c in cams]
    rb = Rasterizer(scene.n, 0, 0, 0, max_views=3, max_pixels=P)
    rb.upload_scene(scene_input(scene))
    rb.forward(rc, scene.n)
    rb.check()
    allc = rb.read("out_color", 4 * P).reshape(P, 4)
    allnc = rb.read("out_ncontrib", P)
    for v, c in enumerate(cams):
        off, _ = rb.view_offset(v)
        rs = Rasterizer(scene.n, c.width, c.height)
        rs.upload_scene(scene_input(scene))
        rs.forward(rc[v], scene.n)
        rs.check()
        Pv = c.width * c.height
        assert np.array_equal(rs.read("out_color", 4 * Pv).reshape(Pv, 4), allc[off:off + Pv])
        assert np.array_equal(rs.read("out_ncontrib", Pv), allnc[off:off + Pv])


def _trainer(scene, cams, precision="f32", deterministic=False, stored_state=False):
    P = sum(c.width * c.height for c in cams)
    r = Rasterizer(scene.n, 0, 0, 0, max_views=len(cams), max_pixels=P, precision=precision,
                   deterministic=deterministic, color_only=True, stored_state=stored_state)
    r.upload_scene(scene_input(scene))
    tgt = np.random.default_rng(1).uniform(0, 1, (P, 4)).astype(np.float32)
    r.write("target", tgt.ravel())
    r.optimizer_init(scene.n)
    return r


def _params(r, n):
    return {k: r.read(k, w * n) for k, w in (("raw_pos", 4), ("raw_scales", 2), ("raw_quat", 4),
                                             ("raw_opacity", 1), ("raw_sh", 48))}


def test_chosen_step_matches_plain_step_fp32():
    scene, cams = multi_view_setup()
    rc = [raster_camera(c, 3) for c in cams]
    adam = AdamSettings(eps=1e-15)
    outs = []
    for form in ("plain", "chosen"):
        r = _trainer(scene, cams)
        for _ in range(2):
            r.train_step(rc, scene.n, StepSettings(0.8, 0.2, adam, form))
        r.check()
        outs.append((_params(r, scene.n), r.read("loss", 6)))
    (pa, la), (pb, lb) = outs
    assert np.allclose(la, lb, rtol=1e-5, atol=1e-6)
    for k in pa:
        d = np.abs(pa[k] - pb[k])
        # Adam normalises each step to ~lr; differences come from float
        # reduction order of the per-surfel gradient sums only.
        assert d.max() < 2e-4, (k, float(d.max()))


def test_gradient_sum_over_views_matches_oracle():
    """Backward over a 3-view forward = Σ over views of the oracle's single-view gradients."""
    scene, cams = multi_view_setup(33, 60)
    P = sum(c.width * c.height for c in cams)
    rc = [raster_camera(c, 3) for c in cams]
    r = Rasterizer(scene.n, 0, 0, 0, max_views=3, max_pixels=P)
    r.upload_scene(scene_input(scene))
    r.forward(rc, scene.n)
    rng = np.random.default_rng(4)
    w = rng.uniform(-1, 1, (P, 3))
    r.write("dl_dcolor", np.concatenate([w, np.zeros((P, 1))], 1).astype(np.float32).ravel())
    r.write("dl_dnormal", np.zeros(4 * P, np.float32))
    r.backward(scene.n)
    r.check()
    n = scene.n
    g = r.read("grad_pos", 4 * n).reshape(n, 4)[:, :3]
    want = np.zeros((n, 3))
    scale = np.zeros((n, 3))  # Σ over views of |per-view gradient|: the sum may cancel
    off = 0
    for c in cams:
        Pv = c.width * c.height
        gv = oracle.gradients(f32_scene(scene), f32_cam(c), w[off:off + Pv])["pos"]
        want += gv
        scale += np.abs(gv)
        off += Pv
    err = np.abs(g - want)
    assert np.all(err <= 1e-5 + 2e-3 * scale), float((err / (scale + 1e-9)).max())


@pytest.mark.parametrize("precision,min_psnr", [("f16", 60.0), ("bf16", 45.0)])
def test_mixed_precision_image_psnr_vs_f64_oracle(precision, min_psnr):
    s = make_surfels(20_000, 11, True, 3, 0.1)
    cam = look_at((0.0, 0.0, 4.0), (0, 0, 0), 320, 240, sh_degree=3)
    r = Rasterizer(s.n, 320, 240, precision=precision)
    r.upload_scene(s.scene_input())
    # the forward through the public API uses the handle's storage precision
    r.forward(cam, s.n)
    r.check()
    img = r.read("out_color", 4 * 320 * 240).reshape(-1, 4)[:, :3]
    sc = oracle.Scene(s.positions.astype(np.float64), s.scales.astype(np.float64), s.quats.astype(np.float64),
                      s.opacities.astype(np.float64), s.sh48().astype(np.float64), 3)
    oc = oracle.Camera(np.array(cam.center, np.float32).astype(np.float64),
                       np.array(cam.quat, np.float32).astype(np.float64), float(np.float32(cam.focal)), 320, 240)
    ref = oracle.render(sc, oc)["color"]
    p = psnr(img, ref)
    print(f"{precision}: PSNR {p:.1f} dB vs the f64 oracle")
    assert p >= min_psnr


def test_tight_binning_keeps_images_and_gradients():
    """Binning by the α-box instead of the reference rect drops only entries
    that cannot reach α ≥ 1/255: colour, alpha, T, depth and normal are
    bit-identical, gradients equal up to reduction order, and fewer entries."""
    s = make_surfels(30_000, 12, True, 3, 0.1)
    cam = look_at((0.0, 0.5, 4.0), (0, 0, 0), 400, 300, sh_degree=3)
    outs = []
    for tight in (False, True):
        r = Rasterizer(s.n, 400, 300, tight=tight)
        r.upload_scene(s.scene_input())
        r.forward(cam, s.n)
        r.check()
        P = 400 * 300
        o = {k: r.read(k, 4 * P) for k in ("out_color", "out_aux", "out_normal")}
        o["E"] = r.entry_count()
        w = np.random.default_rng(2).uniform(-1, 1, (P, 4)).astype(np.float32)
        w[:, 3] = 0
        r.write("dl_dcolor", w.ravel())
        r.write("dl_dnormal", np.zeros(4 * P, np.float32))
        r.backward(s.n)
        r.check()
        o["gpos"] = r.read("grad_pos", 4 * s.n)
        o["gsh"] = r.read("grad_sh", 48 * s.n)
        outs.append(o)
    a, b = outs
    for k in ("out_color", "out_aux", "out_normal"):
        assert np.array_equal(a[k], b[k]), k
    assert b["E"] < a["E"], (a["E"], b["E"])
    for k in ("gpos", "gsh"):
        assert np.allclose(a[k], b[k], rtol=1e-4, atol=1e-6), k
    print(f"entries: reference rects {a['E']}, tight {b['E']} ({a['E'] / b['E']:.2f}x)")


@pytest.mark.parametrize("form", ["chosen", "plain"])
def test_deterministic_step_is_bitwise_reproducible(form):
    """Parameters, moments and the per-view camera gradients repeat bit for bit."""
    scene, cams = multi_view_setup(44, 300)
    rc = [raster_camera(c, 3) for c in cams]
    outs = []
    for _ in range(2):
        r = _trainer(scene, cams, deterministic=True)
        for _ in range(2):
            r.train_step(rc, scene.n, StepSettings(form=form))
        r.check()
        o = _params(r, scene.n)
        o["grad_cam"] = r.read("grad_cam", 16 * len(cams))
        o["m_pos"] = r.read("m_pos", 4 * scene.n)
        outs.append(o)
    assert np.abs(outs[0]["grad_cam"]).max() > 0
    for k in outs[0]:
        assert np.array_equal(outs[0][k], outs[1][k]), k


def test_fused_adam_wait_expiry_reports_timeout_and_skips_update():
    """The chosen step's fused projection backward + Adam waits for its
    optimizer-row copies with a bounded wait. A limit of 0 makes that wait give
    up at once: every block flags the expiry, lets its copies land (the drain
    wait) and exits without updating. The step then reports
    GS_ERR_DEVICE_TIMEOUT, the parameters are unchanged, and the handle keeps
    working once the limit is restored."""
    from splattar_b200 import GsError
    scene, cams = multi_view_setup(45, 300)
    rc = [raster_camera(c, 3) for c in cams]
    r = _trainer(scene, cams)
    before = _params(r, scene.n)
    r.set_wait_limits(0)
    r.train_step(rc, scene.n, StepSettings(form="chosen"))
    with pytest.raises(GsError) as err:
        r.check()
    assert err.value.status == 4  # GS_ERR_DEVICE_TIMEOUT
    mid = _params(r, scene.n)
    for k in before:
        assert np.array_equal(before[k], mid[k]), k
    r.check()  # the error word was cleared by the report
    r.set_wait_limits(2_000_000_000)
    r.train_step(rc, scene.n, StepSettings(form="chosen"))
    r.check()
    after = _params(r, scene.n)
    assert not np.array_equal(after["raw_pos"], before["raw_pos"])
    with pytest.raises(GsError):
        r.set_wait_limits(0, 1000)  # the drain wait must stay long enough for the copies to land


def test_train_step_reduces_loss():
    """A few chosen-form steps toward a target rendered from a perturbed scene lower the loss."""
    scene, cams = multi_view_setup(55, 300)
    rc = [raster_camera(c, 3) for c in cams]
    P = sum(c.width * c.height for c in cams)
    tgt_scene = scene.copy()
    tgt_scene.pos = tgt_scene.pos + 0.02
    rt = Rasterizer(scene.n, 0, 0, 0, max_views=3, max_pixels=P)
    rt.upload_scene(scene_input(tgt_scene))
    rt.forward(rc, scene.n)
    target = rt.read("out_color", 4 * P)
    r = Rasterizer(scene.n, 0, 0, 0, max_views=3, max_pixels=P, color_only=True)
    r.upload_scene(scene_input(scene))
    r.write("target", target)
    r.optimizer_init(scene.n)
    losses = []
    for _ in range(30):
        r.train_step(rc, scene.n, StepSettings(0.8, 0.2, AdamSettings(lr={"pos": 1e-3, "scales": 5e-3,
                                                                         "quat": 1e-3, "opacity": 5e-2,
                                                                         "sh": 2.5e-3}), "chosen"))
        l = r.read("loss", 6)
        losses.append(sum(0.8 * l[2 * v] / (3 * c.width * c.height) + 0.2 * (1 - l[2 * v + 1] / (3 * c.width * c.height))
                          for v, c in enumerate(cams)))
    assert losses[-1] < 0.8 * losses[0], losses[::5]


def test_autotune_keeps_results():
    scene, cams = multi_view_setup(66, 400)
    rc = [raster_camera(c, 3) for c in cams]
    P = sum(c.width * c.height for c in cams)
    r = Rasterizer(scene.n, 0, 0, 0, max_views=3, max_pixels=P)
    r.upload_scene(scene_input(scene))
    r.optimizer_init(scene.n)  # re-derives the activated values through raw space
    r.forward(rc, scene.n)
    before = r.read("out_color", 4 * P)
    r.write("target", before)
    shapes = r.autotune(rc, scene.n)
    assert shapes["fwd_batch"] in (64, 128, 256) and shapes["fwd_pixels_per_thread"] in (1, 2, 4, 8)
    assert (shapes["bwd_batch"], shapes["bwd_pixels_per_thread"]) in ((64, 1), (64, 2), (128, 2), (64, 4), (64, 8),
                                                                      (128, 8))
    r.forward(rc, scene.n)
    assert np.array_equal(r.read("out_color", 4 * P), before)


@pytest.mark.parametrize("deterministic", [True, False])
def test_stored_state_backward_matches_recompute(deterministic):
    """Contributor masks from the forward select exactly the entries the
    recomputing backward would keep: identical parameters after three chosen
    steps (bitwise in deterministic mode)."""
    scene, cams = multi_view_setup(23, 500)
    rc = [raster_camera(c, 3) for c in cams]
    outs = []
    for stored in (False, True):
        r = _trainer(scene, cams, precision="f16", deterministic=deterministic, stored_state=stored)
        for _ in range(3):
            r.train_step(rc, scene.n, StepSettings(0.8, 0.2, AdamSettings(eps=1e-15), "chosen"))
        r.check()
        outs.append(_params(r, scene.n))
    for k in outs[0]:
        if deterministic:
            assert np.array_equal(outs[0][k], outs[1][k]), k
        else:
            assert np.allclose(outs[0][k], outs[1][k], rtol=1e-5, atol=1e-6), k


def test_async_copies_take_device_pointers():
    """write_async/read_async move data between a handle buffer and either
    pinned host memory or device memory (a prefetched input on the device)."""
    import torch
    r = Rasterizer(100, 64, 32)
    P = 64 * 32
    src = torch.arange(4 * P, dtype=torch.float32, device="cuda")
    r.write_async("target", src.data_ptr(), src.numel() * 4, 0, 0)
    back = torch.zeros_like(src)
    r.read_async("target", back.data_ptr(), back.numel() * 4, 0, 0)
    r.check()
    assert np.array_equal(r.read("target", 4 * P), src.cpu().numpy())
    assert torch.equal(back, src)
    host = torch.full((4 * P,), 7.0).pin_memory()
    r.write_async("target", host.data_ptr(), host.numel() * 4, 0, 0)
    r.check()
    assert np.all(r.read("target", 4 * P) == 7.0)


def test_chosen_step_with_no_tile_entries():
    """Every surfel behind every camera: no tile entries, empty ranges, a
    black image, zero gradients, so the Adam step leaves the parameters as
    they were; nothing is reported as an error."""
    scene, cams = multi_view_setup(77, 200)
    rc = [raster_camera(c, 3) for c in cams]
    # The three cameras share a centre and look at the scene: move the scene
    # 50 units behind that centre, away from where they look.
    moved = scene.copy()
    c0 = np.asarray(cams[0].center, np.float64)
    away = (c0 - scene.pos.mean(0)) / np.linalg.norm(c0 - scene.pos.mean(0))
    moved.pos = c0 + 50.0 * away[None, :] + 0.01 * scene.pos
    r = _trainer(moved, cams)
    before = _params(r, moved.n)
    for _ in range(2):
        r.train_step(rc, moved.n, StepSettings(0.8, 0.2, AdamSettings(eps=1e-15), "chosen"))
    r.check()
    assert r.entry_count() == 0
    P = sum(c.width * c.height for c in cams)
    assert np.all(r.read("out_color", 4 * P) == 0)
    after = _params(r, moved.n)
    for k in before:
        assert np.array_equal(before[k], after[k]), k
