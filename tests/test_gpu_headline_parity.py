"""Parity of the form the benchmark times, at the benchmark's workloads,
against the f64 oracle (the protocol of crates/gs-kernels/tests/raster_parity.rs:20-114,
scaled up).

ring8_1m (1,000,000 clustered surfels, SH degree 3, 8 ring views 640x480 ..
1920x1080): the chosen training step with f16 storage, tight binning,
persistent raster kernels, the graph-replayed step and the projection
backward fused with Adam, with the occlusion cut active (two L1+SSIM steps run
first, so each tile is binned only down to the depth its pixels needed).
The third step takes a linear loss sum w.colour whose weights are uniform in
[-1, 1] on every 64th tile of every view and zero elsewhere (and on pixels the
oracle marks marginal). Checked against the oracle at the parameters that step
started from:
  * the step's forward image (colour, alpha, final T) on the sampled pixels,
    3e-3 max / 3e-4 mean (raster_parity.rs:33-35);
  * the last contributor of every non-marginal sampled pixel, identified as a
    surfel through the step's own tile lists (the tight lists number entries
    differently from the reference's rects), exactly;
  * the gradient the fused Adam consumed, recovered from its first moments as
    g = (m_new - beta1 m_old) / (1 - beta1): relative L2 error per parameter
    class <= 1e-3 (the f16 target), and the per-view camera gradients within
    3e-2 (raster_parity.rs camera tolerance);
  * Adam itself, element by element from that gradient: v, raw and activated
    values (first_attempt/crates/gs-train/src/shaders/adam.wgsl:45-74).

small_1view_256 (16,384 surfels, 256x256, f = 256, eye (0, 0, -3)): the full
frame through the reference-exact binning (contributor counts exact on
non-marginal pixels), the 0.8 L1 + 0.2 (1 - SSIM) loss and its image gradient
against oracle.l1_ssim on the same image, and the parameter gradients of that
loss, through gs_rasterizer_backward and through one chosen training step."""
import numpy as np
import pytest

import oracle
from splattar_b200 import AdamSettings, Rasterizer, StepSettings
from splattar_b200.synthetic import workload

pytestmark = pytest.mark.gpu

STRIDE = 64
CLASSES = (("pos", "raw_pos", "m_pos", "v_pos", "positions", 4, 3), ("scales", "raw_scales", "m_scales", "v_scales",
           "scales", 2, 2), ("quat", "raw_quat", "m_quat", "v_quat", "quats", 4, 4),
           ("opacity", "raw_opacity", "m_opacity", "v_opacity", "opacities", 1, 1),
           ("sh", "raw_sh", "m_sh", "v_sh", "sh", 48, 48))
LR = {"pos": 1.6e-4, "scales": 5e-3, "quat": 1e-3, "opacity": 5e-2, "sh": 2.5e-3}


def _scene_of(r, n, sh_degree):
    f = lambda name, w: r.read(name, w * n).reshape(n, w).astype(np.float64)  # noqa: E731
    return oracle.Scene(f("positions", 4)[:, :3].copy(), f("scales", 2), f("quats", 4), f("opacities", 1)[:, 0].copy(),
                        f("sh", 48), sh_degree)


def _ocam(c):
    return oracle.Camera(np.array(c.center, np.float64), np.array(c.quat, np.float64), float(c.focal), c.width,
                         c.height)


def _state(r, n):
    out = {}
    for name, raw, m, v, act, w, _ in CLASSES:
        for key in (raw, m, v, act):
            out[key] = r.read(key, w * n).reshape(n, w)
    return out


def _bias(t, b1=np.float32(0.9), b2=np.float32(0.999)):
    p1 = p2 = np.float32(1.0)
    for _ in range(t):
        p1 = np.float32(p1 * b1)
        p2 = np.float32(p2 * b2)
    return float(np.float32(1.0) / np.float32(1.0 - p1)), float(np.float32(1.0) / np.float32(1.0 - p2))


def _last_surfel(off_tile, cam, n, view, nc, ranges, items, tile=16):
    """Surfel of each pixel's last contributor (-1 if none) from the step's own lists."""
    W, H = cam.width, cam.height
    tx = (W + tile - 1) // tile
    ys, xs = np.divmod(np.arange(W * H), W)
    t = off_tile + (ys // tile) * tx + xs // tile
    out = np.full(W * H, -1, np.int64)
    has = nc > 0
    e = ranges[t[has], 0].astype(np.int64) + nc[has].astype(np.int64) - 1
    assert (e < ranges[t[has], 1]).all(), "contributor index past its tile list"
    item = items[e, 1].astype(np.int64)
    out[has] = item - view * n
    return out


def test_chosen_step_ring8_1m_matches_oracle_on_sampled_tiles():
    wl = workload("ring8_1m")
    cams, n, P = wl.cameras, wl.surfels.n, wl.pixels
    nv = len(cams)
    # tight binning for the target render too (exact; the reference's rects
    # would need several times the entry budget at 8 views)
    r = Rasterizer(n, 0, 0, 24 * n * nv, max_views=nv, max_pixels=P, precision="f16", color_only=True, tight=True)
    r.upload_scene(wl.target_surfels.scene_input())
    r.forward(cams, n)
    r.check()
    r.write("target", r.read("out_color", 4 * P))
    r.upload_scene(wl.surfels.scene_input())
    r.optimizer_init(n)
    r.set_launch_shapes(64, 4, 64, 8)  # the shapes the autotuner keeps on this workload
    adam = AdamSettings(eps=1e-15)
    r.train_step(cams, n, StepSettings(0.8, 0.2, adam, "chosen"))
    r.check()
    full_entries = r.entry_count()  # the first step bins full lists
    r.train_step(cams, n, StepSettings(0.8, 0.2, adam, "chosen"))
    r.check()
    scene = _scene_of(r, n, 3)
    before = _state(r, n)

    # The oracle at the parameters the third step starts from, on every 64th
    # tile of every view (a different offset per view).
    ref, w_all = [], np.zeros((P, 4), np.float32)
    for v, c in enumerate(cams):
        off, _ = r.view_offset(v)
        o = oracle.render(scene, _ocam(c), tile_stride=STRIDE, tile_offset=(7 * v) % STRIDE)
        Pv = c.width * c.height
        keep = o["sampled"] & ~o["marginal"]
        w = np.random.default_rng(300 + v).uniform(-1, 1, (Pv, 3))
        w[~keep] = 0.0
        w_all[off:off + Pv, :3] = w
        ref.append((o, keep, w))
    r.write("dl_dcolor", w_all.ravel())
    r.train_step(cams, n, StepSettings(0.8, 0.2, adam, "chosen", loss="given"))
    r.check()
    cut_entries = r.entry_count()
    assert cut_entries < full_entries // 2, (cut_entries, full_entries)  # the occlusion cut is active
    print(f"tile entries: {full_entries} full lists, {cut_entries} after the cut, "
          f"{int(r.read('incomplete_tiles', 1)[0])} tiles completed in full")
    after = _state(r, n)
    img = r.read("out_color", 4 * P).reshape(P, 4)
    trans = r.read("out_aux", 4 * P).reshape(P, 4)[:, 0]
    nc_all = r.read("out_ncontrib", P)
    n_tiles = sum(((c.width + 15) // 16) * ((c.height + 15) // 16) for c in cams)
    ranges = r.read("ranges", 2 * n_tiles).reshape(n_tiles, 2)
    items = r.read("sorted_items", 2 * int(ranges[:, 1].max())).reshape(-1, 2)
    grad_cam = r.read("grad_cam", 16 * nv).reshape(nv, 16)
    r.close()

    # Forward image and contributor identity.
    errs, worst, mismatched, compared = [], 0.0, 0, 0
    for v, c in enumerate(cams):
        off = sum(cc.width * cc.height for cc in cams[:v])
        toff = sum(((cc.width + 15) // 16) * ((cc.height + 15) // 16) for cc in cams[:v])
        o, keep, _ = ref[v]
        Pv = c.width * c.height
        e = np.abs(img[off:off + Pv, :3][keep] - o["color"][keep])
        ea = np.abs(img[off:off + Pv, 3][keep] - o["alpha"][keep])
        et = np.abs(trans[off:off + Pv][keep] - o["trans"][keep])
        errs.append(e.ravel())
        worst = max(worst, float(e.max(initial=0)), float(ea.max(initial=0)), float(et.max(initial=0)))
        last = _last_surfel(toff, c, n, v, nc_all[off:off + Pv], ranges, items)
        mismatched += int((last[keep] != o["last"][keep]).sum())
        compared += int(keep.sum())
    allerr = np.concatenate(errs)
    assert compared > 50_000, compared
    assert worst < 3e-3 and allerr.mean() < 3e-4, (worst, float(allerr.mean()))
    assert mismatched == 0, f"{mismatched} of {compared} pixels with a different last contributor"

    # The gradient the fused Adam consumed, against the oracle's.
    b1, b2 = np.float32(0.9), np.float32(0.999)
    gref = {k: 0.0 for k, *_ in CLASSES}
    cam_ref = np.zeros((nv, 13))
    for v, c in enumerate(cams):
        o, keep, w = ref[v]
        g = oracle.gradients(scene, _ocam(c), w, tile_stride=STRIDE, tile_offset=(7 * v) % STRIDE)
        for k, *_ in CLASSES:
            gref[k] = gref[k] + g[k].reshape(n, -1)
        cam_ref[v, :9] = g["dl_dr_cam"]
        cam_ref[v, 9:12] = g["cam_center"]
        cam_ref[v, 12] = g["focal"]
    bc1, bc2 = _bias(3)
    report = {}
    for name, raw, m, v_, act, width, used in CLASSES:
        m0, m1 = before[m].astype(np.float64), after[m].astype(np.float64)
        g_rec = (m1 - float(b1) * m0) / float(np.float32(1.0) - b1)
        # oracle gradient with respect to the raw (optimizer) parameters
        a0 = before[act].astype(np.float64)
        gr = np.zeros_like(g_rec)
        gr[:, :used] = gref[name]
        if name == "scales":
            gr = gr * a0
        if name == "opacity":
            gr = gr * a0 * (1 - a0)
        rel = float(np.linalg.norm(g_rec[:, :used] - gr[:, :used]) / np.linalg.norm(gr[:, :used]))
        report[name] = rel
        # Adam from the recovered gradient, element by element.
        v0, v1 = before[v_].astype(np.float64), after[v_].astype(np.float64)
        v_exp = float(b2) * v0 + float(np.float32(1.0) - b2) * g_rec * g_rec
        assert np.all(np.abs(v1 - v_exp) <= 1e-5 * np.abs(v_exp) + 1e-30), name
        r0, r1 = before[raw].astype(np.float64), after[raw].astype(np.float64)
        step = LR[name] * (m1 * bc1) / (np.sqrt(v1 * bc2) + 1e-15)
        ulp = np.spacing(np.abs(after[raw]).astype(np.float32)).astype(np.float64)
        assert np.all(np.abs(r1 - (r0 - step)) <= 1e-5 * np.abs(step) + ulp), name
        act1 = after[act].astype(np.float64)
        want = np.exp(r1) if name == "scales" else (1 / (1 + np.exp(-r1)) if name == "opacity" else r1)
        if name == "pos":
            act1, want = act1[:, :3], want[:, :3]
        assert np.allclose(act1, want, rtol=4e-6, atol=0), name
    print("headline gradient rel L2", {k: f"{e:.2e}" for k, e in report.items()})
    for k, e in report.items():
        assert e <= 1e-3, (k, e)
    cam_err = np.abs(grad_cam[:, :13] - cam_ref)
    assert np.all(cam_err <= 1e-5 + 3e-2 * np.abs(cam_ref).max(axis=1, keepdims=True)), cam_err.max()


def test_config0_full_frame_l1_ssim_matches_oracle():
    wl = workload("small_1view_256")
    c = wl.cameras[0]
    n, P = wl.surfels.n, c.width * c.height
    cam = _ocam(c)
    r = Rasterizer(n, c.width, c.height)
    r.upload_scene(wl.target_surfels.scene_input())
    r.forward(c, n)
    r.check()
    target = r.read("out_color", 4 * P).reshape(P, 4)
    r.write("target", target.ravel())
    r.upload_scene(wl.surfels.scene_input())
    scene = _scene_of(r, n, 0)
    # Full frame, reference-exact binning: colour and contributor counts.
    r.forward(c, n)
    r.check()
    img = r.read("out_color", 4 * P).reshape(P, 4)
    nc = r.read("out_ncontrib", P)
    ref = oracle.render(scene, cam)
    keep = ~ref["marginal"]
    e = np.abs(img[:, :3] - ref["color"])
    assert e.max() < 3e-3 and e.mean() < 3e-4, (float(e.max()), float(e.mean()))
    assert np.array_equal(nc[keep], ref["ncontrib"][keep])
    # L1+SSIM on the GPU image: loss sums and image gradient.
    r.loss_l1_ssim(0.8, 0.2)
    r.check()
    dl = r.read("dl_dcolor", 4 * P).reshape(P, 4)
    sums = r.read("loss", 2)
    loss_o, dl_o, l1_o, ss_o = oracle.l1_ssim(img.astype(np.float64), target.astype(np.float64), c.width, c.height)
    assert abs(sums[0] - l1_o) <= 1e-5 * abs(l1_o) and abs(sums[1] - ss_o) <= 1e-5 * abs(ss_o), (sums, l1_o, ss_o)
    scale = np.abs(dl_o[:, :3]).max()
    assert np.abs(dl[:, :3] - dl_o[:, :3]).max() <= 2e-4 * scale
    # Gradients of that loss through the backward, against the oracle's with
    # the same image gradient (marginal pixels carry none).
    r.write("dl_dnormal", np.zeros(4 * P, np.float32))
    dl64 = dl[:, :3].astype(np.float64)
    dl64[~keep] = 0.0
    r.write("dl_dcolor", np.concatenate([dl64, np.zeros((P, 1))], 1).astype(np.float32).ravel())
    r.backward(n)
    r.check()
    g_gpu = {k: r.read(b, w * n).reshape(n, w)[:, :u] for k, b, w, u in
             (("pos", "grad_pos", 4, 3), ("scales", "grad_scales", 2, 2), ("quat", "grad_quat", 4, 4),
              ("opacity", "grad_opacity", 1, 1), ("sh", "grad_sh", 48, 3))}
    g_ref = oracle.gradients(scene, cam, dl64)
    for k in g_gpu:
        gr = g_ref[k].reshape(n, -1)[:, :g_gpu[k].shape[1]]
        rel = float(np.linalg.norm(g_gpu[k] - gr) / np.linalg.norm(gr))
        assert rel <= 1e-3, (k, rel)

    # One chosen training step: the gradient its fused Adam consumed (from the
    # first moments of the first step, m = (1 - beta1) g) against the oracle's
    # gradient of L1+SSIM of the step's own image. optimizer_init re-derives
    # the activated values through raw space (log/exp, logit/sigmoid), so the
    # step's parameters are read after it.
    r.close()
    r = Rasterizer(n, c.width, c.height, precision="f32", color_only=True)
    r.upload_scene(wl.surfels.scene_input())
    r.write("target", target.ravel())
    r.optimizer_init(n)
    scene = _scene_of(r, n, 0)
    a0 = {k: r.read(k, w * n).reshape(n, w).astype(np.float64) for k, w in (("scales", 2), ("opacities", 1))}
    r.forward(c, n)
    r.check()
    img1 = r.read("out_color", 4 * P).reshape(P, 4)
    r.train_step([c], n, StepSettings(0.8, 0.2, AdamSettings(eps=1e-15), "chosen"))
    r.check()
    img2 = r.read("out_color", 4 * P).reshape(P, 4)
    assert np.array_equal(img2[:, :3], img1[:, :3])  # same parameters, same image (tight binning is exact)
    g_rec = {k: r.read("m_" + k, w * n).reshape(n, w).astype(np.float64) / float(np.float32(1.0) - np.float32(0.9))
             for k, w in (("pos", 4), ("scales", 2), ("quat", 4), ("opacity", 1), ("sh", 48))}
    r.close()
    _, dl_img, _, _ = oracle.l1_ssim(img2.astype(np.float64), target.astype(np.float64), c.width, c.height)
    dlo = dl_img[:, :3].copy()
    g_ref = oracle.gradients(scene, cam, dlo)
    want = {"pos": g_ref["pos"], "scales": g_ref["scales"] * a0["scales"], "quat": g_ref["quat"],
            "opacity": g_ref["opacity"].reshape(n, 1) * a0["opacities"] * (1 - a0["opacities"]),
            "sh": g_ref["sh"][:, :3]}
    for k, wv in want.items():
        got = g_rec[k][:, :wv.shape[1]]
        rel = float(np.linalg.norm(got - wv) / np.linalg.norm(wv))
        assert rel <= 2e-3, (k, rel)
