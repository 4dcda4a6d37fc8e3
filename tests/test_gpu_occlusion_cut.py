"""Occlusion cut of the chosen-form step against full tile lists.

With the cut, each tile is binned only down to the depth its pixels needed in
the previous step plus a margin, and a tile whose truncated list runs out
before all its pixels terminate is binned and rendered again in full within
the same step. The lists binned are then prefixes of the reference's
(tile, depth, entry) lists (crates/gs-kernels/src/binning.rs:5-8), and the
front-to-back walk (rasterize_fwd.wgsl:20-85) never reads past the last
entry a terminated pixel needed. So images, final transmittance and
contributor indices must equal those of full lists bit for bit, and
gradients must agree up to the order of float atomics. The tests compare a
handle with the cut against one built with GS_FLAG_FULL_LISTS on the same
scene and views: over steps that reuse the cuts, with cuts planted too
shallow so that the completion pass runs, after the views change, and over
training steps that move the scene."""
import numpy as np
import pytest

from splattar_b200 import AdamSettings, Rasterizer, StepSettings
from splattar_b200.synthetic import make_surfels, ring_cameras

pytestmark = pytest.mark.gpu

RES = [(320, 240), (256, 256), (200, 160)]
N = 120_000
MOMENTS = ("m_pos", "m_scales", "m_quat", "m_opacity", "m_sh")
WIDTH = {"m_pos": 4, "m_scales": 2, "m_quat": 4, "m_opacity": 1, "m_sh": 48}


def _pair(lr_zero: bool, tile: int = 16, extra_full: bool = False, big: bool = False):
    s = make_surfels(N, 7, True, 3, 0.1)
    t = make_surfels(N, 8, True, 3, 0.1)
    if big:  # 2 % of the surfels eight times larger: tile rects of more than 32 tiles
        s.scales[::50] *= 8.0
    cams = ring_cameras(RES)
    P = sum(w * h for w, h in RES)
    out = []
    for full in (False, True) + ((True,) if extra_full else ()):
        r = Rasterizer(N, 0, 0, N * len(RES) * 64, max_views=len(RES), max_pixels=P, precision="f16",
                       color_only=True, tile=tile, full_lists=full)
        r.upload_scene(t.scene_input())
        r.forward(cams, N)
        r.check()
        r.write("target", r.read("out_color", 4 * P))
        r.upload_scene(s.scene_input())
        r.optimizer_init(N)
        out.append(r)
    adam = AdamSettings(eps=1e-15)
    if lr_zero:
        adam.lr = {k: 0.0 for k in adam.lr}
    step = StepSettings(0.8, 0.2, adam, "chosen")
    if extra_full:
        return out[0], out[1], out[2], cams, P, step
    return out[0], out[1], cams, P, step


def _images(r, P):
    return (r.read("out_color", 4 * P), r.read("out_aux", 4 * P).reshape(P, 4)[:, 0].copy(),
            r.read("out_ncontrib", P))


def _same_step(a, b, P):
    ca, ta, na = _images(a, P)
    cb, tb, nb = _images(b, P)
    assert np.array_equal(ca, cb), f"colour differs on {int((ca != cb).sum())} values"
    assert np.array_equal(ta, tb)
    assert np.array_equal(na, nb)
    assert np.allclose(a.read("loss", 2 * len(RES)), b.read("loss", 2 * len(RES)), rtol=1e-12, atol=0)
    for k in MOMENTS:
        ma, mb = a.read(k, WIDTH[k] * N), b.read(k, WIDTH[k] * N)
        scale = max(float(np.abs(mb).max()), 1e-30)
        assert np.abs(ma - mb).max() <= 1e-4 * scale, k


@pytest.mark.parametrize("big", [False, True])
def test_reused_cuts_give_full_list_results(big):
    """Binning under the cut takes kept-tile bits for rects of up to 32 tiles
    and tests each tile for larger rects; `big` adds surfels whose rects are
    larger."""
    a, b, cams, P, step = _pair(lr_zero=True, big=big)
    for k in range(4):
        a.train_step(cams, N, step)
        b.train_step(cams, N, step)
        a.check(); b.check()
        _same_step(a, b, P)
        if k >= 1:  # the cuts of the step before are in use
            assert a.entry_count() < b.entry_count(), (a.entry_count(), b.entry_count())
    cut = a.read("tile_cut", 2048)
    assert (cut != 0xFFFFFFFF).any()


@pytest.mark.parametrize("tile", [16, 8])
def test_shallow_cuts_run_the_completion_pass(tile):
    a, b, cams, P, step = _pair(lr_zero=True, tile=tile)
    for r in (a, b):
        r.train_step(cams, N, step)
    a.check(); b.check()
    tiles = sum(((w + tile - 1) // tile) * ((h + tile - 1) // tile) for w, h in RES)
    cut = a.read("tile_cut", tiles)
    rng = np.random.default_rng(3)
    finite = np.flatnonzero(cut != 0xFFFFFFFF)
    assert finite.size > 20
    pick = rng.choice(finite, size=finite.size // 2, replace=False)
    planted = cut.copy()
    depth = planted[pick].view(np.float32) * np.float32(0.97)  # a little in front of the recorded cut
    planted[pick] = depth.view(np.uint32)
    planted[pick[: pick.size // 4]] = 0  # and some tiles binned empty
    a.write("tile_cut", planted)
    for r in (a, b):
        r.train_step(cams, N, step)
    a.check(); b.check()
    redone = int(a.read("incomplete_tiles", 1)[0])
    assert redone >= pick.size // 4, redone
    _same_step(a, b, P)
    # the next step starts from the completed tiles' new cuts
    for r in (a, b):
        r.train_step(cams, N, step)
    a.check(); b.check()
    _same_step(a, b, P)


def test_changed_views_start_from_full_lists():
    a, b, cams, P, step = _pair(lr_zero=True)
    for _ in range(2):
        for r in (a, b):
            r.train_step(cams, N, step)
    moved = ring_cameras(RES, radius=3.6)
    for r in (a, b):
        r.train_step(moved, N, step)
    a.check(); b.check()
    assert int(a.read("incomplete_tiles", 1)[0]) == 0
    assert a.entry_count() == b.entry_count()
    _same_step(a, b, P)


def test_training_with_the_cut_tracks_full_lists():
    """Five training steps: the cut handle stays as close to a full-list
    handle as a second full-list handle does. Float atomics make any two
    runs differ slightly, and Adam's normalised step turns the sign of a
    near-zero gradient into a full learning-rate step, so the yardstick is
    the spread between the two full-list runs (mean absolute difference).
    The cut changes which warps add an entry's gradient and in what order,
    not only when; the second full-list run therefore uses another backward
    launch shape, whose emission order differs in the same structural way."""
    a, b, c, cams, P, step = _pair(lr_zero=False, extra_full=True)
    c.set_launch_shapes(64, 4, 128, 8)
    for _ in range(5):
        for r in (a, b, c):
            r.train_step(cams, N, step)
        a.check(); b.check(); c.check()
    for k, w in (("raw_pos", 4), ("raw_scales", 2), ("raw_quat", 4), ("raw_opacity", 1), ("raw_sh", 48)):
        pa, pb, pc = a.read(k, w * N), b.read(k, w * N), c.read(k, w * N)
        d_cut, d_run = float(np.abs(pa - pb).mean()), float(np.abs(pc - pb).mean())
        assert d_cut <= 2.0 * d_run + 1e-7, (k, d_cut, d_run)
    la, lb = a.read("loss", 2 * len(RES)), b.read("loss", 2 * len(RES))
    assert np.allclose(la, lb, rtol=1e-5, atol=1e-6)


def test_cut_is_off_where_documented():
    for kw in (dict(deterministic=True), dict(full_lists=True), dict(stored_state=True, color_only=True)):
        r = Rasterizer(1000, 64, 64, **kw)
        with pytest.raises(Exception, match="GS_ERR_STATE"):
            r.read("incomplete_tiles", 1)


def test_chosen_forward_launch_shapes_agree():
    """The colour-only forward of the training step composites pixel pairs in
    packed FP32 (2, 4 and 8 pixels per thread), single pixels in scalar code
    (1 pixel per thread), or spreads each entry's box over a warp (the
    pixel-compacted kernel): every shape gives bit-identical colour, final T
    and contributor indices."""
    s = make_surfels(20_000, 11, True, 3, 0.1)
    cams = ring_cameras(RES)
    P = sum(w * h for w, h in RES)
    adam = AdamSettings(eps=1e-15)
    adam.lr = {k: 0.0 for k in adam.lr}
    step = StepSettings(0.8, 0.2, adam, "chosen")
    outs = []
    for fb, fp in [(64, 1), (128, 2), (64, 4), (64, 8), (32, 0)]:  # (32, 0): the pixel-compacted kernel
        r = Rasterizer(20_000, 0, 0, 20_000 * len(RES) * 64, max_views=len(RES), max_pixels=P, precision="f16",
                       color_only=True)
        r.upload_scene(s.scene_input())
        r.write("target", np.full(4 * P, 0.5, np.float32))
        r.optimizer_init(20_000)
        r.set_launch_shapes(fb, fp, 128, 8)
        r.train_step(cams, 20_000, step)
        r.check()
        outs.append(_images(r, P))
    for o in outs[1:]:
        for x, y in zip(outs[0], o):
            assert np.array_equal(x, y)
