"""The pixel-compacted raster kernels (launch shape (32, 0) on 16-pixel tiles):
one warp per tile, each entry's alpha-box pixels spread over the lanes. They
must give the training step exactly the images, final transmittance and
contributor indices of the thread-per-pixel kernels, the same gradients up to
the order of float sums, bitwise-repeatable results in deterministic mode,
and the occlusion cut's results (including the completion pass)."""
import numpy as np
import pytest

from splattar_b200 import AdamSettings, Rasterizer, StepSettings
from splattar_b200.synthetic import make_surfels, ring_cameras

pytestmark = pytest.mark.gpu

RES = [(320, 240), (200, 150), (256, 200)]  # partial tiles at the right and bottom edges
N = 40_000
PX = (32, 0, 32, 0)
THREAD = (64, 4, 64, 8)
CLASSES = (("pos", 4), ("scales", 2), ("quat", 4), ("opacity", 1), ("sh", 48))


def _handle(shapes, n=N, res=RES, **kw):
    s = make_surfels(n, 5, True, 3, 0.1)
    cams = ring_cameras(res)
    P = sum(w * h for w, h in res)
    r = Rasterizer(n, 0, 0, n * len(res) * 64, max_views=len(res), max_pixels=P, precision="f16", color_only=True,
                   **kw)
    r.upload_scene(s.scene_input())
    r.write("target", np.random.default_rng(9).uniform(0, 1, 4 * P).astype(np.float32))
    r.optimizer_init(n)
    r.set_launch_shapes(*shapes)
    return r, cams, P


def _out(r, P):
    return (r.read("out_color", 4 * P), r.read("out_aux", 4 * P).reshape(P, 4)[:, 0].copy(),
            r.read("out_ncontrib", P))


def _grads(r):
    """The gradient the first Adam step consumed: m = (1 - beta1) g."""
    k = float(np.float32(1.0) - np.float32(0.9))
    return {c: r.read("m_" + c, w * N).astype(np.float64) / k for c, w in CLASSES}


@pytest.mark.parametrize("loss", ["l1_ssim", "given"])
def test_px_kernels_match_thread_kernels(loss):
    outs = []
    for shapes in (THREAD, PX):
        r, cams, P = _handle(shapes, full_lists=True)
        if loss == "given":
            w = np.random.default_rng(4).uniform(-1, 1, (P, 4)).astype(np.float32)
            w[:, 3] = 0
            r.write("dl_dcolor", w.ravel())
        r.train_step(cams, N, StepSettings(0.8, 0.2, AdamSettings(eps=1e-15), "chosen", loss=loss))
        r.check()
        outs.append((_out(r, P), _grads(r), r.read("grad_cam", 16 * len(RES))))
        r.close()
    (ia, ga, ca), (ib, gb, cb) = outs
    for x, y in zip(ia, ib):
        assert np.array_equal(x, y)
    for c in ga:
        rel = np.linalg.norm(ga[c] - gb[c]) / max(np.linalg.norm(ga[c]), 1e-30)
        assert rel < 1e-5, (c, rel)
    assert np.abs(ca - cb).max() <= 1e-4 * np.abs(ca).max(), (np.abs(ca - cb).max(), np.abs(ca).max())


def test_px_kernels_deterministic_mode_repeats():
    outs = []
    for _ in range(2):
        r, cams, P = _handle(PX, deterministic=True)
        for _ in range(2):
            r.train_step(cams, N, StepSettings(0.8, 0.2, AdamSettings(eps=1e-15), "chosen"))
        r.check()
        outs.append({c: r.read("raw_" + c, w * N) for c, w in CLASSES} | {"cam": r.read("grad_cam", 16 * len(RES))})
        r.close()
    for k in outs[0]:
        assert np.array_equal(outs[0][k], outs[1][k]), k


def test_px_kernels_with_planted_cuts_equal_full_lists():
    # dense enough for most tiles to terminate (and so record a cut)
    n, res = 120_000, [(320, 240), (256, 256), (200, 160)]
    a, cams, P = _handle(PX, n, res)
    b, _, _ = _handle(PX, n, res, full_lists=True)
    adam = AdamSettings(eps=1e-15)
    adam.lr = {k: 0.0 for k in adam.lr}
    step = StepSettings(0.8, 0.2, adam, "chosen")
    for r in (a, b):
        r.train_step(cams, n, step)
    a.check(); b.check()
    n_tiles = sum(((w + 15) // 16) * ((h + 15) // 16) for w, h in res)
    cut = a.read("tile_cut", n_tiles)
    finite = np.flatnonzero(cut != 0xFFFFFFFF)
    assert finite.size > 20
    pick = np.random.default_rng(3).choice(finite, size=finite.size // 2, replace=False)
    planted = cut.copy()
    planted[pick] = (planted[pick].view(np.float32) * np.float32(0.97)).view(np.uint32)
    planted[pick[: pick.size // 4]] = 0  # binned empty: rendered entirely by the completion pass
    a.write("tile_cut", planted)
    for r in (a, b):
        r.train_step(cams, n, step)
    a.check(); b.check()
    assert int(a.read("incomplete_tiles", 1)[0]) >= pick.size // 4
    oa, ob = _out(a, P), _out(b, P)
    assert np.array_equal(oa[0], ob[0]) and np.array_equal(oa[1], ob[1])
    # contributor indices refer to each handle's own lists; the last contributor is the same surfel
    assert np.array_equal(oa[2] > 0, ob[2] > 0)
