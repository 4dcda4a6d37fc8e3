"""Tile sizes 8 and 32 beside the reference's 16 (crates/gs-kernels/src/
rasterizer.rs:13 fixes 16; the batched form's autotuner sweeps 8/16/32).
The oracle's rect arithmetic takes the tile size as a parameter, so every
parity check of the 16-pixel path is repeated per tile size: bit-exact tile
rects and depth keys, forward colour/α/T/depth/normal within the reference
tolerances with exact contributor counts off the marginal band, gradients
within 1e-5 + 2e-3·|g| (aux 6e-3, camera 3e-2), every launch shape of a tile
size bit-identical in the forward, and the chosen training step equal to the
plain one."""
import numpy as np
import pytest

import oracle
from gpu_util import GradCheck, backward, f32_cam, f32_scene, forward, raster_camera, scene_input
from scenes import XorShift, make_scene
from splattar_b200 import AdamSettings, Rasterizer, SceneInput, StepSettings
from splattar_b200.rasterizer import camera_rotation
from splattar_b200.synthetic import make_surfels, ring_cameras
from test_gpu_project_binning import gpu_rects_keys

pytestmark = pytest.mark.gpu

FWD_SHAPES = {8: [(64, 1), (128, 1), (256, 1), (64, 2), (128, 2), (256, 2)],
              16: [(64, 1), (128, 1), (256, 1), (64, 2), (128, 2), (64, 4), (64, 8), (128, 8)],
              32: [(64, 2), (128, 2), (256, 2), (64, 4), (128, 4), (256, 4), (128, 8)]}
BWD_SHAPES = {8: [(64, 1), (64, 2), (128, 2)], 16: [(64, 1), (64, 2), (128, 2), (64, 4), (32, 8), (64, 8), (128, 8)],
              32: [(64, 4), (64, 8)]}


def check_rects_keys(s: SceneInput, deg, cam, tile):
    n = s.positions.shape[0]
    rast = Rasterizer(n, cam.width, cam.height, n * 64 * max(1, (16 // tile) ** 2), tile=tile)
    assert rast.tile == tile
    rast.upload_scene(s)
    rast.forward(cam, n)
    rast.check()
    rects, keys, _, _ = gpu_rects_keys(rast, n)
    pos4 = np.concatenate([s.positions, np.ones((n, 1), np.float32)], axis=1)
    want_r, want_k, _ = oracle.project_f32(pos4, s.scales, s.quats, camera_rotation(cam), np.float32(cam.center),
                                           np.float32(cam.focal), cam.width, cam.height, tile=tile)
    assert np.array_equal(rects, want_r), f"tile {tile}: {int((rects != want_r).any(1).sum())} rects differ"
    assert np.array_equal(keys, want_k)


@pytest.mark.parametrize("tile", [8, 32])
def test_rects_and_keys_bit_exact(tile):
    for seed, n, deg, size in [(101, 20, 0, 64), (404, 2000, 1, 128)]:
        scene, cam = make_scene(seed, n, deg, size)
        check_rects_keys(scene_input(scene), deg, raster_camera(cam, deg), tile)
    s = make_surfels(30_000, 3, True, 3, 0.1)
    for cam in ring_cameras([(1920, 1080), (640, 480)]):
        check_rects_keys(s.scene_input(), 3, cam, tile)


@pytest.mark.parametrize("tile", [8, 32])
@pytest.mark.parametrize("seed,n,deg,size", [(101, 20, 0, 64), (303, 12, 3, 48), (404, 50, 1, 128)])
def test_forward_matches_cpu_oracle(tile, seed, n, deg, size):
    scene, cam = make_scene(seed, n, deg, size)
    cpu = oracle.render(f32_scene(scene), f32_cam(cam), tile=tile)
    _, gpu = forward(scene, cam, tile=tile)
    diff = np.abs(gpu["color"][:, :3] - cpu["color"])
    assert diff.max() < 3e-3 and diff.mean() < 3e-4, (diff.max(), diff.mean())
    assert np.abs(gpu["color"][:, 3] - cpu["alpha"]).max() < 3e-3
    assert np.abs(gpu["aux"][:, 0] - cpu["trans"]).max() < 3e-3
    assert np.abs(gpu["aux"][:, 1] - cpu["depth"]).max() < 3e-2
    assert np.abs(gpu["normal"][:, :3] - cpu["normal"]).max() < 3e-3
    mism = (gpu["ncontrib"].astype(np.int64) != cpu["ncontrib"]) & ~cpu["marginal"]
    assert not mism.any(), f"n_contrib differs on {int(mism.sum())} non-marginal pixels"


@pytest.mark.parametrize("tile", [8, 16, 32])
@pytest.mark.parametrize("persistent", [False, True])
def test_forward_launch_shapes_agree(tile, persistent):
    """Every built (batch, pixels per thread) of a tile size, including the
    multi-round staging of 8-pixel tiles (32 threads, batches up to 256)."""
    scene, cam = make_scene(404, 50, 1, 128)
    outs = []
    for batch, ppt in FWD_SHAPES[tile]:
        _, o = forward(scene, cam, tile=tile, batch=batch, pixels_per_thread=ppt, persistent=persistent)
        outs.append(o)
    for o in outs[1:]:
        for k in ("color", "aux", "normal", "ncontrib"):
            assert np.array_equal(outs[0][k], o[k]), k


def _weights(seed, P, aux):
    rng = XorShift(seed ^ 0xFEED)
    w = np.array([[rng.uniform(-1, 1) for _ in range(3)] for _ in range(P)])
    wd = np.array([rng.uniform(-0.3, 0.3) if aux else 0.0 for _ in range(P)])
    wn = np.array([[rng.uniform(-0.5, 0.5) for _ in range(3)] if aux else [0.0] * 3 for _ in range(P)])
    return w, wd, wn


def grad_parity(tile, seed, n, deg, size, aux=False, rel=2e-3, cam_rel=2e-3, bwd_shape=None, **kw):
    scene, cam = make_scene(seed, n, deg, size)
    P = size * size
    w, wd, wn = _weights(seed, P, aux)
    lam = 0.35 if aux else 0.0
    cpu = oracle.gradients(f32_scene(scene), f32_cam(cam), w, wd, wn, lam, tile=tile)
    rast, _ = forward(scene, cam, tile=tile, **kw)
    if bwd_shape is not None:
        rast.set_launch_shapes(*FWD_SHAPES[tile][0], *bwd_shape)
        rast.forward(raster_camera(cam, deg), n)
    rast.lambda_dist = lam
    g = backward(rast, scene, np.concatenate([w, wd[:, None]], axis=1),
                 np.concatenate([wn, np.zeros((P, 1))], axis=1))
    ck, cc = GradCheck(rel), GradCheck(cam_rel)
    ncoef = (deg + 1) ** 2
    for k in ("pos", "scales", "quat", "opacity"):
        ck.check(k, g[k], cpu[k])
    ck.check("sh", g["sh"][:, :3 * ncoef], cpu["sh"][:, :3 * ncoef])
    cc.check("dl_dR_cam", g["cam"][:9], cpu["dl_dr_cam"])
    cc.check("cam_center", g["cam"][9:12], cpu["cam_center"])
    cc.check("focal", g["cam"][12:13], [cpu["focal"]])
    return g


@pytest.mark.parametrize("tile", [8, 16, 32])
@pytest.mark.parametrize("seed,n,deg,size", [(111, 15, 0, 48), (333, 10, 3, 40)])
def test_backward_matches_cpu_oracle(tile, seed, n, deg, size):
    for shape in BWD_SHAPES[tile]:
        grad_parity(tile, seed, n, deg, size, bwd_shape=shape)


@pytest.mark.parametrize("tile", [8, 32])
def test_backward_aux_losses_match_cpu_oracle(tile):
    grad_parity(tile, 555, 12, 1, 40, aux=True, rel=6e-3, cam_rel=3e-2)


@pytest.mark.parametrize("tile", [8, 32])
def test_backward_deterministic_and_persistent(tile):
    grad_parity(tile, 222, 15, 1, 48, deterministic=True)
    grad_parity(tile, 222, 15, 1, 48, persistent=True)


def _multi_view(seed=21, n=400):
    scene, cam = make_scene(seed, n, 3, 64)
    cams = []
    for k, (w, h) in enumerate([(64, 64), (80, 48), (40, 72)]):
        c = cam.copy()
        c.width, c.height = w, h
        c.quat = np.array(cam.quat) + np.array([0.02 * k, -0.01 * k, 0.0, 0.0])
        cams.append(c)
    return scene, cams


@pytest.mark.parametrize("tile", [8, 32])
def test_chosen_step_matches_plain_step(tile):
    scene, cams = _multi_view()
    rc = [raster_camera(c, 3) for c in cams]
    P = sum(c.width * c.height for c in cams)
    tgt = np.random.default_rng(1).uniform(0, 1, (P, 4)).astype(np.float32)
    outs = []
    for form in ("plain", "chosen"):
        r = Rasterizer(scene.n, 0, 0, scene.n * 3 * 256, max_views=3, max_pixels=P, color_only=True, tile=tile)
        r.upload_scene(scene_input(scene))
        r.write("target", tgt.ravel())
        r.optimizer_init(scene.n)
        for _ in range(2):
            r.train_step(rc, scene.n, StepSettings(0.8, 0.2, AdamSettings(eps=1e-15), form))
        r.check()
        outs.append(({k: r.read(k, w * scene.n) for k, w in (("raw_pos", 4), ("raw_sh", 48))}, r.read("loss", 6)))
    (pa, la), (pb, lb) = outs
    assert np.allclose(la, lb, rtol=1e-5, atol=1e-6)
    for k in pa:
        assert np.abs(pa[k] - pb[k]).max() < 2e-4, k


def test_autotune_tiles_picks_a_built_configuration():
    scene, cams = _multi_view(66, 400)
    rc = [raster_camera(c, 3) for c in cams]
    P = sum(c.width * c.height for c in cams)
    r = Rasterizer(scene.n, 0, 0, scene.n * 3 * 256, max_views=3, max_pixels=P, color_only=True)
    r.upload_scene(scene_input(scene))
    r.optimizer_init(scene.n)
    r.forward(rc, scene.n)
    r.write("target", r.read("out_color", 4 * P))
    res = r.autotune_tiles(rc, scene.n)
    assert res["tile"] in (8, 16, 32) and r.tile == res["tile"]
    assert all(v is not None and v["fwd_ms"] > 0 and v["bwd_ms"] > 0 for v in res["per_tile"].values())
    shapes = FWD_SHAPES[res["tile"]]
    assert (res["fwd_batch"], res["fwd_pixels_per_thread"]) in shapes
    # the training step runs at the chosen tiling
    r.train_step(rc, scene.n, StepSettings(form="chosen"))
    r.check()


def test_tile_size_validation():
    with pytest.raises(Exception, match="GS_ERR_INVALID_ARG"):
        Rasterizer(100, 64, 64, tile=24)
    with pytest.raises(Exception, match="GS_ERR_INVALID_ARG"):
        Rasterizer(100, 64, 64, tile=32, batch=64, pixels_per_thread=1)
    with pytest.raises(Exception, match="GS_ERR_INVALID_ARG"):
        Rasterizer(100, 64, 64, tile=8, stored_state=True, color_only=True)
    r = Rasterizer(100, 64, 64)
    r.tile = 32
    assert r.tile == 32
    with pytest.raises(Exception, match="GS_ERR_INVALID_ARG"):
        r.set_launch_shapes(64, 1, 64, 1)
