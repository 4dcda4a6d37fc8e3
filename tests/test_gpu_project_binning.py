"""Bit-exact integer parts of the path: tile rects and depth keys of the
projection against the f32 restatement of surfel_prep_fwd.wgsl; the binner,
radix sort and scan against CPU references on the reference's test shapes
(crates/gs-kernels/tests/binning.rs:37-158, crates/gs-wgpu/tests/sort.rs:27-113,
crates/gs-wgpu/tests/prefix_sum.rs:57-73)."""
import numpy as np
import pytest

import oracle
from gpu_util import f32_cam, f32_scene, forward, raster_camera, scene_input
from scenes import make_scene
from splattar_b200 import Rasterizer, TileBinner, camera_rotation, exclusive_scan_u32, radix_sort_pairs
from splattar_b200.synthetic import make_surfels, ring_cameras

pytestmark = pytest.mark.gpu


def gpu_rects_keys(rast, n_items):
    rects = rast.read("rects", 4 * n_items).reshape(n_items, 4)
    sk = rast.read("depth_keys", n_items)
    order = rast.read("depth_order", n_items)
    keys = np.zeros(n_items, np.uint32)
    keys[order] = sk
    return rects, keys, sk, order


def check_project_exact(pos, scales, quats, opac, sh, deg, cam):
    n = pos.shape[0]
    from splattar_b200 import SceneInput
    rast = Rasterizer(n, cam.width, cam.height, n * 64)
    rast.upload_scene(SceneInput(pos, scales, quats, opac, sh, (deg + 1) ** 2))
    rast.forward(cam, n)
    rast.check()
    rects, keys, sk, order = gpu_rects_keys(rast, n)
    rot = camera_rotation(cam)
    pos4 = np.concatenate([pos, np.ones((n, 1), np.float32)], axis=1)
    want_r, want_k, _ = oracle.project_f32(pos4, scales, quats, rot, np.float32(cam.center), np.float32(cam.focal),
                                           cam.width, cam.height)
    assert np.array_equal(rects, want_r), f"{int((rects != want_r).any(1).sum())} rects differ"
    assert np.array_equal(keys, want_k), f"{int((keys != want_k).sum())} depth keys differ"
    # The depth order is the stable sort by key, ties by index.
    assert np.array_equal(order, np.argsort(want_k, kind="stable").astype(np.uint32))
    return rast, rects


@pytest.mark.parametrize("seed,n,deg,size", [(101, 20, 0, 64), (202, 200, 1, 64), (303, 500, 3, 48), (404, 2000, 1, 128)])
def test_rects_and_keys_bit_exact_micro(seed, n, deg, size):
    scene, cam = make_scene(seed, n, deg, size)
    si = scene_input(scene)
    check_project_exact(si.positions, si.scales, si.quats, si.opacities, si.sh, deg, raster_camera(cam, deg))
    # and the f64 oracle's rects agree except where it flags a truncation as marginal
    r64, k64, marg, _ = oracle.project(f32_scene(scene), f32_cam(cam))


def test_rects_and_keys_bit_exact_ring_views():
    s = make_surfels(60_000, 3, True, 3, 0.1)
    for cam in ring_cameras([(1920, 1080), (640, 480), (1280, 720)]):
        check_project_exact(s.positions, s.scales, s.quats, s.opacities, s.sh, 3, cam)


def test_rects_agree_with_f64_oracle_except_marginal():
    scene, cam = make_scene(404, 2000, 1, 128)
    rast, gpu = forward(scene, cam)
    rects = rast.read("rects", 4 * scene.n).reshape(scene.n, 4).astype(np.int64)
    r64, k64, marg, _ = oracle.project(f32_scene(scene), f32_cam(cam))
    diff = (rects != r64).any(1) & ~marg
    assert not diff.any(), f"{int(diff.sum())} non-marginal rects differ from the f64 oracle"


# ----------------------------------------------------------------- binner
def cpu_binning(rects, depths, tiles_x, num_tiles):
    entries = []
    for i, (x0, y0, x1, y1) in enumerate(rects):
        if x1 < x0 or y1 < y0:
            continue
        for ty in range(y0, y1 + 1):
            for tx in range(x0, x1 + 1):
                entries.append((ty * tiles_x + tx, int(depths[i]), len(entries), i))
    exp = sorted(entries, key=lambda e: (e[0], e[1], e[2]))
    ranges = np.zeros((num_tiles, 2), np.uint32)
    for k, e in enumerate(exp):
        if k == 0 or exp[k - 1][0] != e[0]:
            ranges[e[0], 0] = k
        ranges[e[0], 1] = k + 1
    items = np.zeros(len(entries), np.uint32)
    for e in entries:
        items[e[2]] = e[3]
    return np.array([e[2] for e in exp], np.uint32), ranges, items


def run_binning_case(rects, depths, tiles_x=64, tiles_y=64):
    import torch
    rects = np.asarray(rects, np.uint32).reshape(-1, 4)
    depths = np.asarray(depths, np.uint32)
    want, want_ranges, want_items = cpu_binning(rects, depths, tiles_x, tiles_x * tiles_y)
    total = len(want)
    b = TileBinner(max(len(rects), 1), max(total, 1), tiles_x * tiles_y)
    tr = torch.from_numpy(rects.view(np.int32).copy()).cuda()
    td = torch.from_numpy(depths.view(np.int32).copy()).cuda()
    b.encode(tr.data_ptr(), td.data_ptr(), len(rects), tiles_x)
    torch.cuda.synchronize()

    def read(which, count, dt):
        p, nbytes = b.buffer(which)
        return dev_to_host(p, count, dt)

    cnt = read("entry_count", 1, np.uint64)[0]
    assert cnt == total
    if total == 0:
        return
    got = read("sorted_entries", total, np.uint32)
    assert np.array_equal(got, want), f"payload mismatch at {int(np.argmax(got != want))}"
    ranges = read("ranges", 2 * tiles_x * tiles_y, np.uint32).reshape(-1, 2)
    assert np.array_equal(ranges, want_ranges)
    items = read("entry_items", total, np.uint32)
    assert np.array_equal(items, want_items)


def dev_to_host(dev_ptr: int, count: int, dtype) -> np.ndarray:
    """Device → host copy of a library buffer through torch (plumbing only)."""
    import torch
    nbytes = count * np.dtype(dtype).itemsize

    class _Iface:
        __cuda_array_interface__ = {"shape": (nbytes,), "typestr": "|u1", "data": (dev_ptr, False), "version": 2}
    t = torch.as_tensor(_Iface(), device="cuda")
    return t.cpu().numpy().view(dtype).copy()


def xorshift32(state):
    x = state
    x ^= (x << 13) & 0xFFFFFFFF
    x ^= x >> 17
    x ^= (x << 5) & 0xFFFFFFFF
    return x


@pytest.mark.parametrize("num_items,seed", [(1, 7), (100, 11), (5000, 13), (100_000, 17)])
def test_binning_matches_cpu_reference(num_items, seed):
    rng = seed
    rects, depths = [], []
    for _ in range(num_items):
        rng = xorshift32(rng); x0 = rng % 64
        rng = xorshift32(rng); y0 = rng % 64
        rng = xorshift32(rng); w = rng % 4
        rng = xorshift32(rng); h = rng % 4
        rects.append([x0, y0, min(x0 + w, 63), min(y0 + h, 63)])
        rng = xorshift32(rng); depths.append(rng % 32)
    run_binning_case(rects, depths)


def test_binning_degenerate_cases():
    run_binning_case([[5, 5, 4, 4]], [1])                                 # culled item
    run_binning_case([[10, 10, 10, 10]] * 500, [i % 3 for i in range(500)])  # all in one tile


# ------------------------------------------------------------ sort / scan
def dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).cuda()


@pytest.mark.parametrize("n", [0, 1, 255, 256, 1024, 4097, 100_000, 1_000_003, 2_000_000, 4_194_304, 10_000_000])
def test_sorts_match_cpu_stable_sort(n):
    import torch
    rng = np.random.default_rng(n)
    keys = (rng.integers(0, 2**32, n, dtype=np.uint64) % 8192).astype(np.uint32)
    vals = np.arange(n, dtype=np.uint32)
    tk, tv = dev(keys), dev(vals)
    radix_sort_pairs(tk.data_ptr(), tv.data_ptr(), n, 32)
    torch.cuda.synchronize()
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(tk.cpu().numpy().view(np.uint32), keys[order])
    assert np.array_equal(tv.cpu().numpy().view(np.uint32), vals[order])


def test_full_range_keys_sort():
    import torch
    n = 65_537
    keys = np.random.default_rng(1).integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
    tk, tv = dev(keys), dev(np.arange(n, dtype=np.uint32))
    radix_sort_pairs(tk.data_ptr(), tv.data_ptr(), n, 32)
    torch.cuda.synchronize()
    assert np.array_equal(tk.cpu().numpy().view(np.uint32), np.sort(keys))


@pytest.mark.parametrize("data", ["rand"] + ["zeros", "ones", "single"])
def test_exclusive_scan_matches_cpu(data):
    import torch
    cases = []
    if data == "rand":
        for n in [1, 2, 255, 1024, 1025, 4096, 100_003, 1_048_576, 10_000_000]:
            cases.append((np.random.default_rng(n).integers(0, 16, n)).astype(np.uint32))
    elif data == "zeros":
        cases.append(np.zeros(4096, np.uint32))
    elif data == "ones":
        cases.append(np.ones(2049, np.uint32))
    else:
        cases.append(np.array([42], np.uint32))
    for inp in cases:
        n = inp.size
        ti, to, tt = dev(inp), dev(np.zeros(n, np.uint32)), dev(np.zeros(1, np.uint32))
        exclusive_scan_u32(ti.data_ptr(), to.data_ptr(), n, tt.data_ptr())
        torch.cuda.synchronize()
        exp = np.concatenate([[0], np.cumsum(inp, dtype=np.uint64)[:-1]]).astype(np.uint32)
        assert np.array_equal(to.cpu().numpy().view(np.uint32), exp), n
        assert int(tt.cpu().numpy().view(np.uint32)[0]) == int(inp.sum())


def test_entry_capacity_overflow_is_reported_not_written():
    """max_entries below the real entry count: the forward must flag
    GS_ERR_CAPACITY and write nothing out of bounds."""
    from splattar_b200 import GsError
    scene, cam = make_scene(404, 50, 1, 128)
    rast = Rasterizer(scene.n, 128, 128, 8)
    rast.upload_scene(scene_input(scene))
    rast.forward(raster_camera(cam, 1), scene.n)
    with pytest.raises(GsError, match="GS_ERR_CAPACITY"):
        rast.check()


@pytest.mark.parametrize("tight,tile", [(False, 16), (True, 16), (True, 8), (False, 32)])
def test_rasterizer_tile_ranges_match_sorted_entries(tight, tile):
    """The tile sort's final pass records each tile's [start, end) in the
    sorted entry list (empty tiles (0, 0)); the result equals the ranges read
    off the sorted keys on the host."""
    s = make_surfels(20_000, 5, True, 1, 0.1)
    cams = ring_cameras([(640, 480), (320, 200)])
    P = sum(c.width * c.height for c in cams)
    r = Rasterizer(s.n, 0, 0, 300 * s.n, max_views=2, max_pixels=P, tight=tight, tile=tile)
    r.upload_scene(s.scene_input())
    r.forward(cams, s.n)
    r.check()
    E = r.entry_count()
    keys = r.read("sorted_items", 2 * E).reshape(E, 2)[:, 0].astype(np.int64)
    assert np.all(np.diff(keys) >= 0)
    tiles = sum(((c.width + tile - 1) // tile) * ((c.height + tile - 1) // tile) for c in cams)
    want = np.zeros((tiles, 2), np.int64)
    present = np.unique(keys)
    want[present, 0] = np.searchsorted(keys, present, side="left")
    want[present, 1] = np.searchsorted(keys, present, side="right")
    got = r.read("ranges", 2 * tiles).reshape(tiles, 2).astype(np.int64)
    assert np.array_equal(got, want)
