"""Host-side mirror of the reference's rasterizer surface over the C ABI.

Names and argument meanings follow the reference's public items:
``Rasterizer`` (crates/gs-kernels/src/rasterizer.rs:56-449), ``RasterCamera``
(:34-41), ``SceneInput`` (:44-54), ``TileBinner`` (crates/gs-kernels/src/
binning.rs:22-238), ``SsimLoss`` (first_attempt/crates/gs-train/src/ssim.rs)
and ``Optimizer`` (first_attempt/crates/gs-train/src/optim.rs). The reference
records into a wgpu command encoder; here every call is stream-ordered on a
CUDA stream (``stream`` = a ``cudaStream_t`` as an int, 0 = default stream).
Where the reference panics on a violated assert, these raise ``GsError``.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

from ._lib import (BUF, FLAG_COLOR_ONLY, FLAG_DETERMINISTIC, FLAG_FULL_LISTS, FLAG_PERSISTENT, FLAG_STORED_STATE,
                   FLAG_TIGHT_BINNING, PREC,
                   AdamConfig, Camera,
                   DensifyConfig, GsError, McmcConfig, RasterConfig, SceneInputC, StepConfig, check, lib)

SH_FLOATS = 48
TILE = 16


@dataclass
class RasterCamera:
    """Camera-to-world pose (``quat`` xyzw, normalised on upload), single focal
    length in pixels, principal point at the image centre."""
    center: tuple
    quat: tuple
    focal: float
    sh_degree: int
    width: int
    height: int

    def c(self) -> Camera:
        cam = Camera()
        for k in range(4):
            cam.quat[k] = float(self.quat[k])
        for k in range(3):
            cam.center[k] = float(self.center[k])
        cam.focal = float(self.focal)
        cam.width = int(self.width)
        cam.height = int(self.height)
        cam.sh_degree = int(self.sh_degree)
        return cam


def camera_array(cams) -> C.Array:
    if isinstance(cams, RasterCamera):
        cams = [cams]
    arr = (Camera * len(cams))()
    for k, c in enumerate(cams):
        arr[k] = c.c()
    return arr


def camera_rotation(cam: RasterCamera) -> np.ndarray:
    """Column-major camera-to-world rotation exactly as the forward builds it."""
    out = (C.c_float * 9)()
    c = cam.c()
    check(lib().gs_camera_rotation(C.byref(c), out))
    return np.array(out[:], np.float32)


@dataclass
class SceneInput:
    """Activated parameters, host arrays (float32)."""
    positions: np.ndarray  # (n,3)
    scales: np.ndarray     # (n,2)
    quats: np.ndarray      # (n,4) xyzw
    opacities: np.ndarray  # (n,)
    sh: np.ndarray         # (n, sh_coeffs*3) coefficient-major rgb
    sh_coeffs: int
    _keep: list = field(default_factory=list, repr=False)

    def c(self) -> SceneInputC:
        arrs = [np.ascontiguousarray(a, np.float32) for a in
                (self.positions, self.scales, self.quats, self.opacities, self.sh)]
        self._keep = arrs
        n = arrs[0].shape[0]
        if not (arrs[1].shape == (n, 2) and arrs[2].shape == (n, 4) and arrs[3].shape == (n,)
                and arrs[4].size == n * self.sh_coeffs * 3):
            raise GsError(1, "SceneInput arrays disagree in length")
        return SceneInputC(*[a.ctypes.data for a in arrs], self.sh_coeffs, n)


_DTYPES = {
    "out_ncontrib": np.uint32, "ranges": np.uint32, "sorted_items": np.uint32, "entry_count": np.uint64,
    "loss": np.float64, "rects": np.uint32, "depth_keys": np.uint32, "depth_order": np.uint32,
    "normal_loss": np.float64, "incomplete_tiles": np.uint32, "tile_cut": np.uint32,
}


class Rasterizer:
    """Rasterizer::new(ctx, capacity, width, height, max_entries), plus the
    batched-view and precision options of this build."""

    def __init__(self, capacity: int, width: int, height: int, max_entries: int = 0, *, max_views: int = 1,
                 max_pixels: int = 0, precision: str = "f32", deterministic: bool = False,
                 persistent: bool = False, color_only: bool = False, tight: bool = False, batch: int = 128,
                 pixels_per_thread: int = 0, stored_state: bool = False, tile: int = 16, full_lists: bool = False):
        self._h = None
        flags = (FLAG_DETERMINISTIC if deterministic else 0) | (FLAG_PERSISTENT if persistent else 0) | (
            FLAG_COLOR_ONLY if color_only else 0) | (FLAG_TIGHT_BINNING if tight else 0) | (
            FLAG_STORED_STATE if stored_state else 0) | (FLAG_FULL_LISTS if full_lists else 0)
        cfg = RasterConfig(capacity, width, height, max_views, max_pixels, max_entries, tile, batch, PREC[precision],
                           flags, pixels_per_thread)
        h = C.c_void_p()
        check(lib().gs_rasterizer_create(C.byref(cfg), C.byref(h)))
        self._h = h
        self.capacity, self.width, self.height = capacity, width, height
        self._lambda_dist = 0.0
        self.cams = None

    def close(self):
        if self._h:
            lib().gs_rasterizer_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _chk(self, status):
        check(status, self._h)

    @property
    def handle(self):
        return self._h

    @property
    def lambda_dist(self) -> float:
        return self._lambda_dist

    @lambda_dist.setter
    def lambda_dist(self, v: float):
        self._lambda_dist = float(v)
        self._chk(lib().gs_rasterizer_set_lambda_dist(self._h, float(v)))

    def set_wait_limits(self, copy_wait_cycles: int, drain_wait_cycles: int = 2_000_000_000):
        """Limits (SM cycles) of the fused projection backward + Adam kernel's bounded waits."""
        self._chk(lib().gs_rasterizer_set_wait_limits(self._h, copy_wait_cycles, drain_wait_cycles))

    def upload_scene(self, scene: SceneInput, stream: int = 0):
        s = scene.c()
        self._chk(lib().gs_rasterizer_upload_scene(self._h, C.byref(s), stream))

    def forward(self, cameras, num_surfels: int, stream: int = 0):
        self.cams = camera_array(cameras)
        self._chk(lib().gs_rasterizer_forward(self._h, self.cams, len(self.cams), num_surfels, stream))

    def backward(self, num_surfels: int, stream: int = 0):
        self._chk(lib().gs_rasterizer_backward(self._h, num_surfels, stream))

    def check(self, stream: int = 0):
        """Synchronise and raise on a sticky device error (entry capacity, timeouts)."""
        self._chk(lib().gs_rasterizer_check(self._h, stream))

    def buffer(self, name: str):
        p, n = C.c_void_p(), C.c_size_t()
        self._chk(lib().gs_rasterizer_buffer(self._h, BUF[name], C.byref(p), C.byref(n)))
        return p.value, n.value

    def view_offset(self, view: int):
        po, to = C.c_uint64(), C.c_uint32()
        self._chk(lib().gs_rasterizer_view_offset(self._h, view, C.byref(po), C.byref(to)))
        return po.value, to.value

    def read(self, name: str, count: int, dtype=None, offset: int = 0, stream: int = 0) -> np.ndarray:
        """Blocking readback of ``count`` elements (buffers::readback)."""
        dt = np.dtype(dtype or _DTYPES.get(name, np.float32))
        out = np.empty(count, dt)
        self._chk(lib().gs_rasterizer_read(self._h, BUF[name], offset * dt.itemsize, out.ctypes.data, out.nbytes,
                                           stream))
        return out

    def write(self, name: str, array: np.ndarray, offset_elems: int = 0, stream: int = 0):
        """Blocking upload (queue.write_buffer)."""
        a = np.ascontiguousarray(array)
        self._chk(lib().gs_rasterizer_write(self._h, BUF[name], offset_elems * a.dtype.itemsize, a.ctypes.data,
                                            a.nbytes, stream))

    def read_async(self, name: str, host_ptr: int, nbytes: int, offset_bytes: int = 0, stream: int = 0):
        self._chk(lib().gs_rasterizer_read_async(self._h, BUF[name], offset_bytes, host_ptr, nbytes, stream))

    def write_async(self, name: str, host_ptr: int, nbytes: int, offset_bytes: int = 0, stream: int = 0):
        self._chk(lib().gs_rasterizer_write_async(self._h, BUF[name], offset_bytes, host_ptr, nbytes, stream))

    def raster_work(self, stream: int = 0) -> dict:
        """Work of the raster kernels on the last forward, counted on the device."""
        out = (C.c_uint64 * 4)()
        self._chk(lib().gs_raster_work(self._h, out, stream))
        return {"fwd_evals": int(out[0]), "contrib_pairs": int(out[1]), "bwd_evals": int(out[2]), "pixels": int(out[3])}

    def entry_count(self) -> int:
        return int(self.read("entry_count", 1)[0])

    # --- SsimLoss::encode and Optimizer over the handle's buffers ---
    def loss_l1_ssim(self, w_l1: float, w_ssim: float, stream: int = 0):
        self._chk(lib().gs_loss_l1_ssim(self._h, w_l1, w_ssim, stream))

    def optimizer_init(self, num_surfels: int, stream: int = 0):
        self._chk(lib().gs_optimizer_init(self._h, num_surfels, stream))

    def optimizer_step(self, adam: "AdamSettings", num_surfels: int, stream: int = 0):
        cfg = adam.c()
        self._chk(lib().gs_optimizer_step(self._h, C.byref(cfg), num_surfels, stream))

    def train_step(self, cameras, num_surfels: int, step: "StepSettings", stream: int = 0):
        cams = camera_array(cameras)
        self.cams = cams
        cfg = step.c()
        self._chk(lib().gs_train_step(self._h, cams, len(cams), num_surfels, C.byref(cfg), stream))

    STAGES = ("project", "depth_sort_scan", "expand", "tile_sort", "ranges", "raster_fwd", "l1_ssim",
              "raster_bwd", "project_bwd_adam")

    def train_step_profiled(self, cameras, num_surfels: int, step: "StepSettings", stream: int = 0) -> dict:
        cams = camera_array(cameras)
        self.cams = cams
        cfg = step.c()
        ms = (C.c_float * 9)()
        ns = C.c_uint32()
        self._chk(lib().gs_train_step_profiled(self._h, cams, len(cams), num_surfels, C.byref(cfg), stream, ms,
                                               C.byref(ns)))
        return {k: float(ms[i]) for i, k in enumerate(self.STAGES)}

    def autotune(self, cameras, num_surfels: int, stream: int = 0) -> dict:
        """Time the raster launch shapes on these cameras and keep the fastest."""
        cams = camera_array(cameras)
        out = (C.c_uint32 * 4)()
        self._chk(lib().gs_autotune(self._h, cams, len(cams), num_surfels, stream, out))
        return {"fwd_batch": out[0], "fwd_pixels_per_thread": out[1], "bwd_batch": out[2],
                "bwd_pixels_per_thread": out[3]}

    def autotune_tiles(self, cameras, num_surfels: int, stream: int = 0) -> dict:
        """Time every tile size (8, 16, 32) with each of its raster launch shapes and keep the fastest."""
        cams = camera_array(cameras)
        out = (C.c_uint32 * 5)()
        times = (C.c_float * 6)()
        self._chk(lib().gs_autotune_tiles(self._h, cams, len(cams), num_surfels, stream, out, times))
        per_tile = {t: (None if times[2 * i] < 0 else {"fwd_ms": float(times[2 * i]), "bwd_ms": float(times[2 * i + 1])})
                    for i, t in enumerate((8, 16, 32))}
        return {"tile": out[0], "fwd_batch": out[1], "fwd_pixels_per_thread": out[2], "bwd_batch": out[3],
                "bwd_pixels_per_thread": out[4], "per_tile": per_tile}

    @property
    def tile(self) -> int:
        return int(lib().gs_tile_size(self._h))

    @tile.setter
    def tile(self, t: int):
        self._chk(lib().gs_set_tile_size(self._h, t))

    def set_launch_shapes(self, fwd_batch: int, fwd_pixels_per_thread: int, bwd_batch: int,
                          bwd_pixels_per_thread: int):
        """Apply raster launch shapes (e.g. a stored autotune result) without timing."""
        arr = (C.c_uint32 * 4)(fwd_batch, fwd_pixels_per_thread, bwd_batch, bwd_pixels_per_thread)
        self._chk(lib().gs_set_launch_shapes(self._h, arr))

    def loss_normal(self, lam: float, alpha_min: float = 0.2, stream: int = 0):
        """NormalLoss::encode for every view of the last forward (writes dl_dnormal and dl_dcolor.w)."""
        self._chk(lib().gs_loss_normal(self._h, lam, alpha_min, stream))

    def mcmc_seed(self, xorshift_state: int, stream: int = 0):
        self._chk(lib().gs_mcmc_seed(self._h, xorshift_state, stream))

    def mcmc_relocate(self, num_surfels: int, dead_threshold: float = 0.005, split_ratio: float = 8.0,
                      stream: int = 0):
        """Trainer::mcmc_relocate on the device (no readback)."""
        cfg = McmcConfig(dead_threshold, split_ratio)
        self._chk(lib().gs_mcmc_relocate(self._h, C.byref(cfg), num_surfels, stream))

    def mcmc_stats(self, stream: int = 0) -> dict:
        out = (C.c_uint32 * 4)()
        st = C.c_uint64()
        self._chk(lib().gs_mcmc_stats(self._h, out, C.byref(st), stream))
        return {"dead": out[0], "relocated": out[1], "split": out[2], "deferred": out[3], "rng_state": st.value}

    def mcmc_noise(self, num_surfels: int, seed: int, sigma: float, opacity_k: float = 5.0, stream: int = 0):
        self._chk(lib().gs_mcmc_noise(self._h, num_surfels, seed, sigma, opacity_k, stream))

    def save_ply(self, path: str, num_surfels: int, stream: int = 0):
        """The activated surfels [0, num_surfels) to a 3DGS-layout PLY file."""
        self._chk(lib().gs_rasterizer_save_ply(self._h, os.fsencode(path), num_surfels, stream))

    def load_ply(self, path: str, stream: int = 0) -> int:
        """A splat PLY file into the handle; returns its surfel count."""
        n = C.c_uint32()
        self._chk(lib().gs_rasterizer_load_ply(self._h, os.fsencode(path), C.byref(n), stream))
        return n.value

    def densify_prune(self, grad_threshold: float, opacity_threshold: float, num_surfels: int,
                      stream: int = 0) -> int:
        cfg = DensifyConfig(grad_threshold, opacity_threshold)
        out = C.c_uint32()
        self._chk(lib().gs_densify_prune(self._h, C.byref(cfg), num_surfels, C.byref(out), stream))
        return out.value


CLASSES = ("pos", "scales", "quat", "opacity", "sh")


@dataclass
class AdamSettings:
    """Per-class learning rates and L1 priors of the trainer's five classes
    (first_attempt/crates/gs-train/src/trainer.rs:757-761, defaults :471-476)."""
    lr: dict = field(default_factory=lambda: {"pos": 1.6e-4, "scales": 5e-3, "quat": 1e-3, "opacity": 5e-2,
                                              "sh": 2.5e-3})
    reg: dict = field(default_factory=lambda: {k: 0.0 for k in CLASSES})
    beta1: float = 0.9
    beta2: float = 0.999
    eps: float = 1e-8

    def c(self) -> AdamConfig:
        a = AdamConfig()
        for k, name in enumerate(CLASSES):
            a.lr[k] = float(self.lr[name])
            a.reg[k] = float(self.reg.get(name, 0.0))
        a.beta1, a.beta2, a.eps = self.beta1, self.beta2, self.eps
        return a


@dataclass
class StepSettings:
    w_l1: float = 0.8
    w_ssim: float = 0.2
    adam: AdamSettings = field(default_factory=AdamSettings)
    form: str = "chosen"  # "plain" or "chosen"
    loss: str = "l1_ssim"  # "l1_ssim" (against the target) or "given" (the caller's dl_dcolor)

    def c(self) -> StepConfig:
        return StepConfig(self.w_l1, self.w_ssim, self.adam.c(), 0 if self.form == "plain" else 1,
                          {"l1_ssim": 0, "given": 1}[self.loss])


class TileBinner:
    """TileBinner::new(ctx, max_items, max_entries, num_tiles). ``encode`` takes
    device pointers of uint4 rects and u32 depth keys (e.g. torch tensors'
    ``data_ptr()``)."""

    def __init__(self, max_items: int, max_entries: int, num_tiles: int):
        self._h = None
        h = C.c_void_p()
        check(lib().gs_binner_create(max_items, max_entries, num_tiles, C.byref(h)))
        self._h = h
        self.num_tiles = num_tiles

    def close(self):
        if self._h:
            lib().gs_binner_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def encode(self, rects_ptr: int, depths_ptr: int, num_items: int, tiles_x: int, stream: int = 0):
        check(lib().gs_binner_encode(self._h, rects_ptr, depths_ptr, num_items, tiles_x, stream))

    def buffer(self, which: str):
        idx = {"sorted_entries": 0, "entry_items": 1, "ranges": 2, "entry_count": 3}[which]
        p, n = C.c_void_p(), C.c_size_t()
        check(lib().gs_binner_buffer(self._h, idx, C.byref(p), C.byref(n)))
        return p.value, n.value


def camera_step_grad(grad_cam16, quat4) -> np.ndarray:
    """camera_step_grad (crates/gs-track/src/lib.rs:289-307)."""
    g = np.ascontiguousarray(grad_cam16, np.float32)
    q = np.ascontiguousarray(quat4, np.float32)
    out = np.zeros(6, np.float32)
    f = C.POINTER(C.c_float)
    check(lib().gs_camera_step_grad(g.ctypes.data_as(f), q.ctypes.data_as(f), out.ctypes.data_as(f)))
    return out


def camera_adam6(m, v, t: int, grad6, lr_rot: float, lr_center: float) -> np.ndarray:
    """adam6 (lib.rs:310-328); m and v (float32 arrays of 6) are updated in place."""
    g = np.ascontiguousarray(grad6, np.float32)
    step = np.zeros(6, np.float32)
    f = C.POINTER(C.c_float)
    check(lib().gs_camera_adam6(m.ctypes.data_as(f), v.ctypes.data_as(f), t, g.ctypes.data_as(f), lr_rot, lr_center,
                                step.ctypes.data_as(f)))
    return step


def camera_apply_step(cam: "RasterCamera", step6) -> "RasterCamera":
    """apply_camera_step (lib.rs:330-337) on a copy of the camera."""
    c = cam.c()
    s = np.ascontiguousarray(step6, np.float32)
    check(lib().gs_camera_apply_step(C.byref(c), s.ctypes.data_as(C.POINTER(C.c_float))))
    return RasterCamera(tuple(c.center[:]), tuple(c.quat[:]), c.focal, cam.sh_degree, cam.width, cam.height)


def scene_extent(positions) -> float:
    """Position-LR scale (first_attempt/crates/gs-train/src/trainer.rs:740-746):
    half the bounding-box diagonal of (n, >=3) positions, at least 1e-3."""
    p = np.ascontiguousarray(positions, np.float32)
    out = C.c_float()
    check(lib().gs_scene_extent(p.ctypes.data_as(C.POINTER(C.c_float)), p.shape[0], p.shape[1], C.byref(out)))
    return out.value


def schedule_t(iteration: int, iters: int, anneal=None) -> float:
    """schedule_t (trainer.rs:407-416); anneal = (start, len, t0) or None."""
    from ._lib import Anneal
    out = C.c_float()
    a = None if anneal is None else C.byref(Anneal(*anneal))
    check(lib().gs_schedule_t(iteration, iters, a, C.byref(out)))
    return out.value


def position_lr(lr_pos: float, extent: float, final_factor: float, t: float) -> float:
    """The exponential position-LR decay of trainer.rs:1150."""
    out = C.c_float()
    check(lib().gs_position_lr(lr_pos, extent, final_factor, t, C.byref(out)))
    return out.value


def write_ply(path: str, positions4, scales2, quats4, opacities, sh48):
    """write_3dgs_ply (first_attempt/crates/gs-io/src/ply/writer.rs) from host
    arrays of activated values: positions (n,4), scales (n,2), quats xyzw
    (n,4), opacities (n,), SH (n,48) coefficient-major."""
    arrs = [np.ascontiguousarray(a, np.float32) for a in (positions4, scales2, quats4, opacities, sh48)]
    n = arrs[3].shape[0]
    check(lib().gs_ply_write(os.fsencode(path), n, *[a.ctypes.data for a in arrs]))


def read_ply(path: str) -> dict:
    """load_ply of a splat file (ply/reader.rs): activated positions (n,3),
    scales (n,3), quats xyzw (n,4), opacities (n,), SH (n, coeffs*3)."""
    n, nc = C.c_uint32(), C.c_uint32()
    check(lib().gs_ply_info(os.fsencode(path), C.byref(n), C.byref(nc)))
    k = n.value
    out = {"positions": np.zeros((k, 3), np.float32), "scales": np.zeros((k, 3), np.float32),
           "quats": np.zeros((k, 4), np.float32), "opacities": np.zeros(k, np.float32),
           "sh": np.zeros((k, 3 * nc.value), np.float32)}
    got = C.c_uint32()
    check(lib().gs_ply_read(os.fsencode(path), k, out["positions"].ctypes.data, out["scales"].ctypes.data,
                            out["quats"].ctypes.data, out["opacities"].ctypes.data, out["sh"].ctypes.data,
                            C.byref(got)))
    out["sh_coeffs"] = nc.value
    return out


def radix_sort_pairs(keys_ptr: int, vals_ptr: int, n: int, key_bits: int = 32, stream: int = 0):
    """RadixSorter::encode on caller device arrays (stable, in place)."""
    check(lib().gs_radix_sort_pairs(keys_ptr, vals_ptr, n, key_bits, stream))


def radix_sort_pairs_noalloc(keys_ptr: int, vals_ptr: int, n: int, key_bits: int = 32, stream: int = 0):
    """The same sort for callers that cannot let the library allocate: scratch
    is a fixed device array for at most 1,048,576 pairs; overlapping calls on
    the GPU race. Stream-ordered (does not synchronise)."""
    check(lib().gs_radix_sort_pairs_noalloc(keys_ptr, vals_ptr, n, key_bits, stream))


def exclusive_scan_u32(in_ptr: int, out_ptr: int, n: int, total_ptr: int = 0, stream: int = 0):
    """PrefixSum::encode on caller device arrays."""
    check(lib().gs_exclusive_scan_u32(in_ptr, out_ptr, n, total_ptr or None, stream))


def adam_flat(raw_ptr, grad_ptr, m_ptr, v_ptr, act_ptr, n, activation, lr, beta1=0.9, beta2=0.999, eps=1e-8, reg=0.0,
              t=1, stream=0):
    check(lib().gs_adam_flat(raw_ptr, grad_ptr, m_ptr, v_ptr, act_ptr or None, n, activation, lr, beta1, beta2, eps,
                             reg, t, stream))
