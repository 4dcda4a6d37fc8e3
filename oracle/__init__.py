"""Correctness oracle for the surfel training step — TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this package, and only as the checker or the timed CPU
baseline. The shipped library never calls it.

PARITY STATUS: unpinned against golden vectors. The reference ships no
known-answer files for this path and its own oracle (crates/gs-cpu-ref, Rust)
cannot be built here. ``gs_oracle.hpp`` restates it line by line in C++ and the
restatement is certified by central finite differences (the reference's own
gate, crates/gs-cpu-ref/tests/gradcheck.rs) and analytic known answers.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None


def build(force: bool = False) -> str:
    """Compile liboracle.so with the committed Makefile (g++, OpenMP)."""
    src = [os.path.join(_HERE, f) for f in ("gs_oracle.cpp", "gs_oracle.hpp", "Makefile")]
    stale = not os.path.exists(_LIB_PATH) or any(os.path.getmtime(s) > os.path.getmtime(_LIB_PATH) for s in src)
    if force or stale:
        env = dict(os.environ)
        env.pop("CXX", None)
        subprocess.run(["make", "-C", _HERE, "-s", "liboracle.so"], check=True, env=env)
    return _LIB_PATH


class _Scene(C.Structure):
    _fields_ = [("n", C.c_int), ("sh_degree", C.c_int), ("pos", C.c_void_p), ("scales", C.c_void_p),
                ("quat", C.c_void_p), ("opacity", C.c_void_p), ("sh", C.c_void_p)]


class _Camera(C.Structure):
    _fields_ = [("center", C.c_double * 3), ("quat", C.c_double * 4), ("focal", C.c_double),
                ("width", C.c_int), ("height", C.c_int)]


class _Grads(C.Structure):
    _fields_ = [(k, C.c_void_p) for k in
                ("pos", "scales", "quat", "opacity", "sh", "cam_center", "cam_quat", "focal", "dl_dr_cam")]


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        vp, i32, f64 = C.c_void_p, C.c_int, C.c_double
        L.orc_project.argtypes = [vp, vp, i32, vp, vp, vp, vp]
        L.orc_project.restype = i32
        L.orc_render.argtypes = [vp, vp, i32, i32, i32, vp, vp, vp, vp, vp, vp, vp]
        L.orc_render.restype = i32
        L.orc_gradients.argtypes = [vp, vp, i32, vp, vp, vp, f64, i32, vp]
        L.orc_gradients.restype = i32
        L.orc_render_sampled.argtypes = [vp, vp, i32, i32, i32, i32, vp, vp, vp, vp, vp, vp, vp, vp, vp]
        L.orc_render_sampled.restype = i32
        L.orc_gradients_sampled.argtypes = [vp, vp, i32, i32, i32, vp, vp, vp, f64, i32, vp]
        L.orc_gradients_sampled.restype = i32
        L.orc_distortion_loss.argtypes = [vp, vp, i32]
        L.orc_distortion_loss.restype = f64
        L.orc_project_f32.argtypes = [i32, vp, vp, vp, vp, vp, C.c_float, i32, i32, i32, vp, vp, vp]
        L.orc_project_f32.restype = i32
        L.orc_camera_rotation_f32.argtypes = [vp, vp]
        L.orc_camera_rotation_f32.restype = None
        L.orc_gauss_weights.argtypes = [vp]
        L.orc_sh_color.argtypes = [i32, vp, vp, vp, vp]
        L.orc_sh_color.restype = i32
        L.orc_triple.argtypes = [vp, vp, vp, vp, vp, vp]
        L.orc_quat_to_mat.argtypes = [vp, vp]
        L.orc_quat_to_mat.restype = None
        L.orc_quat_grad.argtypes = [vp, vp, vp]
        L.orc_quat_grad.restype = None
        L.orc_sh_basis.argtypes = [i32, vp, vp, vp]
        L.orc_sh_basis.restype = i32
        L.orc_triple.restype = f64
        L.orc_gauss_weights.restype = None
        L.orc_l1_ssim.argtypes = [vp, vp, i32, i32, f64, f64, vp, vp, vp]
        L.orc_l1_ssim.restype = f64
        L.orc_adam.argtypes = [i32, vp, vp, vp, vp, vp, i32, f64, f64, f64, f64, f64, i32]
        L.orc_adam.restype = None
        L.orc_cpu_step_timed.argtypes = [vp, vp, i32, i32, i32, vp, vp]
        L.orc_cpu_step_timed.restype = i32
        L.orc_max_threads.argtypes = []
        L.orc_max_threads.restype = i32
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data


@dataclass
class Scene:
    """Activated surfel parameters in float64 (the oracle's precision)."""
    pos: np.ndarray      # (n,3)
    scales: np.ndarray   # (n,2) activated
    quat: np.ndarray     # (n,4) xyzw, unnormalised
    opacity: np.ndarray  # (n,)
    sh: np.ndarray       # (n,48) coefficient-major rgb, padded to 16 coefficients
    sh_degree: int

    @property
    def n(self):
        return self.pos.shape[0]

    def c(self):
        self.pos = np.ascontiguousarray(self.pos, np.float64)
        self.scales = np.ascontiguousarray(self.scales, np.float64)
        self.quat = np.ascontiguousarray(self.quat, np.float64)
        self.opacity = np.ascontiguousarray(self.opacity, np.float64)
        self.sh = np.ascontiguousarray(self.sh, np.float64)
        s = _Scene(self.n, self.sh_degree, _p(self.pos), _p(self.scales), _p(self.quat), _p(self.opacity),
                   _p(self.sh))
        return s

    def copy(self):
        return Scene(self.pos.copy(), self.scales.copy(), self.quat.copy(), self.opacity.copy(), self.sh.copy(),
                     self.sh_degree)


@dataclass
class Camera:
    center: np.ndarray  # (3,)
    quat: np.ndarray    # (4,) camera-to-world xyzw
    focal: float
    width: int
    height: int

    def c(self):
        cam = _Camera()
        for k in range(3):
            cam.center[k] = float(self.center[k])
        for k in range(4):
            cam.quat[k] = float(self.quat[k])
        cam.focal = float(self.focal)
        cam.width = int(self.width)
        cam.height = int(self.height)
        return cam

    def copy(self):
        return Camera(np.array(self.center, np.float64), np.array(self.quat, np.float64), float(self.focal),
                      self.width, self.height)


def project(scene: Scene, cam: Camera, tile: int = 16):
    n = scene.n
    rects = np.zeros((n, 4), np.int32)
    keys = np.zeros(n, np.uint32)
    marg = np.zeros(n, np.uint8)
    pos = np.zeros(n, np.int32)
    s, c = scene.c(), cam.c()
    lib().orc_project(C.byref(s), C.byref(c), tile, _p(rects), _p(keys), _p(marg), _p(pos))
    return rects, keys, marg.astype(bool), pos


def render(scene: Scene, cam: Camera, tile: int = 16, literal: bool = False, threads: int = 0,
           tile_stride: int = 1, tile_offset: int = 0):
    """Per-pixel forward outputs. With tile_stride > 1 only the pixels of
    tiles t with t % tile_stride == tile_offset (row-major tile ids) are
    rendered (the others stay zero, `sampled` marks the rendered ones).
    Except for the literal walk, `last` holds each rendered pixel's last
    contributing surfel (input index, -1 if none) and `count` its number of
    contributing surfels."""
    P = cam.width * cam.height
    out = dict(color=np.zeros((P, 3)), alpha=np.zeros(P), depth=np.zeros(P), normal=np.zeros((P, 3)),
               trans=np.zeros(P), ncontrib=np.zeros(P, np.int32), marginal=np.zeros(P, np.uint8),
               last=np.full(P, -1, np.int32), count=np.zeros(P, np.int32))
    s, c = scene.c(), cam.c()
    if not literal:
        rc = lib().orc_render_sampled(C.byref(s), C.byref(c), tile, tile_stride, tile_offset, threads,
                                      _p(out["color"]), _p(out["alpha"]), _p(out["depth"]), _p(out["normal"]),
                                      _p(out["trans"]), _p(out["ncontrib"]), _p(out["marginal"]), _p(out["last"]),
                                      _p(out["count"]))
        assert rc == 0, "bad tile sample"
    else:
        lib().orc_render(C.byref(s), C.byref(c), tile, int(literal), threads, _p(out["color"]), _p(out["alpha"]),
                         _p(out["depth"]), _p(out["normal"]), _p(out["trans"]), _p(out["ncontrib"]),
                         _p(out["marginal"]))
    out["marginal"] = out["marginal"].astype(bool)
    out["sampled"] = sampled_pixels(cam, tile, tile_stride, tile_offset)
    return out


def sampled_pixels(cam: Camera, tile: int = 16, tile_stride: int = 1, tile_offset: int = 0) -> np.ndarray:
    """Mask (P,) of the pixels whose row-major tile id t has t % tile_stride == tile_offset."""
    tiles_x = (cam.width + tile - 1) // tile
    ys, xs = np.divmod(np.arange(cam.width * cam.height), cam.width)
    t = (ys // tile) * tiles_x + xs // tile
    return (t % tile_stride) == tile_offset


def gradients(scene: Scene, cam: Camera, dl_dcolor, dl_ddepth=None, dl_dnormal=None, lambda_dist: float = 0.0,
              tile: int = 16, threads: int = 0, tile_stride: int = 1, tile_offset: int = 0):
    """Parameter and camera gradients of a loss with the given per-pixel image
    gradients. With tile_stride > 1 only the pixels of the sampled tiles
    (t % tile_stride == tile_offset) are walked: the exact gradient of a loss
    whose image gradient is zero elsewhere."""
    n = scene.n
    g = dict(pos=np.zeros((n, 3)), scales=np.zeros((n, 2)), quat=np.zeros((n, 4)), opacity=np.zeros(n),
             sh=np.zeros((n, 48)), cam_center=np.zeros(3), cam_quat=np.zeros(4), focal=np.zeros(1),
             dl_dr_cam=np.zeros(9))
    gs = _Grads(*[_p(g[k]) for k in ("pos", "scales", "quat", "opacity", "sh", "cam_center", "cam_quat", "focal",
                                      "dl_dr_cam")])
    dlc = np.ascontiguousarray(dl_dcolor, np.float64).reshape(-1, 3)
    dld = None if dl_ddepth is None else np.ascontiguousarray(dl_ddepth, np.float64).reshape(-1)
    dln = None if dl_dnormal is None else np.ascontiguousarray(dl_dnormal, np.float64).reshape(-1, 3)
    s, c = scene.c(), cam.c()
    if tile_stride > 1:
        rc = lib().orc_gradients_sampled(C.byref(s), C.byref(c), tile, tile_stride, tile_offset, _p(dlc), _p(dld),
                                         _p(dln), float(lambda_dist), threads, C.byref(gs))
        assert rc == 0, "bad tile sample"
    else:
        lib().orc_gradients(C.byref(s), C.byref(c), tile, _p(dlc), _p(dld), _p(dln), float(lambda_dist), threads,
                            C.byref(gs))
    g["focal"] = float(g["focal"][0])
    return g


def distortion_loss(scene: Scene, cam: Camera, tile: int = 16) -> float:
    s, c = scene.c(), cam.c()
    return lib().orc_distortion_loss(C.byref(s), C.byref(c), tile)


def camera_rotation_f32(quat) -> np.ndarray:
    q = np.ascontiguousarray(quat, np.float32)
    r = np.zeros(9, np.float32)
    lib().orc_camera_rotation_f32(_p(q), _p(r))
    return r


def project_f32(pos4, scales2, quats4, rot9, center3, focal, width, height, tile=16):
    """f32 mirror of the projection: (rects (n,4) u32, keys (n,) u32, cam (n,12) f32)."""
    pos4 = np.ascontiguousarray(pos4, np.float32)
    scales2 = np.ascontiguousarray(scales2, np.float32)
    quats4 = np.ascontiguousarray(quats4, np.float32)
    rot9 = np.ascontiguousarray(rot9, np.float32)
    center3 = np.ascontiguousarray(center3, np.float32)
    n = pos4.shape[0]
    rects = np.zeros((n, 4), np.uint32)
    keys = np.zeros(n, np.uint32)
    camo = np.zeros((n, 12), np.float32)
    lib().orc_project_f32(n, _p(pos4), _p(scales2), _p(quats4), _p(rot9), _p(center3), float(focal), width, height,
                          tile, _p(rects), _p(keys), _p(camo))
    return rects, keys, camo


def sh_color(degree: int, coeffs, direction):
    """(rgb, clamp mask) of max(0.5 + sum sh_k basis_k(dir), 0); coeffs (k, 3)."""
    sh = np.zeros(48)
    c = np.asarray(coeffs, np.float64).reshape(-1)
    sh[:c.size] = c
    d = np.ascontiguousarray(direction, np.float64)
    rgb = np.zeros(3)
    cm = np.zeros(3, np.int32)
    lib().orc_sh_color(degree, _p(sh), _p(d), _p(rgb), cm.ctypes.data)
    return rgb, cm.astype(bool)


def quat_to_mat(q) -> np.ndarray:
    """Column-major rotation (as a 3x3 array indexed [col][row]) of an xyzw quaternion."""
    q = np.ascontiguousarray(q, np.float64)
    r = np.zeros(9)
    lib().orc_quat_to_mat(_p(q), _p(r))
    return r.reshape(3, 3)


def quat_grad(q, dl_dr_cols) -> np.ndarray:
    """dL/dq for dL/dR given as [col][row]."""
    q = np.ascontiguousarray(q, np.float64)
    w = np.ascontiguousarray(dl_dr_cols, np.float64).reshape(9)
    out = np.zeros(4)
    lib().orc_quat_grad(_p(q), _p(w), _p(out))
    return out


def sh_basis(degree: int, direction):
    """(basis values (k,), d basis / d dir (k, 3))."""
    d = np.ascontiguousarray(direction, np.float64)
    b, g = np.zeros(16), np.zeros(48)
    nb = lib().orc_sh_basis(degree, _p(d), _p(b), _p(g))
    return b[:nb], g[:3 * nb].reshape(nb, 3)


def triple(a, b, c):
    """(a . (b x c), d/da, d/db, d/dc)."""
    a, b, c = (np.ascontiguousarray(x, np.float64) for x in (a, b, c))
    ga, gb, gc = np.zeros(3), np.zeros(3), np.zeros(3)
    t = lib().orc_triple(_p(a), _p(b), _p(c), _p(ga), _p(gb), _p(gc))
    return t, ga, gb, gc


def gauss_weights() -> np.ndarray:
    w = np.zeros(6)
    lib().orc_gauss_weights(_p(w))
    return w


def l1_ssim(img_rgba, ref_rgba, width, height, w_l1=0.8, w_ssim=0.2):
    """(loss, dL/dimg rgba, l1 channel sum, ssim channel sum) in float64."""
    img = np.ascontiguousarray(img_rgba, np.float64).reshape(-1, 4)
    ref = np.ascontiguousarray(ref_rgba, np.float64).reshape(-1, 4)
    dl = np.zeros_like(img)
    l1 = C.c_double()
    ss = C.c_double()
    loss = lib().orc_l1_ssim(_p(img), _p(ref), width, height, w_l1, w_ssim, _p(dl), C.byref(l1), C.byref(ss))
    return loss, dl, l1.value, ss.value


def adam(raw, grad_act, m, v, activation, lr, beta1=0.9, beta2=0.999, eps=1e-8, reg=0.0, t=1):
    """One Adam step in float64 (in place on raw/m/v); returns the activated values."""
    raw = np.ascontiguousarray(raw, np.float64)
    g = np.ascontiguousarray(grad_act, np.float64)
    m = np.ascontiguousarray(m, np.float64)
    v = np.ascontiguousarray(v, np.float64)
    act = np.zeros_like(raw)
    lib().orc_adam(raw.size, _p(raw), _p(g), _p(m), _p(v), _p(act), activation, lr, beta1, beta2, eps, reg, t)
    return raw, m, v, act


def max_threads() -> int:
    return lib().orc_max_threads()


def cpu_step_timed(scene: Scene, cam: Camera, target_rgba, tile=16, tile_stride=1, threads=0):
    """Seconds per phase (prep+bin, fwd, loss, bwd, chain, adam) of one CPU step."""
    times = np.zeros(6)
    tgt = np.ascontiguousarray(target_rgba, np.float64).reshape(-1, 4)
    s, c = scene.c(), cam.c()
    lib().orc_cpu_step_timed(C.byref(s), C.byref(c), tile, tile_stride, threads, _p(tgt), _p(times))
    return times


def densify(arrays: dict, widths: dict, moments: set, grad_norm_sum, steps: int, opacity_act,
            grad_threshold: float, opacity_threshold: float, capacity: int):
    """Clone/prune compaction restated in numpy (the reference has no such
    pass; it relocates at a fixed budget, first_attempt/crates/gs-train/src/
    trainer.rs:1558-1689). A surfel is kept when its activated opacity is at
    least `opacity_threshold`; a kept surfel is cloned when its mean
    |dL/dpos| over the accumulated steps exceeds `grad_threshold`. Survivors
    keep their order, clones follow in the order of their sources, and clones
    past `capacity` are dropped. Clones copy every array except the moment
    arrays (names in `moments`), which start at zero. Returns (new arrays,
    new count)."""
    n = len(opacity_act)
    keep = np.asarray(opacity_act, np.float32) >= np.float32(opacity_threshold)
    inv = np.float32(1.0 / steps) if steps else np.float32(0.0)
    mean = np.asarray(grad_norm_sum, np.float32) * inv
    clone = keep & (mean > np.float32(grad_threshold))
    kept_idx = np.nonzero(keep)[0]
    clone_idx = np.nonzero(clone)[0][:max(0, capacity - len(kept_idx))]
    out = {}
    for name, a in arrays.items():
        w = widths[name]
        rows = np.asarray(a).reshape(-1, w)[:n]
        cl = np.zeros((len(clone_idx), w), rows.dtype) if name in moments else rows[clone_idx]
        out[name] = np.concatenate([rows[kept_idx], cl], axis=0)
    return out, len(kept_idx) + len(clone_idx)


_M64 = (1 << 64) - 1


def _xorshift(x: int) -> int:
    x ^= (x << 13) & _M64
    x ^= x >> 7
    x ^= (x << 17) & _M64
    return x


def mcmc_pairs(opacity_act, scales_act, rng_state: int, dead_threshold=0.005, split_ratio=8.0):
    """Restatement of the reference's host sampler (first_attempt/crates/
    gs-train/src/trainer.rs:1558-1647): dead = activated opacity below the
    threshold; per dead surfel in index order one xorshift64 draw r·total
    picks the first alive surfel whose cumulative (f64) opacity reaches it; a
    pick equal to the dead index or already used defers the dead surfel;
    leftover dead slots then split unused alive surfels larger than
    split_ratio × the median alive size, largest first. Returns
    (pairs [(dead, alive, mode)], new generator state)."""
    op = np.asarray(opacity_act, np.float32)
    n = len(op)
    thr = np.float32(dead_threshold)
    dead = [i for i in range(n) if op[i] < thr]
    if not dead:
        return [], rng_state
    cum = []
    total = 0.0
    for o in op:
        if o >= thr:
            total += float(o)
        cum.append(total)
    if total <= 0.0:
        return [], rng_state
    cum = np.array(cum)
    used = np.zeros(n, bool)
    spent = np.zeros(len(dead), bool)
    pairs = []
    x = rng_state
    for di, d in enumerate(dead):
        x = _xorshift(x)
        r = float(x >> 11) / float(1 << 53) * total
        a = min(int(np.searchsorted(cum, r, side="left")), n - 1)
        if a == d or used[a]:
            continue
        used[a] = True
        spent[di] = True
        pairs.append((d, a, 0))
    if split_ratio > 0.0:
        sc = np.asarray(scales_act, np.float32).reshape(n, 2)
        size = np.maximum(sc[:, 0], sc[:, 1])
        alive = op >= thr
        alive_sizes = np.sort(size[alive], kind="stable")
        if len(alive_sizes) >= 16:
            med = alive_sizes[len(alive_sizes) // 2]
            cap = np.float32(split_ratio) * med
            over = [i for i in range(n) if alive[i] and size[i] > cap and not used[i]]
            over.sort(key=lambda i: -size[i])  # stable: ties keep index order
            left = [d for di, d in enumerate(dead) if not spent[di]]
            for big, slot in zip(over, left):
                used[big] = True
                pairs.append((slot, big, 1))
    return pairs, x


def mcmc_apply(raw: dict, opacity_act, pairs):
    """relocate.wgsl relocate_params/relocate_moments on numpy float32 copies:
    raw = {"pos" (n,4), "scales" (n,2), "quat" (n,4), "opacity" (n,), "sh" (n,48),
    "m_*"/"v_*" moments}. Returns the updated dict."""
    out = {k: np.array(v, np.float32, copy=True) for k, v in raw.items()}
    op = np.asarray(opacity_act, np.float32)
    f = np.float32
    for d, a, mode in pairs:
        alpha = np.clip(op[a], f(1e-4), f(0.999))
        an = np.clip(f(1.0) - np.sqrt(f(1.0) - alpha), f(1e-4), f(0.999))
        logit = np.log(an / (f(1.0) - an))
        out["opacity"][d] = logit
        out["opacity"][a] = logit
        q = out["quat"][a].copy()
        out["quat"][d] = q
        s = out["scales"][a].copy()
        if mode == 1:
            qn = q / np.sqrt((q * q).sum(dtype=np.float32))
            x, y, z, w = qn
            col0 = np.array([1 - 2 * (y * y + z * z), 2 * (x * y + w * z), 2 * (x * z - w * y)], np.float32)
            col1 = np.array([2 * (x * y - w * z), 1 - 2 * (x * x + z * z), 2 * (y * z + w * x)], np.float32)
            sw = np.exp(s)
            axis = col0 * sw[0] if not sw[1] > sw[0] else col1 * sw[1]
            c = out["pos"][a].copy()
            out["pos"][d] = c + np.append(f(0.6) * axis, f(0.0))
            out["pos"][a] = c - np.append(f(0.6) * axis, f(0.0))
            s = s - f(0.51)
        else:
            out["pos"][d] = out["pos"][a]
            s = s - f(0.16)
        out["scales"][a] = s
        out["scales"][d] = s
        out["sh"][d] = out["sh"][a]
        for k in list(out):
            if k.startswith(("m_", "v_")):
                out[k][d] = 0
                out[k][a] = 0
    return out


def normal_loss(alpha, depth_acc, normal, W: int, H: int, focal: float, lam: float, alpha_min: float = 0.2):
    """Restatement in float64 of the normal-consistency loss (first_attempt/
    crates/gs-train/src/shaders/normal_loss.wgsl:52-145) for one view:
    L = lam/(W·H) Σ_q α_q (1 − n̂_q·N_d(q)), α and the orientation sign
    detached. Inputs per pixel (row-major): alpha (P,), depth_acc (P,),
    normal (P,3). Returns (Σ α(1 − n̂·N_d), dL/dnormal (P,3), dL/ddepth_acc (P,))."""
    a = np.asarray(alpha, np.float64).reshape(H, W)
    d = np.asarray(depth_acc, np.float64).reshape(H, W)
    nv = np.asarray(normal, np.float64).reshape(H, W, 3)
    ys, xs = np.mgrid[0:H, 0:W]
    ray = np.stack([(xs + 0.5 - W / 2) / focal, -(ys + 0.5 - H / 2) / focal, -np.ones_like(xs, np.float64)], -1)
    tbar = np.where(a >= alpha_min, d / np.where(a > 0, a, 1), 0.0)
    P = tbar[..., None] * ray
    lam_px = lam / (W * H)
    dl_dn = np.zeros((H, W, 3))
    cpx = np.zeros((H, W, 3))
    cpy = np.zeros((H, W, 3))
    total = 0.0
    for y in range(H - 1):
        for x in range(W - 1):
            if a[y, x] < alpha_min or a[y, x + 1] < alpha_min or a[y + 1, x] < alpha_min:
                continue
            p = P[y, x]
            dpx, dpy = P[y, x + 1] - p, P[y + 1, x] - p
            m = np.cross(dpx, dpy)
            l2 = m @ m
            if l2 < 1e-18:
                continue
            ln = np.sqrt(l2)
            mh = m / ln
            sign = -1.0 if mh @ p > 0 else 1.0
            nd = sign * mh
            av = nv[y, x]
            la2 = av @ av
            if la2 < 1e-18:
                continue
            la = np.sqrt(la2)
            nh = av / la
            aq = a[y, x]
            total += (1 - nh @ nd) * aq
            dl_dnd = -lam_px * aq * nh
            dl_dnh = -lam_px * aq * nd
            dl_dn[y, x] = (dl_dnh - nh * (nh @ dl_dnh)) / la
            dl_dm = sign * (dl_dnd - mh * (mh @ dl_dnd)) / ln
            cpx[y, x] = np.cross(dpy, dl_dm)
            cpy[y, x] = np.cross(dl_dm, dpx)
    acc = -cpx - cpy
    acc[:, 1:] += cpx[:, :-1]
    acc[1:, :] += cpy[:-1, :]
    dd = np.where(a >= alpha_min, (ray * acc).sum(-1) / np.where(a > 0, a, 1), 0.0)
    return total, dl_dn.reshape(-1, 3), dd.reshape(-1)
