"""Seeded synthetic surfel scenes and camera rigs for the training-step workloads.

The reference trains on posed photos or video that are not part of this path;
these generators stand in for them with fixed distributions (numpy PCG64,
seeded):

* centres uniform in [-1,1]^3 (small scene) or drawn from 64 isotropic
  Gaussian clusters (sigma 0.15) whose means are uniform in [-2,2]^3;
* two tangent scales exp(N(-3.5, 0.5)); uniform random unit quaternions
  (Shoemake's method); opacity sigmoid(N(0,1));
* SH degree 0 with coefficients N(0, 0.3), or degree 3 with N(0, 0.1).

Cameras follow Camera::look_at (crates/gs-core/src/camera.rs:40-49): eye,
target and world up +y give the camera-to-world frame (right, up, -forward).
Where no focal length is given the reference's default 60 degree vertical
field of view is used: f = 0.5 H / tan(30 deg) (camera.rs:28-32, 57).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .rasterizer import RasterCamera, SceneInput

RING_RESOLUTIONS = [(640, 480), (800, 600), (1024, 768), (1280, 720), (1280, 720), (1600, 900), (1920, 1080),
                    (1920, 1080)]


@dataclass
class Surfels:
    positions: np.ndarray
    scales: np.ndarray
    quats: np.ndarray
    opacities: np.ndarray
    sh: np.ndarray  # (n, coeffs*3)
    sh_degree: int

    @property
    def n(self):
        return self.positions.shape[0]

    def scene_input(self) -> SceneInput:
        return SceneInput(self.positions, self.scales, self.quats, self.opacities, self.sh, (self.sh_degree + 1) ** 2)

    def sh48(self) -> np.ndarray:
        out = np.zeros((self.n, 48), self.sh.dtype)
        out[:, :self.sh.shape[1]] = self.sh
        return out


def shoemake_quats(rng: np.random.Generator, n: int) -> np.ndarray:
    u1, u2, u3 = rng.random(n), rng.random(n), rng.random(n)
    a, b = np.sqrt(1 - u1), np.sqrt(u1)
    q = np.stack([a * np.sin(2 * np.pi * u2), a * np.cos(2 * np.pi * u2), b * np.sin(2 * np.pi * u3),
                  b * np.cos(2 * np.pi * u3)], axis=1)
    return q


def make_surfels(n: int, seed: int, clustered: bool, sh_degree: int, sh_sigma: float) -> Surfels:
    rng = np.random.default_rng(seed)
    if clustered:
        means = rng.uniform(-2.0, 2.0, size=(64, 3))
        which = rng.integers(0, 64, size=n)
        pos = means[which] + rng.normal(0.0, 0.15, size=(n, 3))
    else:
        pos = rng.uniform(-1.0, 1.0, size=(n, 3))
    scales = np.exp(rng.normal(-3.5, 0.5, size=(n, 2)))
    quats = shoemake_quats(rng, n)
    opac = 1.0 / (1.0 + np.exp(-rng.normal(0.0, 1.0, size=n)))
    ncoef = (sh_degree + 1) ** 2
    sh = rng.normal(0.0, sh_sigma, size=(n, ncoef * 3))
    f = np.float32
    return Surfels(pos.astype(f), scales.astype(f), quats.astype(f), opac.astype(f), sh.astype(f), sh_degree)


def quat_from_matrix(m: np.ndarray) -> np.ndarray:
    """xyzw quaternion of a rotation matrix (columns = images of e0, e1, e2)."""
    t = m[0, 0] + m[1, 1] + m[2, 2]
    if t > 0:
        s = math.sqrt(t + 1.0) * 2
        w, x, y, z = 0.25 * s, (m[2, 1] - m[1, 2]) / s, (m[0, 2] - m[2, 0]) / s, (m[1, 0] - m[0, 1]) / s
    elif m[0, 0] > m[1, 1] and m[0, 0] > m[2, 2]:
        s = math.sqrt(1.0 + m[0, 0] - m[1, 1] - m[2, 2]) * 2
        w, x, y, z = (m[2, 1] - m[1, 2]) / s, 0.25 * s, (m[0, 1] + m[1, 0]) / s, (m[0, 2] + m[2, 0]) / s
    elif m[1, 1] > m[2, 2]:
        s = math.sqrt(1.0 + m[1, 1] - m[0, 0] - m[2, 2]) * 2
        w, x, y, z = (m[0, 2] - m[2, 0]) / s, (m[0, 1] + m[1, 0]) / s, 0.25 * s, (m[1, 2] + m[2, 1]) / s
    else:
        s = math.sqrt(1.0 + m[2, 2] - m[0, 0] - m[1, 1]) * 2
        w, x, y, z = (m[1, 0] - m[0, 1]) / s, (m[0, 2] + m[2, 0]) / s, (m[1, 2] + m[2, 1]) / s, 0.25 * s
    return np.array([x, y, z, w])


def look_at(eye, target, width: int, height: int, focal: float | None = None, sh_degree: int = 0,
            up=(0.0, 1.0, 0.0)) -> RasterCamera:
    eye, target, up = (np.asarray(v, np.float64) for v in (eye, target, up))
    fwd = target - eye
    fwd /= np.linalg.norm(fwd)
    right = np.cross(fwd, up)
    right /= np.linalg.norm(right)
    up2 = np.cross(right, fwd)
    m = np.stack([right, up2, -fwd], axis=1)
    f = focal if focal is not None else 0.5 * height / math.tan(math.radians(30.0))
    return RasterCamera(tuple(eye), tuple(quat_from_matrix(m)), float(f), sh_degree, width, height)


def ring_cameras(resolutions, radius: float = 4.0, sh_degree: int = 3):
    cams = []
    nv = len(resolutions)
    for k, (w, h) in enumerate(resolutions):
        a = 2 * math.pi * k / nv
        cams.append(look_at((radius * math.sin(a), 0.0, radius * math.cos(a)), (0, 0, 0), w, h, sh_degree=sh_degree))
    return cams


@dataclass
class Workload:
    name: str
    surfels: Surfels
    target_surfels: Surfels
    cameras: list
    note: str

    @property
    def pixels(self) -> int:
        return sum(c.width * c.height for c in self.cameras)


def workload(name: str) -> Workload:
    """The benchmark's named configurations."""
    if name == "small_1view_256":  # 16,384 surfels, one 256x256 view, SH deg 0
        s = make_surfels(16384, 0, False, 0, 0.3)
        t = make_surfels(16384, 1, False, 0, 0.3)
        cams = [look_at((0, 0, -3), (0, 0, 0), 256, 256, focal=256.0, sh_degree=0)]
        return Workload(name, s, t, cams, "16,384 surfels U[-1,1]^3, SH deg 0, one 256x256 view, f=256")
    if name == "mid_1view_720p":  # 300,000 surfels, one 1280x720 view, SH deg 3
        s = make_surfels(300_000, 0, False, 3, 0.1)
        t = make_surfels(300_000, 1, False, 3, 0.1)
        cams = [look_at((0, 0, -3), (0, 0, 0), 1280, 720, sh_degree=3)]
        return Workload(name, s, t, cams, "300,000 surfels U[-1,1]^3, SH deg 3, one 1280x720 view")
    if name == "ring8_1m":  # 1,000,000 surfels, 8 uneven views up to 1080p
        s = make_surfels(1_000_000, 0, True, 3, 0.1)
        t = make_surfels(1_000_000, 1, True, 3, 0.1)
        cams = ring_cameras(RING_RESOLUTIONS)
        return Workload(name, s, t, cams, "1,000,000 surfels in 64 clusters, SH deg 3, 8 ring views 640x480..1920x1080")
    if name == "ring2_200k":  # profiling case: larger than L2, ~1 GB on the device
        s = make_surfels(200_000, 0, True, 3, 0.1)
        t = make_surfels(200_000, 1, True, 3, 0.1)
        cams = ring_cameras([(1920, 1080), (1920, 1080)])
        return Workload(name, s, t, cams, "200,000 surfels in 64 clusters, SH deg 3, 2 views 1920x1080")
    if name == "ring8_250k":  # profiling case with the 8-view rig: a quarter of the surfels
        s = make_surfels(250_000, 0, True, 3, 0.1)
        t = make_surfels(250_000, 1, True, 3, 0.1)
        cams = ring_cameras(RING_RESOLUTIONS)
        return Workload(name, s, t, cams, "250,000 surfels in 64 clusters, SH deg 3, 8 ring views 640x480..1920x1080")
    if name == "mp4x1080_3m":
        s = make_surfels(3_000_000, 0, True, 3, 0.1)
        t = make_surfels(3_000_000, 1, True, 3, 0.1)
        cams = ring_cameras([(1920, 1080)] * 4)
        return Workload(name, s, t, cams, "3,000,000 surfels in 64 clusters, SH deg 3, 4 views 1920x1080")
    if name == "full16_3m":  # the 16-view rig at half the surfels (deterministic-mode memory)
        s = make_surfels(3_000_000, 0, True, 3, 0.1)
        t = make_surfels(3_000_000, 1, True, 3, 0.1)
        rng = np.random.default_rng(7)
        res = [RING_RESOLUTIONS[i] for i in rng.integers(0, len(RING_RESOLUTIONS), 16)]
        cams = ring_cameras(res)
        return Workload(name, s, t, cams, "3,000,000 surfels in 64 clusters, SH deg 3, 16 views per step")
    if name == "full16_6m":
        s = make_surfels(6_000_000, 0, True, 3, 0.1)
        t = make_surfels(6_000_000, 1, True, 3, 0.1)
        rng = np.random.default_rng(7)
        res = [RING_RESOLUTIONS[i] for i in rng.integers(0, len(RING_RESOLUTIONS), 16)]
        cams = ring_cameras(res)
        return Workload(name, s, t, cams, "6,000,000 surfels in 64 clusters, SH deg 3, 16 views per step")
    raise KeyError(name)
