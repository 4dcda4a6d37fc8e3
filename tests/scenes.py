"""Seeded micro-scene generators shared by the parity and gradient tests.

``make_scene`` restates the reference tests' generator
(crates/gs-kernels/tests/common/mod.rs:7-82 and the gradcheck variant at
crates/gs-cpu-ref/tests/gradcheck.rs:10-85): a 64-bit xorshift (13, 7, 17)
mapped to [0, 1) by ``(x >> 11) / 2**53``, a camera jittered around the origin,
and surfels placed inside the view frustum at depths 2..6.
"""
from __future__ import annotations

import numpy as np

from oracle import Camera, Scene

_M64 = (1 << 64) - 1


class XorShift:
    def __init__(self, seed: int):
        self.s = seed & _M64

    def next(self) -> float:
        x = self.s
        x ^= (x << 13) & _M64
        x ^= x >> 7
        x ^= (x << 17) & _M64
        self.s = x
        return (x >> 11) / float(1 << 53)

    def uniform(self, lo, hi):
        return lo + (hi - lo) * self.next()


def quat_to_mat(q):
    q = np.asarray(q, np.float64)
    x, y, z, w = q / np.linalg.norm(q)
    return np.array([
        [1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
        [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
        [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)],
    ])


def make_scene(seed: int, n: int, sh_degree: int, size: int, focal=None, scale_hi=0.5):
    """Scene + camera as the reference's GPU parity tests draw them.

    ``focal=None`` gives ``0.9 * size`` (raster_parity); the gradcheck tests use
    ``focal=30`` and ``scale_hi=0.4``.
    """
    rng = XorShift(seed)
    center = np.array([rng.uniform(-0.3, 0.3) for _ in range(3)])
    quat = np.array([rng.uniform(-0.08, 0.08) for _ in range(3)] + [1.0])
    f = size * 0.9 if focal is None else float(focal)
    r = quat_to_mat(quat)
    ncoef = (sh_degree + 1) ** 2
    pos = np.zeros((n, 3)); scales = np.zeros((n, 2)); quats = np.zeros((n, 4))
    opac = np.zeros(n); sh = np.zeros((n, 48))
    for i in range(n):
        z = -rng.uniform(2.0, 6.0)
        ext = -z * (size * 0.5) / f * 0.7
        p_cam = np.array([rng.uniform(-ext, ext), rng.uniform(-ext, ext), z])
        coeffs = [rng.uniform(-0.8, 0.8) for _ in range(3)]
        for _ in range(1, ncoef):
            coeffs += [rng.uniform(-0.25, 0.25) for _ in range(3)]
        sh[i, :len(coeffs)] = coeffs
        pos[i] = center + r @ p_cam
        scales[i] = [rng.uniform(0.1, scale_hi), rng.uniform(0.1, scale_hi)]
        quats[i] = [rng.uniform(-1, 1), rng.uniform(-1, 1), rng.uniform(-1, 1), rng.uniform(-1, 1) + 1.5]
        opac[i] = rng.uniform(0.25, 0.85)
    scene = Scene(pos, scales, quats, opac, sh, sh_degree)
    cam = Camera(center, quat, f, size, size)
    return scene, cam


def make_weights(seed: int, n: int, lo=-1.0, hi=1.0, dims=3):
    rng = XorShift(seed)
    return np.array([[rng.uniform(lo, hi) for _ in range(dims)] for _ in range(n)])
