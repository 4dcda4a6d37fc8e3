"""Trainer schedule on the host, through the C ABI
(first_attempt/crates/gs-train/src/trainer.rs): scene extent (:740-746),
schedule_t with and without the anneal tail (:407-416, tests :425-455 ported
with their constants), and the exponential position-LR decay (:1150)."""
import numpy as np

from splattar_b200 import position_lr, scene_extent, schedule_t


def test_anneal_schedule_is_continuous_monotonic_and_completes():
    iters, start, length = 20_000, 6_000, 2_000
    a = (start, length, start / iters)
    assert abs(schedule_t(start, iters) - schedule_t(start, iters, a)) < 1e-6
    prev = -np.inf
    for i in range(start, start + length + 1):
        t = schedule_t(i, iters, a)
        assert t >= prev - 1e-7, (i, prev, t)
        prev = t
    assert abs(schedule_t(start + length, iters, a) - 1.0) < 1e-6
    assert abs(schedule_t(start + 3 * length, iters, a) - 1.0) < 1e-6


def test_nominal_schedule_is_unchanged():
    assert schedule_t(0, 7000) == 0.0
    assert abs(schedule_t(3500, 7000) - 0.5) < 1e-6
    assert abs(schedule_t(7000, 7000) - 1.0) < 1e-6


def test_scene_extent_and_position_lr():
    rng = np.random.default_rng(0)
    p = rng.uniform(-2, 3, (1000, 4)).astype(np.float32)
    want = max(float(np.linalg.norm(p[:, :3].max(0) - p[:, :3].min(0))), 1e-3) * 0.5
    assert abs(scene_extent(p) - want) < 1e-5 * want
    assert abs(scene_extent(np.zeros((5, 3), np.float32)) - 0.5e-3) < 1e-9  # the 1e-3 floor, halved
    ext = scene_extent(p)
    for t in (0.0, 0.25, 1.0):
        want = 1.6e-4 * ext * 0.01 ** t
        assert abs(position_lr(1.6e-4, ext, 0.01, t) - want) < 1e-6 * want  # computed in f32
