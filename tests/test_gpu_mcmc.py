"""MCMC relocation and exploration noise on the GPU against the restatement
of the reference's host sampler and copy kernels (oracle.mcmc_pairs /
oracle.mcmc_apply: first_attempt/crates/gs-train/src/trainer.rs:1558-1689,
shaders/relocate.wgsl) and of shaders/mcmc.wgsl: the same (dead, alive,
mode) pairs and generator state for the same seed, identical copies, the
relocation arithmetic within f32 rounding, zeroed moments."""
import numpy as np
import pytest

import oracle
from splattar_b200 import Rasterizer
from splattar_b200.synthetic import look_at, make_surfels

pytestmark = pytest.mark.gpu

CLASSES = (("pos", "positions", 4), ("scales", "scales", 2), ("quat", "quats", 4), ("opacity", "opacities", 1),
           ("sh", "sh", 48))


def _setup(n=4000, seed=3):
    s = make_surfels(n, seed, False, 3, 0.1)
    rng = np.random.default_rng(seed)
    dead = rng.choice(n, 300, replace=False)
    s.opacities[dead] = rng.uniform(0.0005, 0.004, 300).astype(np.float32)
    big = rng.choice(np.setdiff1d(np.arange(n), dead), 25, replace=False)
    s.scales[big] *= 30.0
    cam = look_at((0.0, 0.0, -3.0), (0.0, 0.0, 0.0), 128, 128, sh_degree=3)
    r = Rasterizer(n, 128, 128, 96 * n)
    r.upload_scene(s.scene_input())
    r.optimizer_init(n)
    # Two plain optimizer steps make the moments nonzero.
    from splattar_b200.rasterizer import AdamSettings
    for _ in range(2):
        r.forward(cam, n)
        w = rng.uniform(-1, 1, (128 * 128, 4)).astype(np.float32)
        w[:, 3] = 0
        r.write("dl_dcolor", w.ravel())
        r.write("dl_dnormal", np.zeros(4 * 128 * 128, np.float32))
        r.backward(n)
        r.optimizer_step(AdamSettings(), n)
    r.check()
    return r, n


def _state(r, n):
    st = {}
    for name, act, w in CLASSES:
        st[name] = r.read(f"raw_{name}", w * n).reshape(n, w) if w > 1 else r.read(f"raw_{name}", n)
        st["act_" + name] = r.read(act, w * n).reshape(n, w) if w > 1 else r.read(act, n)
        for mv in ("m", "v"):
            a = r.read(f"{mv}_{name}", w * n)
            st[f"{mv}_{name}"] = a.reshape(n, w) if w > 1 else a
    return st


def test_mcmc_relocation_matches_reference_sampler():
    r, n = _setup()
    before = _state(r, n)
    seed = 0x1234567890ABCDEF
    pairs, state_after = oracle.mcmc_pairs(before["act_opacity"], before["act_scales"], seed, 0.005, 8.0)
    assert any(m == 0 for _, _, m in pairs) and any(m == 1 for _, _, m in pairs), "vacuous case"
    want = oracle.mcmc_apply({k: v for k, v in before.items() if not k.startswith("act_")}, before["act_opacity"], pairs)
    r.mcmc_seed(seed)
    r.mcmc_relocate(n, 0.005, 8.0)
    r.check()
    got = _state(r, n)
    stats = r.mcmc_stats()
    assert stats["relocated"] == sum(1 for p in pairs if p[2] == 0)
    assert stats["split"] == sum(1 for p in pairs if p[2] == 1)
    assert stats["dead"] == int((before["act_opacity"] < np.float32(0.005)).sum())
    assert stats["rng_state"] == state_after
    touched = sorted({i for d, a, _ in pairs for i in (d, a)})
    untouched = np.setdiff1d(np.arange(n), touched)
    for k in want:
        g, w = got[k], want[k]
        assert np.array_equal(g[untouched], before[k][untouched]), k
        assert np.allclose(g[touched], w[touched], rtol=2e-6, atol=1e-7), (k, np.abs(g - w).max())
    # activated copies follow the raw values
    assert np.array_equal(got["act_pos"], got["pos"])
    assert np.allclose(got["act_scales"], np.exp(got["scales"]), rtol=1e-6)
    assert np.allclose(got["act_opacity"], 1 / (1 + np.exp(-got["opacity"].astype(np.float64))), rtol=1e-6)
    assert np.array_equal(got["act_sh"], got["sh"])


def test_mcmc_relocation_continues_the_generator():
    r, n = _setup(seed=4)
    seed = 88172645463325252
    r.mcmc_seed(seed)
    st = _state(r, n)
    _, s1 = oracle.mcmc_pairs(st["act_opacity"], st["act_scales"], seed)
    r.mcmc_relocate(n)
    assert r.mcmc_stats()["rng_state"] == s1
    st = _state(r, n)
    pairs2, s2 = oracle.mcmc_pairs(st["act_opacity"], st["act_scales"], s1)
    r.mcmc_relocate(n)
    assert r.mcmc_stats()["rng_state"] == s2


def _pcg(v):
    v = np.uint32(v)
    with np.errstate(over="ignore"):
        state = v * np.uint32(747796405) + np.uint32(2891336453)
        word = ((state >> ((state >> np.uint32(28)) + np.uint32(4))) ^ state) * np.uint32(277803737)
    return (word >> np.uint32(22)) ^ word


def test_mcmc_noise_matches_restatement():
    r, n = _setup(n=2000, seed=5)
    st = _state(r, n)
    seed, sigma, k = 0x9E3779B9 * 7 & 0xFFFFFFFF, 0.01, 5.0
    r.mcmc_noise(n, seed, sigma, k)
    r.check()
    got = r.read("raw_pos", 4 * n).reshape(n, 4)
    f = np.float32
    want = st["pos"].copy()
    for i in range(n):
        s = st["act_scales"][i]
        amp = f(sigma) * (f(0.5) * (s[0] + s[1])) * np.exp(f(-k) * st["act_opacity"][i], dtype=np.float32)
        if not amp > 0:
            continue
        base = _pcg(np.uint32(i) ^ np.uint32(seed))
        for d, salt in enumerate((0x68BC21EB, 0x2C1B3C6D, 0x1F123BB5)):
            acc, sv = f(0.0), np.uint32(base ^ np.uint32(salt))
            for _ in range(4):
                sv = _pcg(sv)
                acc += f(int(sv) & 0xFFFFFF) / f(16777216.0)
            want[i, d] += amp * (acc - f(2.0))
    assert np.allclose(got, want, rtol=1e-6, atol=1e-7)
    assert np.array_equal(r.read("positions", 4 * n).reshape(n, 4), got)
