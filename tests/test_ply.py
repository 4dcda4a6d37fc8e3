"""Surfel PLY import/export through the C ABI (host-only, no GPU), restating
the reference's own tests: first_attempt/crates/gs-io/tests/ply_tests.rs
(in-memory fixtures with hand-verifiable values, error cases) and
writer_roundtrip.rs (write baked surfels, read back, compare activated
values). A GPU test saves a handle's surfels and loads them into another."""
import math
import struct

import numpy as np
import pytest

from splattar_b200 import GsError
from splattar_b200.rasterizer import read_ply, write_ply


def splat_ply(rows, rest_per_channel, extra_prop=None):
    names = ["x", "y", "z"]
    if extra_prop:
        names.append(extra_prop)
    names += [f"f_dc_{i}" for i in range(3)] + [f"f_rest_{i}" for i in range(rest_per_channel * 3)]
    names += ["opacity"] + [f"scale_{i}" for i in range(3)] + [f"rot_{i}" for i in range(4)]
    out = f"ply\nformat binary_little_endian 1.0\ncomment fixture\nelement vertex {len(rows)}\n".encode()
    for n in names:
        out += f"property float {n}\n".encode()
    out += b"end_header\n"
    for row in rows:
        assert len(row) == len(names)
        out += struct.pack(f"<{len(row)}f", *row)
    return out


def deg1_row():
    row = [1.0, 2.0, 3.0, 0.5, -0.5, 0.25]
    row += [i * 0.1 for i in range(1, 10)]
    row += [0.0]
    row += [math.log(0.1), math.log(0.2), math.log(0.3)]
    row += [1.0, 0.0, 0.0, 0.0]
    return row


def load_bytes(tmp_path, data, name="f.ply"):
    p = tmp_path / name
    p.write_bytes(data)
    return read_ply(str(p))


def test_splat_deg1_values_and_interleave(tmp_path):
    s = load_bytes(tmp_path, splat_ply([deg1_row()], 3))
    assert s["positions"].shape == (1, 3) and s["sh_coeffs"] == 4
    assert np.array_equal(s["positions"][0], [1.0, 2.0, 3.0])
    expect = [0.5, -0.5, 0.25, 0.1, 0.4, 0.7, 0.2, 0.5, 0.8, 0.3, 0.6, 0.9]
    assert np.allclose(s["sh"][0], expect, atol=1e-6)
    assert abs(s["opacities"][0] - 0.5) < 1e-6
    assert np.allclose(s["scales"][0], [0.1, 0.2, 0.3], atol=1e-6)
    assert np.allclose(s["quats"][0], [0, 0, 0, 1], atol=1e-6)  # rot_0 is w


def test_splat_nonidentity_quat_is_normalized_and_reordered(tmp_path):
    row = deg1_row()
    row[-4:] = [2.0, 0.0, 0.0, 2.0]
    q = load_bytes(tmp_path, splat_ply([row], 3))["quats"][0]
    inv = 1.0 / math.sqrt(2.0)
    assert abs(q[3] - inv) < 1e-6 and abs(q[2] - inv) < 1e-6 and abs(np.linalg.norm(q) - 1) < 1e-6


def test_degenerate_quat_falls_back_to_identity(tmp_path):
    row = deg1_row()
    row[-4:] = [0.0, 0.0, 0.0, 0.0]
    assert np.array_equal(load_bytes(tmp_path, splat_ply([row], 3))["quats"][0], [0, 0, 0, 1])


def test_splat_deg0_no_rest(tmp_path):
    row = [0.0, 0.0, 0.0, 0.5, 0.5, 0.5, 10.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0]
    s = load_bytes(tmp_path, splat_ply([row], 0))
    assert s["sh_coeffs"] == 1 and s["sh"].shape == (1, 3)
    assert s["opacities"][0] > 0.99 and np.array_equal(s["scales"][0], [1, 1, 1])


def test_extra_property_takes_offset_path_with_same_values(tmp_path):
    row = deg1_row()
    row.insert(3, 42.0)
    s = load_bytes(tmp_path, splat_ply([row], 3, "nx"))
    assert np.array_equal(s["positions"][0], [1.0, 2.0, 3.0])
    assert abs(s["sh"][0, 3] - 0.1) < 1e-6 and abs(s["sh"][0, 4] - 0.4) < 1e-6
    assert np.allclose(s["scales"][0], [0.1, 0.2, 0.3], atol=1e-6)


def _err(tmp_path, data):
    with pytest.raises(GsError) as e:
        load_bytes(tmp_path, data)
    return str(e.value)


def test_ascii_format_is_rejected(tmp_path):
    msg = _err(tmp_path, b"ply\nformat ascii 1.0\nelement vertex 0\nproperty float x\nend_header\n")
    assert "GS_ERR_FORMAT" in msg and "ascii" in msg


def test_truncated_payload_reports_eof(tmp_path):
    data = splat_ply([deg1_row(), deg1_row()], 3)[:-40]
    msg = _err(tmp_path, data)
    assert "expected 2" in msg


def test_missing_rot_is_unknown_layout(tmp_path):
    out = b"ply\nformat binary_little_endian 1.0\nelement vertex 0\n"
    for n in ["x", "y", "z", "f_dc_0", "f_dc_1", "f_dc_2", "opacity", "scale_0", "scale_1", "scale_2", "rot_0",
              "rot_1", "rot_2"]:
        out += f"property float {n}\n".encode()
    out += b"end_header\n"
    msg = _err(tmp_path, out)
    assert "rot_3" in msg and "rot_2" in msg


def test_garbage_is_not_ply(tmp_path):
    assert "not a ply" in _err(tmp_path, b"not a ply at all\n")


def test_wrong_rest_count_is_rejected(tmp_path):
    row = deg1_row()[:6] + [0.1] * 5 + deg1_row()[15:]
    names_rest = 5
    out = b"ply\nformat binary_little_endian 1.0\nelement vertex 1\n"
    for n in ["x", "y", "z", "f_dc_0", "f_dc_1", "f_dc_2"] + [f"f_rest_{i}" for i in range(names_rest)] + \
            ["opacity", "scale_0", "scale_1", "scale_2", "rot_0", "rot_1", "rot_2", "rot_3"]:
        out += f"property float {n}\n".encode()
    out += b"end_header\n" + struct.pack(f"<{len(row)}f", *row)
    assert "f_rest count 5" in _err(tmp_path, out)


def test_write_then_read_roundtrip(tmp_path):
    count = 3
    positions = (np.arange(count * 4) * 0.25).astype(np.float32).reshape(count, 4)
    scales = (0.05 + np.arange(count * 2) * 0.01).astype(np.float32).reshape(count, 2)
    quats = []
    for i in range(count):
        a = 0.3 + i
        quats.append([0.0, math.sin(a / 2), 0.0, math.cos(a / 2)])  # rotation about y
    quats = np.array(quats, np.float32)
    opac = np.array([0.25, 0.5, 0.9], np.float32)
    sh = np.sin(np.arange(count * 48) * 0.013).astype(np.float32).reshape(count, 48) * 0.4
    p = str(tmp_path / "roundtrip.ply")
    write_ply(p, positions, scales, quats, opac, sh)
    s = read_ply(p)
    assert s["positions"].shape[0] == count and s["sh_coeffs"] == 16
    assert np.abs(s["positions"] - positions[:, :3]).max() < 1e-6
    assert np.abs(s["scales"][:, :2] - scales).max() < 1e-6
    assert np.all(s["scales"][:, 2] < 1e-4), "third scale must be flattened"
    assert np.abs(s["opacities"] - opac).max() < 1e-5
    assert np.abs(s["quats"] - quats).max() < 1e-5
    assert np.abs(s["sh"] - sh).max() < 1e-6


@pytest.mark.gpu
def test_handle_save_and_load_ply(tmp_path):
    from gpu_util import raster_camera, scene_input
    from scenes import make_scene
    from splattar_b200 import Rasterizer
    scene, cam = make_scene(404, 50, 3, 64)
    a = Rasterizer(scene.n, 64, 64, 64 * scene.n)
    a.upload_scene(scene_input(scene))
    a.forward(raster_camera(cam, 3), scene.n)
    a.check()
    p = str(tmp_path / "scene.ply")
    a.save_ply(p, scene.n)
    b = Rasterizer(scene.n, 64, 64, 64 * scene.n)
    n = b.load_ply(p)
    assert n == scene.n
    b.forward(raster_camera(cam, 3), n)
    b.check()
    ia, ib = a.read("out_color", 4 * 64 * 64), b.read("out_color", 4 * 64 * 64)
    assert np.abs(ia - ib).max() < 1e-4
    for k, w in (("positions", 4), ("scales", 2), ("opacities", 1), ("sh", 48)):
        assert np.allclose(a.read(k, w * n), b.read(k, w * n), rtol=1e-5, atol=1e-6), k
    qa, qb = a.read("quats", 4 * n).reshape(n, 4), b.read("quats", 4 * n).reshape(n, 4)
    qa = qa / np.linalg.norm(qa, axis=1, keepdims=True)  # the reader normalises
    assert np.allclose(qa, qb, atol=1e-6)
