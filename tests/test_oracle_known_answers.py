"""Known-answer checks that pin the oracle's building blocks to the reference's
own unit tests, restated with the same inputs and tolerances:

* SH colour: crates/gs-core/src/sh.rs:84-125 (degree-0 view independence,
  degree-1 along +z, the +0.5 offset and the clamp at 0); the SH basis of
  crates/gs-cpu-ref/src/math.rs:127-156 uses the same constants and signs;
* math: crates/gs-cpu-ref/src/math.rs:199-267 (quaternion, triple-product
  and SH-basis gradients against central differences, h = 1e-6);
* cameras: crates/gs-core/src/camera.rs:68-101 (look_at faces its target,
  focal length from the vertical field of view), for the synthetic rigs.

The SH normalisation constants are also checked against their closed forms
1/(2 sqrt(pi)) and sqrt(3)/(2 sqrt(pi)).
"""
import math

import numpy as np

import oracle

SH_C0 = 1.0 / (2.0 * math.sqrt(math.pi))
SH_C1 = math.sqrt(3.0) / (2.0 * math.sqrt(math.pi))


def test_sh_constants_closed_form():
    b, _ = oracle.sh_basis(1, [0.0, 0.0, 1.0])
    assert abs(b[0] - SH_C0) < 1e-12
    assert abs(b[2] - SH_C1) < 1e-12  # +z term
    assert abs(SH_C0 - 0.28209479) < 1e-8 and abs(SH_C1 - 0.48860251) < 1e-8


def test_sh_degree0_is_view_independent():
    coeffs = [[1.0, -0.5, 0.25]]
    a, _ = oracle.sh_color(0, coeffs, [0.0, 0.0, 1.0])
    b, _ = oracle.sh_color(0, coeffs, [0.5773503, -0.5773503, 0.5773503])
    assert np.array_equal(a, b)
    assert abs((a[0] - 0.5) - SH_C0) < 1e-6


def test_sh_degree1_axis_direction():
    coeffs = np.zeros((4, 3))
    coeffs[0] = 0.2
    coeffs[1] = 10.0  # y term: no contribution along +z
    coeffs[2] = 0.3
    coeffs[3] = 10.0  # x term: no contribution along +z
    got, _ = oracle.sh_color(1, coeffs, [0.0, 0.0, 1.0])
    assert abs((got[0] - 0.5) - (SH_C0 * 0.2 + SH_C1 * 0.3)) < 1e-6


def test_sh_color_offset_and_clamp():
    c, clamped = oracle.sh_color(0, [[-10.0, 0.0, 0.0]], [0.0, 0.0, 1.0])
    assert c[0] == 0.0 and clamped[0]
    assert abs(c[1] - 0.5) < 1e-6 and not clamped[1]


def test_quat_grad_matches_fd():
    q = np.array([0.3, -0.5, 0.2, 0.8])
    w = np.array([[0.3, -1.2, 0.7], [0.9, 0.1, -0.4], [-0.6, 0.8, 0.5]])  # columns

    def loss(qq):
        return float(np.sum(oracle.quat_to_mat(qq) * w))

    an = oracle.quat_grad(q, w)
    h = 1e-6
    for k in range(4):
        e = np.zeros(4)
        e[k] = h
        fd = (loss(q + e) - loss(q - e)) / (2 * h)
        assert abs(fd - an[k]) < 1e-7, (k, fd, an[k])


def test_triple_grads_match_fd():
    a, b, c = np.array([0.3, -0.7, 1.1]), np.array([-0.2, 0.9, 0.4]), np.array([0.8, 0.1, -0.5])
    _, ga, gb, gc = oracle.triple(a, b, c)
    h = 1e-6
    for i in range(3):
        e = np.zeros(3)
        e[i] = h
        assert abs((oracle.triple(a + e, b, c)[0] - oracle.triple(a - e, b, c)[0]) / (2 * h) - ga[i]) < 1e-8
        assert abs((oracle.triple(a, b + e, c)[0] - oracle.triple(a, b - e, c)[0]) / (2 * h) - gb[i]) < 1e-8
        assert abs((oracle.triple(a, b, c + e)[0] - oracle.triple(a, b, c - e)[0]) / (2 * h) - gc[i]) < 1e-8


def test_sh_basis_grad_matches_fd():
    d = np.array([0.48, -0.6, 0.64])
    for degree in range(4):
        _, g = oracle.sh_basis(degree, d)
        h = 1e-6
        for i in range(3):
            e = np.zeros(3)
            e[i] = h
            bp, _ = oracle.sh_basis(degree, d + e)
            bm, _ = oracle.sh_basis(degree, d - e)
            fd = (bp - bm) / (2 * h)
            assert np.all(np.abs(fd - g[:, i]) < 1e-6), (degree, i)


def test_quat_to_mat_is_rotation_of_normalised_quaternion():
    rng = np.random.default_rng(1)
    for _ in range(10):
        q = rng.normal(size=4) * 3
        r = oracle.quat_to_mat(q)
        assert np.allclose(r @ r.T, np.eye(3), atol=1e-12)
        assert abs(np.linalg.det(r) - 1) < 1e-12
        assert np.allclose(oracle.quat_to_mat(q / np.linalg.norm(q)), r, atol=1e-14)


def test_synthetic_look_at_faces_target_and_fov_focal():
    from splattar_b200.synthetic import look_at
    cam = look_at((5.0, 3.0, 5.0), (0.0, 0.0, 0.0), 1600, 900)
    r = oracle.quat_to_mat(np.array(cam.quat, np.float64))  # [col][row]: col 2 = camera +z
    forward = -r[2]
    expect = -np.array(cam.center) / np.linalg.norm(cam.center)
    assert np.linalg.norm(forward - expect) < 1e-5
    # 60 degree vertical field of view by default: f = 0.5 H / tan(30 deg)
    assert abs(cam.focal - 0.5 * 900 / math.tan(math.radians(30))) < 1e-3
    cam90 = look_at((0.0, 0.0, 5.0), (0.0, 0.0, 0.0), 1600, 900, focal=0.5 * 900 / math.tan(math.radians(45)))
    assert abs(cam90.focal - 450.0) < 1e-3
