"""Shared helpers of the GPU parity tests: f64 oracle scenes → float32 inputs
of the C ABI (the reference's to_gpu, crates/gs-kernels/tests/common/mod.rs:95-134),
and one-call forward/backward runs through splattar_b200.Rasterizer."""
import numpy as np

import oracle
from splattar_b200 import RasterCamera, Rasterizer, SceneInput


def scene_input(scene: oracle.Scene) -> SceneInput:
    ncoef = (scene.sh_degree + 1) ** 2
    return SceneInput(scene.pos.astype(np.float32), scene.scales.astype(np.float32), scene.quat.astype(np.float32),
                      scene.opacity.astype(np.float32), scene.sh[:, :3 * ncoef].astype(np.float32), ncoef)


def raster_camera(cam: oracle.Camera, sh_degree: int) -> RasterCamera:
    return RasterCamera(tuple(np.float32(cam.center)), tuple(np.float32(cam.quat)), float(np.float32(cam.focal)),
                        sh_degree, cam.width, cam.height)


def f32_scene(scene: oracle.Scene) -> oracle.Scene:
    """The scene rounded to the float32 values the GPU receives, in float64."""
    r = lambda a: a.astype(np.float32).astype(np.float64)  # noqa: E731
    return oracle.Scene(r(scene.pos), r(scene.scales), r(scene.quat), r(scene.opacity), r(scene.sh), scene.sh_degree)


def f32_cam(cam: oracle.Camera) -> oracle.Camera:
    r = lambda a: np.asarray(a, np.float32).astype(np.float64)  # noqa: E731
    return oracle.Camera(r(cam.center), r(cam.quat), float(np.float32(cam.focal)), cam.width, cam.height)


def forward(scene, cam, rast=None, **kw):
    n = scene.n
    if rast is None:
        # 64 entries per surfel at 16-pixel tiles (the reference trainer's
        # budget), scaled by the tile-count ratio for smaller tiles.
        tile = kw.get("tile", 16)
        rast = Rasterizer(n, cam.width, cam.height, kw.pop("max_entries", n * 64 * max(1, (16 // tile) ** 2)), **kw)
    rast.upload_scene(scene_input(scene))
    rast.forward(raster_camera(cam, scene.sh_degree), n)
    rast.check()
    P = cam.width * cam.height
    out = dict(color=rast.read("out_color", 4 * P).reshape(P, 4), aux=rast.read("out_aux", 4 * P).reshape(P, 4),
               normal=rast.read("out_normal", 4 * P).reshape(P, 4), ncontrib=rast.read("out_ncontrib", P))
    return rast, out


def backward(rast, scene, dl_dcolor4, dl_dnormal4=None):
    P = dl_dcolor4.shape[0]
    rast.write("dl_dcolor", dl_dcolor4.astype(np.float32).reshape(-1))
    dn = np.zeros((P, 4), np.float32) if dl_dnormal4 is None else dl_dnormal4.astype(np.float32)
    rast.write("dl_dnormal", dn.reshape(-1))
    n = scene.n
    rast.backward(n)
    rast.check()
    return dict(pos=rast.read("grad_pos", 4 * n).reshape(n, 4)[:, :3],
                scales=rast.read("grad_scales", 2 * n).reshape(n, 2),
                quat=rast.read("grad_quat", 4 * n).reshape(n, 4), opacity=rast.read("grad_opacity", n),
                sh=rast.read("grad_sh", 48 * n).reshape(n, 48), cam=rast.read("grad_cam", 16))


class GradCheck:
    """raster_parity.rs:83-114: err ≤ 1e-5 + rel_tol·max(|gpu|, |cpu|).

    With `outliers` > 0, up to that fraction of the entries may exceed the
    tolerance, none by more than `outlier_rel` of the array's largest
    gradient (f32 against f64 on scenes dense enough to hold near-grazing
    surfels, whose ray-branch gradients scale with 1/det and amplify f32
    rounding)."""

    def __init__(self, rel_tol, outliers=0.0, outlier_rel=2e-2):
        self.rel_tol = rel_tol
        self.outliers, self.outlier_rel = outliers, outlier_rel
        self.worst, self.label = 0.0, ""

    def check(self, label, gpu, cpu):
        gpu = np.asarray(gpu, np.float64).ravel()
        cpu = np.asarray(cpu, np.float64).ravel()
        denom = np.maximum(np.abs(gpu), np.abs(cpu))
        err = np.abs(gpu - cpu)
        rel = np.where(denom > 1e-6, err / np.maximum(denom, 1e-30), 0.0)
        sel = err > 1e-6
        if sel.any() and rel[sel].max() > self.worst:
            self.worst, self.label = float(rel[sel].max()), f"{label}[{int(np.argmax(np.where(sel, rel, 0)))}]"
        bad = err > 1e-5 + self.rel_tol * denom
        if self.outliers > 0:
            far = err > 1e-5 + self.outlier_rel * float(np.abs(cpu).max(initial=0.0))
            assert not far.any(), (f"{label}: {int(far.sum())} beyond {self.outlier_rel}, first at "
                                   f"{int(np.argmax(far))}: gpu {gpu[far][0]:.6e} vs cpu {cpu[far][0]:.6e}")
            assert bad.sum() <= self.outliers * bad.size, (f"{label}: {int(bad.sum())} of {bad.size} beyond "
                                                           f"{self.rel_tol}")
            return
        assert not bad.any(), (f"{label}: {int(bad.sum())} mismatches, first at {int(np.argmax(bad))}: gpu "
                               f"{gpu[bad][0]:.6e} vs cpu {cpu[bad][0]:.6e}")
