"""The C-ABI library loads without a GPU and exports every entry point that
include/gs_cuda.h declares; the ctypes binding types every one of them. Only
host-only entry points are called here (no device work)."""
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "gs_cuda.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:gs_status|const char\*)\s+(gs_\w+)\s*\(", text, flags=re.M)))


@pytest.fixture(scope="module")
def L():
    from splattar_b200 import build as b
    b.build()
    from splattar_b200 import _lib
    return _lib.lib()


def test_header_declares_the_reference_surface():
    names = declared_functions()
    for must in ("gs_rasterizer_create", "gs_rasterizer_forward", "gs_rasterizer_backward", "gs_loss_l1_ssim",
                 "gs_optimizer_step", "gs_train_step", "gs_densify_prune", "gs_binner_encode",
                 "gs_radix_sort_pairs", "gs_exclusive_scan_u32", "gs_last_error"):
        assert must in names


def test_library_exports_every_declared_symbol(L):
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing


def test_binding_types_every_declared_symbol(L):
    from splattar_b200 import _lib
    bound = set(_lib.exported_symbols())
    assert set(declared_functions()) <= bound, sorted(set(declared_functions()) - bound)
    for n in declared_functions():
        assert getattr(L, n).restype is not None


def test_version_string(L):
    v = L.gs_version().decode()
    assert "sm_100a" in v or "gs_cuda" in v


def test_null_handles_are_rejected_without_device_work(L):
    import ctypes as C
    from splattar_b200 import _lib
    arr = (C.c_uint32 * 4)(128, 1, 64, 4)
    assert L.gs_set_launch_shapes(None, arr) == 1
    assert L.gs_rasterizer_destroy(None) in (0, 1)
    assert L.gs_rasterizer_check(None, None) == 1
    assert L.gs_autotune(None, None, 0, 0, None, None) == 1
    assert L.gs_binner_encode(None, None, None, 0, 0, None) == 1
    buf = C.create_string_buffer(256)
    assert L.gs_last_error(None, buf, 256) == 0
    assert _lib.STATUS[1] == "GS_ERR_INVALID_ARG"


def test_camera_rotation_host_only_matches_f32_restatement(L):
    import oracle
    from splattar_b200.rasterizer import RasterCamera, camera_rotation
    rng = np.random.default_rng(3)
    for _ in range(20):
        q = rng.normal(size=4) * rng.uniform(0.2, 3.0)
        cam = RasterCamera(center=(0.0, 0.0, 0.0), quat=tuple(q.tolist()), focal=100.0, sh_degree=0, width=64, height=64)
        got = np.asarray(camera_rotation(cam), dtype=np.float32)
        ref = np.asarray(oracle.camera_rotation_f32(q), dtype=np.float32)
        assert np.array_equal(got.reshape(-1), ref.reshape(-1))
