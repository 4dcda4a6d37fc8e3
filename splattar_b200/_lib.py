"""ctypes binding of libgs_cuda.so (include/gs_cuda.h).

The library is the product: there is no Python or CPU fallback. Loading fails
loudly when the shared object has not been built.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgs_cuda.so")

GS_OK = 0
STATUS = {0: "GS_OK", 1: "GS_ERR_INVALID_ARG", 2: "GS_ERR_CAPACITY", 3: "GS_ERR_CUDA", 4: "GS_ERR_DEVICE_TIMEOUT",
          5: "GS_ERR_NONFINITE", 6: "GS_ERR_STATE", 7: "GS_ERR_IO", 8: "GS_ERR_FORMAT"}

PREC = {"f32": 0, "f16": 1, "bf16": 2}
FLAG_DETERMINISTIC = 1
FLAG_PERSISTENT = 2
FLAG_COLOR_ONLY = 4
FLAG_TIGHT_BINNING = 8
FLAG_STORED_STATE = 16
FLAG_FULL_LISTS = 32

BUF = {
    "positions": 0, "scales": 1, "quats": 2, "opacities": 3, "sh": 4, "out_color": 5, "out_aux": 6,
    "out_normal": 7, "out_ncontrib": 8, "dl_dcolor": 9, "dl_dnormal": 10, "grad_pos": 11, "grad_scales": 12,
    "grad_quat": 13, "grad_opacity": 14, "grad_sh": 15, "grad_cam": 16, "target": 17, "ranges": 18,
    "sorted_items": 19, "entry_count": 20, "loss": 21, "raw_pos": 22, "raw_scales": 23, "raw_quat": 24,
    "raw_opacity": 25, "raw_sh": 26, "rects": 27, "depth_keys": 28, "depth_order": 29,
    "grad_norm_sum": 30, "m_pos": 31, "m_scales": 32, "m_quat": 33, "m_opacity": 34, "m_sh": 35, "v_pos": 36,
    "v_scales": 37, "v_quat": 38, "v_opacity": 39, "v_sh": 40, "normal_loss": 41,
    "incomplete_tiles": 42, "tile_cut": 43,
}


class GsError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


class RasterConfig(C.Structure):
    _fields_ = [("capacity", C.c_uint32), ("width", C.c_uint32), ("height", C.c_uint32), ("max_views", C.c_uint32),
                ("max_pixels", C.c_uint64), ("max_entries", C.c_uint64), ("tile", C.c_uint32),
                ("batch", C.c_uint32), ("precision", C.c_uint32), ("flags", C.c_uint32),
                ("pixels_per_thread", C.c_uint32)]


class Camera(C.Structure):
    _fields_ = [("quat", C.c_float * 4), ("center", C.c_float * 3), ("focal", C.c_float), ("width", C.c_uint32),
                ("height", C.c_uint32), ("sh_degree", C.c_uint32)]


class SceneInputC(C.Structure):
    _fields_ = [("positions", C.c_void_p), ("scales", C.c_void_p), ("quats", C.c_void_p), ("opacities", C.c_void_p),
                ("sh", C.c_void_p), ("sh_coeffs", C.c_uint32), ("n", C.c_uint32)]


class McmcConfig(C.Structure):
    _fields_ = [("dead_threshold", C.c_float), ("split_ratio", C.c_float)]


class AdamConfig(C.Structure):
    _fields_ = [("lr", C.c_float * 5), ("reg", C.c_float * 5), ("beta1", C.c_float), ("beta2", C.c_float),
                ("eps", C.c_float)]


class StepConfig(C.Structure):
    _fields_ = [("w_l1", C.c_float), ("w_ssim", C.c_float), ("adam", AdamConfig), ("form", C.c_uint32),
                ("loss", C.c_uint32)]


class Anneal(C.Structure):
    _fields_ = [("start", C.c_uint32), ("len", C.c_uint32), ("t0", C.c_float)]


class DensifyConfig(C.Structure):
    _fields_ = [("grad_threshold", C.c_float), ("opacity_threshold", C.c_float)]


_lib = None


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with splattar_b200.build.build() (nvcc, sm_100a)")
    L = C.CDLL(LIB_PATH)
    vp, u32, u64, f32, i32 = C.c_void_p, C.c_uint32, C.c_uint64, C.c_float, C.c_int
    sigs = {
        "gs_rasterizer_create": [C.POINTER(RasterConfig), C.POINTER(vp)],
        "gs_rasterizer_destroy": [vp],
        "gs_rasterizer_upload_scene": [vp, C.POINTER(SceneInputC), vp],
        "gs_rasterizer_set_lambda_dist": [vp, f32],
        "gs_rasterizer_set_wait_limits": [vp, u64, u64],
        "gs_rasterizer_forward": [vp, C.POINTER(Camera), u32, u32, vp],
        "gs_rasterizer_backward": [vp, u32, vp],
        "gs_rasterizer_buffer": [vp, i32, C.POINTER(vp), C.POINTER(C.c_size_t)],
        "gs_rasterizer_view_offset": [vp, u32, C.POINTER(u64), C.POINTER(u32)],
        "gs_rasterizer_read": [vp, i32, u64, vp, C.c_size_t, vp],
        "gs_rasterizer_write": [vp, i32, u64, vp, C.c_size_t, vp],
        "gs_rasterizer_read_async": [vp, i32, u64, vp, C.c_size_t, vp],
        "gs_rasterizer_write_async": [vp, i32, u64, vp, C.c_size_t, vp],
        "gs_rasterizer_check": [vp, vp],
        "gs_last_error": [vp, C.c_char_p, C.c_size_t],
        "gs_loss_l1_ssim": [vp, f32, f32, vp],
        "gs_optimizer_init": [vp, u32, vp],
        "gs_optimizer_step": [vp, C.POINTER(AdamConfig), u32, vp],
        "gs_adam_flat": [vp, vp, vp, vp, vp, u64, u32, f32, f32, f32, f32, f32, u32, vp],
        "gs_train_step": [vp, C.POINTER(Camera), u32, u32, C.POINTER(StepConfig), vp],
        "gs_train_step_profiled": [vp, C.POINTER(Camera), u32, u32, C.POINTER(StepConfig), vp,
                                   C.POINTER(C.c_float), C.POINTER(u32)],
        "gs_densify_prune": [vp, C.POINTER(DensifyConfig), u32, C.POINTER(u32), vp],
        "gs_autotune": [vp, C.POINTER(Camera), u32, u32, vp, C.POINTER(u32)],
        "gs_set_launch_shapes": [vp, C.POINTER(u32)],
        "gs_raster_work": [vp, C.POINTER(u64), vp],
        "gs_autotune_tiles": [vp, C.POINTER(Camera), u32, u32, vp, C.POINTER(u32), C.POINTER(f32)],
        "gs_set_tile_size": [vp, u32],
        "gs_tile_size": [vp],
        "gs_binner_create": [u32, u64, u32, C.POINTER(vp)],
        "gs_binner_destroy": [vp],
        "gs_binner_encode": [vp, vp, vp, u32, u32, vp],
        "gs_binner_buffer": [vp, u32, C.POINTER(vp), C.POINTER(C.c_size_t)],
        "gs_radix_sort_pairs": [vp, vp, u64, u32, vp],
        "gs_radix_sort_pairs_noalloc": [vp, vp, u64, u32, vp],
        "gs_exclusive_scan_u32": [vp, vp, u64, vp, vp],
        "gs_camera_rotation": [C.POINTER(Camera), C.POINTER(C.c_float)],
        "gs_loss_normal": [vp, f32, f32, vp],
        "gs_camera_step_grad": [C.POINTER(f32), C.POINTER(f32), C.POINTER(f32)],
        "gs_camera_adam6": [C.POINTER(f32), C.POINTER(f32), u32, C.POINTER(f32), f32, f32, C.POINTER(f32)],
        "gs_camera_apply_step": [C.POINTER(Camera), C.POINTER(f32)],
        "gs_scene_extent": [C.POINTER(f32), u32, u32, C.POINTER(f32)],
        "gs_schedule_t": [u32, u32, C.POINTER(Anneal), C.POINTER(f32)],
        "gs_position_lr": [f32, f32, f32, f32, C.POINTER(f32)],
        "gs_mcmc_seed": [vp, u64, vp],
        "gs_mcmc_relocate": [vp, C.POINTER(McmcConfig), u32, vp],
        "gs_mcmc_stats": [vp, C.POINTER(u32), C.POINTER(u64), vp],
        "gs_mcmc_noise": [vp, u32, u32, f32, f32, vp],
        "gs_ply_write": [C.c_char_p, u32, vp, vp, vp, vp, vp],
        "gs_ply_info": [C.c_char_p, C.POINTER(u32), C.POINTER(u32)],
        "gs_ply_read": [C.c_char_p, u32, vp, vp, vp, vp, vp, C.POINTER(u32)],
        "gs_rasterizer_save_ply": [vp, C.c_char_p, u32, vp],
        "gs_rasterizer_load_ply": [vp, C.c_char_p, C.POINTER(u32), vp],
        "gs_shutdown": [],
    }
    for name, args in sigs.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = C.c_int
    L.gs_version.argtypes = []
    L.gs_version.restype = C.c_char_p
    _lib = L
    return L


def last_error(handle=None) -> str:
    buf = C.create_string_buffer(1024)
    lib().gs_last_error(handle, buf, 1024)
    return buf.value.decode(errors="replace")


def check(status: int, handle=None):
    if status != GS_OK:
        raise GsError(status, last_error(handle))


def exported_symbols() -> list[str]:
    """Names of the C entry points (for the ABI-completeness test)."""
    lib()
    return ["gs_version"] + [
        "gs_rasterizer_create", "gs_rasterizer_destroy", "gs_rasterizer_upload_scene", "gs_rasterizer_set_lambda_dist",
        "gs_rasterizer_set_wait_limits", "gs_rasterizer_forward", "gs_rasterizer_backward", "gs_rasterizer_buffer", "gs_rasterizer_view_offset",
        "gs_rasterizer_read", "gs_rasterizer_write", "gs_rasterizer_read_async", "gs_rasterizer_write_async",
        "gs_rasterizer_check", "gs_last_error", "gs_loss_l1_ssim", "gs_optimizer_init", "gs_optimizer_step",
        "gs_adam_flat", "gs_train_step", "gs_train_step_profiled", "gs_densify_prune", "gs_autotune", "gs_autotune_tiles", "gs_set_tile_size", "gs_tile_size", "gs_set_launch_shapes", "gs_raster_work", "gs_binner_create",
        "gs_binner_destroy", "gs_binner_encode", "gs_binner_buffer", "gs_radix_sort_pairs", "gs_radix_sort_pairs_noalloc",
        "gs_exclusive_scan_u32",
        "gs_camera_rotation", "gs_shutdown", "gs_loss_normal", "gs_camera_step_grad", "gs_camera_adam6",
        "gs_camera_apply_step", "gs_scene_extent", "gs_schedule_t", "gs_position_lr", "gs_mcmc_seed", "gs_mcmc_relocate", "gs_mcmc_stats", "gs_mcmc_noise",
        "gs_ply_write", "gs_ply_info", "gs_ply_read", "gs_rasterizer_save_ply",
        "gs_rasterizer_load_ply"]
