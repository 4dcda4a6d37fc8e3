"""B200-native differentiable 2D-Gaussian-surfel training step.

The compute path is libgs_cuda.so (hand-written sm_100a CUDA kernels behind
the C ABI of include/gs_cuda.h); this package is its host-side mirror of the
reference's Rasterizer / TileBinner / SsimLoss / Optimizer surface.
"""
from ._lib import GsError, lib  # noqa: F401
from .rasterizer import (AdamSettings, RasterCamera, Rasterizer, SceneInput, StepSettings, TileBinner,  # noqa: F401
                         adam_flat, camera_array, camera_rotation, exclusive_scan_u32, position_lr, radix_sort_pairs,
                         scene_extent, schedule_t)

__all__ = ["GsError", "lib", "Rasterizer", "RasterCamera", "SceneInput", "TileBinner", "AdamSettings",
           "StepSettings", "radix_sort_pairs", "exclusive_scan_u32", "adam_flat", "camera_array", "camera_rotation",
           "scene_extent", "schedule_t", "position_lr"]
