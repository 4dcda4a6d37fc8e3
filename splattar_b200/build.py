"""Builds libgs_cuda.so in-tree for sm_100a with nvcc.

Each translation unit compiles separately (in parallel); ``gs_project.cu`` is
built with ``--fmad=false`` so its tile-rect and depth-key arithmetic is free
of fused multiply-adds and matches an f32 restatement bit for bit (its adjoint
is in ``gs_project_bwd.cu``, built normally). ptxas
resource usage of every kernel is written to ``_build/ptxas_<unit>.txt``.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libgs_cuda.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

UNITS = {
    "gs_api.cu": [],
    "gs_project.cu": ["--fmad=false"],
    "gs_project_bwd.cu": [],
    "gs_raster.cu": [],
    "gs_raster_t8.cu": [],
    "gs_raster_t32.cu": [],
    "gs_sort.cu": [],
    "gs_loss.cu": [],
    "gs_optim.cu": [],
    "gs_noalloc.cu": [],
    "gs_mcmc.cu": [],
    "gs_ply.cpp": [],
}
HEADERS = ["gs_common.cuh", "gs_kernels.h", "gs_geom.cuh", "gs_raster.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xptxas", "-v", "-I", INCLUDE]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def _deps_mtime() -> float:
    paths = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "gs_cuda.h"), __file__]
    return max(os.path.getmtime(p) for p in paths)


def _compile(unit: str, extra: list[str], force: bool) -> str:
    src = os.path.join(CSRC, unit)
    obj = os.path.join(BUILD, os.path.splitext(unit)[0] + ".o")
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), _deps_mtime()):
        return obj
    cmd = [_nvcc(), *FLAGS, *extra, "-c", src, "-o", obj]
    res = subprocess.run(cmd, capture_output=True, text=True)
    with open(os.path.join(BUILD, "ptxas_" + os.path.splitext(unit)[0] + ".txt"), "w") as f:
        f.write(" ".join(cmd) + "\n" + res.stdout + res.stderr)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {unit}:\n{res.stderr[-6000:]}")
    return obj


def build(force: bool = False, jobs: int = 6) -> str:
    """Compile every CUDA unit and link libgs_cuda.so; returns its path."""
    os.makedirs(BUILD, exist_ok=True)
    with ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(lambda kv: _compile(kv[0], kv[1], force), UNITS.items()))
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        tmp = LIB + ".tmp"
        cmd = [_nvcc(), *ARCH, "-shared", "-o", tmp, *objs, "-Xcompiler", "-fPIC"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stderr[-4000:]}")
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
