"""Build librakali.so (sm_100a) in-tree with nvcc.

Usage: python -m rakali_b200.build [--force] [--jobs N]

The FP64 step and kernel-level translation units are compiled with
--fmad=false so every a*b+c rounds twice, as the reference's arithmetic
does; the FP32 surface form uses contracted, flush-to-zero arithmetic; the
host-only units are compiled by nvcc as well so the library links against
the static CUDA runtime.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG.parent / "_build" / "rakali_b200"
LIB = PKG / "librakali.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
          "--expt-relaxed-constexpr"]
# translation units with their extra flags
UNITS = {
    "rkb_step_f64.cu": ["--fmad=false"],
    "rkb_kernel_api.cu": ["--fmad=false"],
    "rkb_adjoint.cu": ["--fmad=false"],
    "rkb_gauges.cu": ["--fmad=false"],
    # FP32 surface form: contracted multiply-adds, flush-to-zero, approximate
    # reciprocal and square root (the well-balanced products are written
    # with explicit round-to-nearest intrinsics and are never contracted)
    "rkb_step_f32.cu": ["-ftz=true", "-prec-div=false", "-prec-sqrt=false"],
    # FP32 adjoint batches: FP32 arithmetic with fast division and square root,
    # uncontracted, so the fused and the taped forward kernels round alike
    "rkb_adjoint32.cu": ["--fmad=false", "-ftz=true", "-prec-div=false", "-prec-sqrt=false"],
    "rkb_sim.cu": [],
    "rkb_batch.cu": [],
    "rkb_api.cu": [],
    "rkb_config.cpp": [],
    "rkb_netcdf.cpp": [],
}


def nvcc():
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(exe).exists():
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build librakali.so")
    return exe


def _deps_newer(src: Path, obj: Path) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    for f in list(CSRC.glob("*.h")) + list(CSRC.glob("*.hpp")) + list(CSRC.glob("*.cuh")) + \
            [PKG.parent / "include" / "rakali.h", src]:
        if f.exists() and f.stat().st_mtime > t:
            return True
    return False


def compile_unit(name: str, extra: list[str], force: bool) -> Path:
    src = CSRC / name
    obj = BUILD / (name + ".o")
    if force or _deps_newer(src, obj):
        cmd = [nvcc(), *ARCH, *COMMON, *extra, "-x", "cu", "-c", str(src), "-o", str(obj)]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"nvcc failed for {name}:\n{res.stdout}\n{res.stderr}")
    return obj


def build(force: bool = False, jobs: int | None = None) -> Path:
    BUILD.mkdir(parents=True, exist_ok=True)
    jobs = jobs or min(len(UNITS), os.cpu_count() or 4)
    with cf.ThreadPoolExecutor(jobs) as ex:
        objs = list(ex.map(lambda kv: compile_unit(kv[0], kv[1], force), UNITS.items()))
    newest = max(o.stat().st_mtime for o in objs)
    if force or not LIB.exists() or LIB.stat().st_mtime < newest:
        tmp = LIB.with_suffix(".so.tmp")
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(tmp), *map(str, objs), "-cudart", "static"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=None)
    a = ap.parse_args()
    print(build(a.force, a.jobs))
    sys.exit(0)
