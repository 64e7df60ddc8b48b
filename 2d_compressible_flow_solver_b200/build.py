"""Builds the stage engine's shared library, libcfs.so, in this folder.

Kernels are compiled by nvcc for sm_100a only (``-gencode
arch=compute_100a,code=sm_100a``); kernels_exact.cu with ``-fmad=false`` so the
CFS_FP64_EXACT path keeps the reference's rounding sequence; march_inst.cu once
per form (FP32-mixed, FP64) and row-march feature set (0..7), sixteen objects.
Stale objects are compiled in parallel.  Host C++ is
compiled by g++ with ``-ffp-contract=off`` (the immersed-boundary set-up must
reproduce the reference's doubles).  Objects go to ``_build/``; a file is
rebuilt when it or a header it may include is newer than its object.

Usage: ``python build.py [--force]``.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
INCLUDE = HERE.parent / "include"
OUT_DIR = HERE / "_build"
LIB = HERE / "libcfs.so"
CUDA_HOME = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
NVCC = str(CUDA_HOME / "bin" / "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

# (object name, source, extra nvcc flags)
CU_UNITS = [
    ("kernels_exact.cu", "kernels_exact.cu", ["-fmad=false"]),
    ("kernels_fast.cu", "kernels_fast.cu", []),
    ("cfl_static.cu", "cfl_static.cu", ["-fmad=false"]),
    ("fp_peaks.cu", "fp_peaks.cu", []),
    ("ib_device.cu", "ib_device.cu", ["-fmad=false"]),
] + [
    (f"march_{form}_{feat}.cu", "march_inst.cu",
     [f"-DCFS_MARCH_POL={pol}", f"-DCFS_MARCH_FEAT={feat}", f"-DCFS_MARCH_FN=launch_march_{form}_{feat}"])
    for form, pol in (("f32", "PolF32"), ("f64", "PolF64")) for feat in range(8)
]
CPP_SOURCES = ["cfs_api.cpp", "cfs_batch.cpp", "ib_setup.cpp", "tma_maps.cpp", "host_stage.cpp"]


def _headers() -> list[Path]:
    return sorted(CSRC.glob("*.h")) + sorted(CSRC.glob("*.cuh")) + sorted(INCLUDE.glob("*.h"))


def _stale(src: Path, obj: Path, deps: list[Path]) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return src.stat().st_mtime > t or any(d.stat().st_mtime > t for d in deps)


def _run(cmd: list[str]) -> None:
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build(force: bool = False, verbose_ptxas: bool = False) -> Path:
    """Compiles what is stale and links libcfs.so; returns its path."""
    OUT_DIR.mkdir(exist_ok=True)
    deps = _headers()
    objs, jobs = [], []
    for name, source, extra in CU_UNITS:
        src, obj = CSRC / source, OUT_DIR / (name + ".o")
        objs.append(obj)
        if force or _stale(src, obj, deps):
            cmd = [NVCC, "-std=c++17", "-O3", *ARCH, "-lineinfo", "-Xcompiler", "-fPIC",
                   f"-I{CSRC}", f"-I{INCLUDE}", *extra, "-c", str(src), "-o", str(obj)]
            if verbose_ptxas:
                cmd.insert(1, "-Xptxas=-v")
            jobs.append(cmd)
    for name in CPP_SOURCES:
        src, obj = CSRC / name, OUT_DIR / (name + ".o")
        objs.append(obj)
        if force or _stale(src, obj, deps):
            jobs.append(["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-fPIC", "-pthread", "-Wall", "-Wextra",
                         f"-I{CSRC}", f"-I{INCLUDE}", f"-I{CUDA_HOME / 'include'}", "-c", str(src), "-o", str(obj)])
    relink = force or not LIB.exists() or bool(jobs)
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        for f in [ex.submit(_run, cmd) for cmd in jobs]:
            f.result()
    if relink:
        _run([NVCC, "-shared", *ARCH, "-Xcompiler", "-fPIC", *map(str, objs), "-lpthread", "-o", str(LIB)])
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose_ptxas="--ptxas" in sys.argv)
