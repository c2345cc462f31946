"""Builds the in-tree native libraries of the package.

  libtoothpaste_gpu.so   CUDA kernels + C ABI (include/toothpaste_gpu.h), sm_100a
  libtoothpaste_host.so  C++ drop-in operator classes over that C ABI

Each .cu unit compiles separately (the per-ring-size kernel units in parallel)
and is rebuilt only when a source or header is newer than its object.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
HOST = PKG / "host"
OBJ = PKG / "_build"
GPU_LIB = PKG / "libtoothpaste_gpu.so"
HOST_LIB = PKG / "libtoothpaste_host.so"

NVCC = os.environ.get("NVCC", "nvcc")
CUDA_HOME = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
CXX = os.environ.get("CXX", "g++")
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC",
    f"-I{ROOT / 'include'}",
]


def _newest(paths) -> float:
    return max((p.stat().st_mtime for p in paths), default=0.0)


def _run(cmd: list[str]) -> str:
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"build failed: {' '.join(cmd)}\n{res.stdout}\n{res.stderr}")
    return res.stdout + res.stderr


def build_gpu(force: bool = False, verbose: bool = False, jobs: int | None = None) -> Path:
    OBJ.mkdir(exist_ok=True)
    headers = list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + [ROOT / "include" / "toothpaste_gpu.h"]
    hdr_time = _newest(headers)
    units = sorted(CSRC.glob("*.cu"))
    todo = []
    for u in units:
        o = OBJ / (u.stem + ".o")
        if force or not o.exists() or o.stat().st_mtime < max(u.stat().st_mtime, hdr_time):
            todo.append((u, o))
    extra = ["-Xptxas", "-v"] if verbose else []

    def compile_one(item):
        u, o = item
        return u.name, _run([NVCC, *NVCC_FLAGS, *extra, "-c", str(u), "-o", str(o)])

    if todo:
        with cf.ThreadPoolExecutor(max_workers=jobs or min(len(todo), os.cpu_count() or 4)) as ex:
            for name, log in ex.map(compile_one, todo):
                if verbose:
                    print(f"== {name}\n{log}", file=sys.stderr)
    objs = [OBJ / (u.stem + ".o") for u in units]
    if force or not GPU_LIB.exists() or GPU_LIB.stat().st_mtime < _newest(objs):
        _run([NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", str(GPU_LIB),
              *map(str, objs), "-lcudart"])
    return GPU_LIB


def build_host(force: bool = False) -> Path | None:
    srcs = sorted(HOST.glob("*.cpp"))
    if not srcs:
        return None
    deps = srcs + list(HOST.glob("*.h")) + [ROOT / "include" / "toothpaste_gpu.h", GPU_LIB]
    if force or not HOST_LIB.exists() or HOST_LIB.stat().st_mtime < _newest(deps):
        _run([CXX, "-std=c++20", "-O2", "-fPIC", "-shared", f"-I{ROOT / 'include'}", f"-I{HOST}",
              f"-I{CUDA_HOME / 'include'}", *map(str, srcs), "-o", str(HOST_LIB), f"-L{PKG}",
              "-ltoothpaste_gpu", f"-L{CUDA_HOME / 'lib64'}", "-lcudart", "-Wl,-rpath,$ORIGIN"])
    return HOST_LIB


def build(force: bool = False, verbose: bool = False) -> None:
    build_gpu(force=force, verbose=verbose)
    build_host(force=force)


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
