"""Build libmarfa_gpu.so in-tree with nvcc for sm_100a.

    python -m marfa_b200.build          # or marfa_b200.build.build()

The library is plain CUDA C++ with a C ABI (include/marfa_gpu.h); it is
loaded with ctypes, so no Python extension module is involved.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libmarfa_gpu.so"
PROBE = PKG / "libmarfa_probe.so"   # FMA throughput probe of the benchmark
CLI = PKG / "marfa"
SOURCES = ["marfa_kernels.cu", "marfa_adjoint.cu", "marfa_api.cu", "marfa_static.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def flags(extra=()):
    return ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                   "-I", str(ROOT / "include"), "-I", str(CSRC), *extra]


def _compile(src: str, extra) -> Path:
    obj = BUILD / (Path(src).stem + ".o")
    cmd = [nvcc(), *flags(extra), "-c", str(CSRC / src), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj


def stale() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    if not CLI.exists() or not PROBE.exists():
        return True
    deps = list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + \
        list(CSRC.glob("*.cpp")) + \
        list((ROOT / "include").glob("*.h")) + [Path(__file__)]
    return any(d.stat().st_mtime > t for d in deps)


def build(force: bool = False, extra=()) -> Path:
    if not force and not stale():
        return LIB
    BUILD.mkdir(exist_ok=True)
    with ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        objs = list(ex.map(lambda s: _compile(s, extra), SOURCES))
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc(), *ARCH, "-shared", "-cudart", "static", "-o", str(tmp), *map(str, objs)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    # the benchmark's FMA throughput probe (a library of its own, not part of
    # the line-by-line interface)
    cmd = [nvcc(), *flags(), "-shared", "-cudart", "static", str(CSRC / "marfa_probe.cu"), "-o", str(PROBE)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode:
        raise RuntimeError(f"probe build failed:\n{r.stdout}\n{r.stderr}")
    # the `marfa` command (host driver over the C ABI)
    cmd = [nvcc(), "-O2", "-std=c++17", "-I", str(ROOT / "include"), str(CSRC / "marfa_cli.cpp"),
           "-o", str(CLI), "-L", str(PKG), "-lmarfa_gpu", "-Xlinker", "-rpath=$ORIGIN"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode:
        raise RuntimeError(f"marfa command build failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    force = "--force" in sys.argv
    print(build(force=force))
