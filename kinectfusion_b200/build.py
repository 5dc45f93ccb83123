"""Builds the sm_100a CUDA library (kinectfusion_b200/libkf_b200.so) in-tree.

Every translation unit is compiled with --fmad=false (plus the default
-prec-div=true / -prec-sqrt=true): the kernels evaluate the reference's float
expressions with separately rounded multiplies and adds, which is what makes
them bit-comparable with the host implementation.
"""

from __future__ import annotations

import concurrent.futures
import os
import pathlib
import shutil
import subprocess
import sys

HERE = pathlib.Path(__file__).resolve().parent
CSRC = HERE / "csrc"
LIB = HERE / "libkf_b200.so"
BUILD_DIR = HERE / "_build"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
HOST_CXX = "/usr/bin/g++"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--fmad=false", "-prec-div=true", "-prec-sqrt=true",
         "-ftz=false", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2", "-ccbin", HOST_CXX,
         "--expt-relaxed-constexpr"]


def _sources():
    return sorted(CSRC.glob("*.cu"))


def _needs_build() -> bool:
    if not LIB.exists():
        return True
    stamp = LIB.stat().st_mtime
    deps = list(CSRC.glob("*")) + [HERE.parent / "include" / "kf_b200.h", pathlib.Path(__file__)]
    return any(d.stat().st_mtime > stamp for d in deps if d.exists())


def _compile(src: pathlib.Path, extra: list[str]) -> pathlib.Path:
    obj = BUILD_DIR / (src.stem + ".o")
    cmd = [NVCC, *ARCH, *FLAGS, *extra, "-c", str(src), "-o", str(obj)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{res.stdout}\n{res.stderr}")
    if res.stderr.strip():
        sys.stderr.write(res.stderr)
    return obj


def build(force: bool = False, verbose_ptxas: bool = False) -> pathlib.Path:
    if not force and not _needs_build():
        return LIB
    BUILD_DIR.mkdir(exist_ok=True)
    extra = ["-Xptxas", "-v"] if verbose_ptxas else []
    with concurrent.futures.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as pool:
        objs = list(pool.map(lambda s: _compile(s, extra), _sources()))
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [NVCC, *ARCH, "-shared", "-ccbin", HOST_CXX, "-o", str(tmp), *map(str, objs), "-lz"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
    os.replace(tmp, LIB)
    shutil.rmtree(BUILD_DIR, ignore_errors=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose_ptxas="--ptxas" in sys.argv)
    print(LIB)
