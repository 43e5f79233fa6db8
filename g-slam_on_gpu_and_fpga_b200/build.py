"""Builds libgslam.so (sm_100a) and the GSLAM command-line program in-tree.

    python g-slam_on_gpu_and_fpga_b200/build.py [--force]

Outputs: g-slam_on_gpu_and_fpga_b200/lib/libgslam.so, g-slam_on_gpu_and_fpga_b200/bin/GSLAM and
the host-only dataset tool g-slam_on_gpu_and_fpga_b200/bin/gslam-data (g++).
nvcc cross-compiles for sm_100a without a GPU. Every translation unit is built
with -fmad=false: the FP64 path must round every product and sum separately to
match the reference's arithmetic; FP32 kernels call fused multiply-adds
explicitly where they want them.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INC = os.path.join(ROOT, "include")
OBJ = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "lib", "libgslam.so")
CLI = os.path.join(PKG, "bin", "GSLAM")
DATA_TOOL = os.path.join(PKG, "bin", "gslam-data")

NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-fmad=false", "-Xcompiler", "-fPIC",
          "-Xcompiler", "-ffp-contract=off", "-I", CSRC, "-I", INC]

LIB_SOURCES = ["structure.cpp", "kernels.cu", "pcg.cu", "pcg_resident.cu", "pcg_mixed.cu", "pcg_static.cu",
               "adjoint.cu", "batch.cu", "gj.cu", "api.cu", "batch_api.cu", "dropin.cu", "logio.cpp"]
CLI_SOURCES = ["cli.cpp"]
DATA_SOURCES = ["datasets.cpp"]
# the dataset tool reproduces CPython's float arithmetic: C library math calls kept as calls
DATA_FLAGS = ["-O2", "-std=c++17", "-ffp-contract=off", "-fno-builtin", "-fno-fast-math"]


def _newer(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _headers() -> list[str]:
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs += [os.path.join(INC, f) for f in os.listdir(INC) if f.endswith(".h")]
    return hs


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    os.makedirs(os.path.dirname(CLI), exist_ok=True)
    headers = _headers()
    jobs = []
    objs = []
    for src in LIB_SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(OBJ, src + ".o")
        objs.append(obj)
        if force or _newer(obj, [path] + headers):
            jobs.append([NVCC, *ARCH, *COMMON, "-c", path, "-o", obj])
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        list(ex.map(_run, jobs))
    if force or jobs or _newer(LIB, objs):
        _run([NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-cudart", "static"])
    cli_src = [os.path.join(CSRC, s) for s in CLI_SOURCES]
    if force or _newer(CLI, cli_src + [LIB] + headers):
        _run([NVCC, *ARCH, *COMMON, "-o", CLI, *cli_src, "-L", os.path.dirname(LIB), "-lgslam",
              "-Xlinker", "-rpath,$ORIGIN/../lib"])
    data_src = [os.path.join(CSRC, s) for s in DATA_SOURCES]
    if force or _newer(DATA_TOOL, data_src):
        _run([os.environ.get("CXX", "g++"), *DATA_FLAGS, "-o", DATA_TOOL, *data_src, "-lm"])
    if verbose:
        print("built", LIB, "and", CLI)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
