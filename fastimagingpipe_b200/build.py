"""Builds libfip_b200.so and the sharedlibrary_gpu command line, in tree.

    python -m fastimagingpipe_b200.build

Compiles every CUDA translation unit for sm_100a only.  fip_plain.cu gets
--use_fast_math (the reference's own build flags: the plain form reproduces
its FP32 arithmetic); the other units are IEEE.  Objects go to
fastimagingpipe_b200/_build/, the library and the CLI next to this file.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
REPO = os.path.dirname(HERE)
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
LIB = os.path.join(HERE, "libfip_b200.so")
CLI = os.path.join(HERE, "bin", "sharedlibrary_gpu")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
          "-I" + os.path.join(REPO, "include"), "-I" + CSRC] + ARCH
UNITS = {
    "fip_plain.cu": ["--use_fast_math"],
    "fip_precise.cu": [],
    "fip_host.cu": [],
    "fip_noalloc.cu": [],
    "fip_server.cu": [],
    "fip_locate.cu": [],
}
HOST_CXX = ["fits_io.cpp"]


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _headers():
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))] + [
        os.path.join(REPO, "include", "fip.h")]


def build(verbose_ptxas: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(os.path.dirname(CLI), exist_ok=True)
    hdrs = _headers()
    objs = []
    for src, extra in UNITS.items():
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src.replace(".cu", ".o"))
        objs.append(o)
        if _stale(o, [s] + hdrs) or verbose_ptxas:
            cmd = [NVCC, "-c", s, "-o", o] + COMMON + extra
            if verbose_ptxas:
                cmd += ["-Xptxas", "-v"]
            _run(cmd)
    for src in HOST_CXX:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src.replace(".cpp", ".o"))
        objs.append(o)
        if _stale(o, [s] + hdrs):
            _run([NVCC, "-c", s, "-o", o, "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
                  "-Wno-deprecated-gpu-targets",
                  "-I" + os.path.join(REPO, "include"), "-I" + CSRC])
    if _stale(LIB, objs):
        _run([NVCC, "-shared", "-o", LIB] + objs + ARCH +
             ["-L" + os.path.join(CUDA_HOME, "lib64"), "-lcufft",
              "-Xlinker", "-rpath", "-Xlinker", os.path.join(CUDA_HOME, "lib64")])
    cli_src = os.path.join(CSRC, "sharedlibrary_gpu.cpp")
    cli_deps = [cli_src, LIB, os.path.join(CSRC, "fits_io.cpp")] + hdrs
    if os.path.exists(cli_src) and _stale(CLI, cli_deps):
        _run([NVCC, cli_src, "-o", CLI, "-O2", "-std=c++17", "-Wno-deprecated-gpu-targets", "-I" + os.path.join(REPO, "include"),
              "-I" + CSRC, "-L" + HERE, "-lfip_b200", "-Xlinker", "-rpath", "-Xlinker",
              "$ORIGIN/..", "-Xlinker", "-rpath", "-Xlinker",
              os.path.join(CUDA_HOME, "lib64")])
    return LIB


if __name__ == "__main__":
    build(verbose_ptxas="-v" in sys.argv)
