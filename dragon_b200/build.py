"""In-tree build of the CUDA library (sm_100a) behind include/dragon_gpu.h.

Each translation unit is compiled on its own, then linked into
dragon_b200/libdragon_gpu.so:
  * the FP64 kernels with --fmad=false, so no a*b+c is fused: together with
    IEEE division and square root this keeps the FP64 path's arithmetic
    identical to the reference's (compiled without contraction);
  * the mixed-precision kernels (step_mixed.cu, step_mhd_mixed.cu,
    step1d_mixed.cu, step3d_mixed.cu, step3d_mhd_mixed.cu, batch_mixed.cu) with FMA contraction and fast
    single-precision division / square root; the division, square-root and
    denormal flags act on FP32 only, and the contraction also fuses the FP64
    arithmetic of these files (the mixed path is not held to bit parity).
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(ROOT, "_build", "obj")
LIB = os.path.join(HERE, "libdragon_gpu.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
BASE = ["-std=c++17", "-O3", "-lineinfo", *ARCH, "-Xcompiler", "-fPIC", "-I" + os.path.join(ROOT, "include")]
EXACT = ["--fmad=false"]
FAST32 = ["--fmad=true", "-prec-div=false", "-prec-sqrt=false", "-ftz=true"]
PER_FILE = {"step_mixed.cu": FAST32, "step_mhd_mixed.cu": FAST32, "step1d_mixed.cu": FAST32,
            "batch_mixed.cu": FAST32, "step3d_mixed.cu": FAST32, "step3d_mhd_mixed.cu": FAST32}


def _sources():
    return [f for f in sorted(os.listdir(CSRC)) if f.endswith(".cu")]


def _headers():
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))] + [
        os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include")) if f.endswith(".h")] + [
        os.path.abspath(__file__)]


def _deps():
    return [os.path.join(CSRC, f) for f in _sources()] + _headers()


def _stale(src: str, obj: str, newest_header: float) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return os.path.getmtime(src) > t or newest_header > t


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(p) > t for p in _deps())


def _host_stale() -> bool:
    deps = [HOST_SRC, DIST_SRC, os.path.join(ROOT, "include", "dragon", "dragon.hpp"),
            os.path.join(ROOT, "include", "dragon", "hoard.hpp"),
            os.path.join(ROOT, "include", "dragon", "dist.hpp"), os.path.join(ROOT, "include", "dragon_gpu.h"), LIB]
    outs = list(HOST_LIBS.values()) + [os.path.join(HERE, "libdragon_dist.so"), os.path.join(HERE, "libdragon_dist_mhd.so")]
    return any(not os.path.exists(o) or any(os.path.getmtime(d) > os.path.getmtime(o) for d in deps) for o in outs)


def build(force: bool = False, verbose: bool = False) -> str:
    """Compiles dragon_b200/libdragon_gpu.so with nvcc (cross-compiles without a GPU)."""
    if not force and not needs_build():
        if _host_stale():
            build_host(verbose=verbose)
        return LIB
    nvcc = os.environ.get("NVCC", "nvcc")
    os.makedirs(OBJ, exist_ok=True)

    newest_header = max(os.path.getmtime(h) for h in _headers())

    def compile_one(src):
        obj = os.path.join(OBJ, src.replace(".cu", ".o"))
        if not force and not _stale(os.path.join(CSRC, src), obj, newest_header):
            return obj
        cmd = [nvcc, *BASE, *PER_FILE.get(src, EXACT), "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True, cwd=CSRC)
        return obj

    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(compile_one, _sources()))
    subprocess.run([nvcc, *ARCH, "-shared", "-o", LIB + ".tmp", *objs, "-ldl", "-lz"], check=True)
    os.replace(LIB + ".tmp", LIB)
    build_host(force=True, verbose=verbose)
    return LIB


HOST_SRC = os.path.join(HERE, "host", "dragon_host.cpp")
DIST_SRC = os.path.join(HERE, "host", "dragon_dist.cpp")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
HOST_LIBS = {"": os.path.join(HERE, "libdragon_host.so"), "-DMHD": os.path.join(HERE, "libdragon_host_mhd.so")}


def build_host(force: bool = False, verbose: bool = False) -> None:
    """Compiles the C++23 host layer (include/dragon/dragon.hpp) over the C ABI:
    libdragon_host.so (hydro) and libdragon_host_mhd.so (built with MHD), both
    linked against libdragon_gpu.so in the same directory."""
    cxx = os.environ.get("CXX", "g++")
    deps = [HOST_SRC, os.path.join(ROOT, "include", "dragon", "dragon.hpp"), os.path.join(ROOT, "include", "dragon", "hoard.hpp"),
            os.path.join(ROOT, "include", "dragon_gpu.h"), LIB]
    for flag, out in HOST_LIBS.items():
        if not force and os.path.exists(out) and all(os.path.getmtime(d) <= os.path.getmtime(out) for d in deps):
            continue
        cmd = [cxx, "-std=c++23", "-O2", "-fPIC", "-Wall", "-Wextra", "-shared", *([flag] if flag else []),
               "-I" + os.path.join(ROOT, "include"), HOST_SRC, "-L" + HERE, "-ldragon_gpu", "-Wl,-rpath,$ORIGIN",
               "-o", out + ".tmp"]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
        os.replace(out + ".tmp", out)
    build_dist(force=force, verbose=verbose)


def build_dist(force: bool = False, verbose: bool = False) -> None:
    """Compiles the C++ DistGrid (include/dragon/dist.hpp) over NCCL:
    libdragon_dist.so and libdragon_dist_mhd.so, linked against the host layer
    of the same physics, libdragon_gpu.so, libcudart and libnccl."""
    cxx = os.environ.get("CXX", "g++")
    deps = [DIST_SRC, os.path.join(ROOT, "include", "dragon", "dist.hpp"), os.path.join(ROOT, "include", "dragon", "dragon.hpp"),
            LIB]
    for flag, host_out in HOST_LIBS.items():
        sfx = "_mhd" if flag else ""
        out = os.path.join(HERE, f"libdragon_dist{sfx}.so")
        if not force and os.path.exists(out) and all(os.path.getmtime(d) <= os.path.getmtime(out) for d in deps):
            continue
        cmd = [cxx, "-std=c++23", "-O2", "-fPIC", "-Wall", "-Wextra", "-shared", *([flag] if flag else []),
               "-I" + os.path.join(ROOT, "include"), "-I" + os.path.join(CUDA_HOME, "include"), DIST_SRC,
               "-L" + HERE, f"-ldragon_host{sfx}", "-ldragon_gpu", "-L" + os.path.join(CUDA_HOME, "lib64"), "-lcudart",
               "-lnccl", "-Wl,-rpath,$ORIGIN", "-Wl,-rpath," + os.path.join(CUDA_HOME, "lib64"), "-o", out + ".tmp"]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
        os.replace(out + ".tmp", out)


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
