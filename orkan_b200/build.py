"""Build the Orkan-B200 shared libraries in-tree (nvcc for sm_100a + gcc for the C host layer).

Products (git-ignored, they travel with the source tree to GPU hosts):
  orkan_b200/liborkan_b200.so     LOG_TILE_DIM=5 (32x32 tiles, the reference Release geometry)
  orkan_b200/liborkan_b200_t3.so  LOG_TILE_DIM=3 (8x8 tiles, the reference Debug geometry)

The CUDA objects do not depend on LOG_TILE_DIM (the tile size is a kernel argument), so
they are compiled once and linked into both libraries; the C host layer is compiled
once per tile geometry.  Rebuilds are incremental on file modification times.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
INCLUDE = os.path.join(ROOT, "include")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I" + INCLUDE]
CC_FLAGS = ["-std=gnu17", "-O2", "-fPIC", "-Wall", "-Wno-unused-function", "-I" + INCLUDE,
            "-I" + os.path.join(CUDA_HOME, "include")]

CU_SOURCES = ["orkan_cu.cu", "scratch.cu", "noalloc.cu", "qaoa.cu", "mlp.cu", "sample.cu"]
C_SOURCES = ["runtime.c", "state.c", "gate.c", "fuse.c", "channel.c", "meas.c", "circ.c", "sample.c"]
LIBS = {5: "liborkan_b200.so", 3: "liborkan_b200_t3.so"}


def _headers():
    out = []
    for d in (os.path.join(CSRC, "cuda"), os.path.join(CSRC, "host"), INCLUDE):
        for f in os.listdir(d):
            if f.endswith((".h", ".cuh")):
                out.append(os.path.join(d, f))
    return out


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError("build step failed: " + os.path.basename(cmd[-1]))
    return r


def library_path(log_tile: int = 5) -> str:
    return os.path.join(PKG, LIBS[log_tile])


def build(verbose: bool = False, extra_cu=None, extra_c=None) -> list[str]:
    """Compile every CUDA and C source and link both libraries; returns their paths."""
    os.makedirs(BUILD, exist_ok=True)
    hdrs = _headers()
    cu_sources = CU_SOURCES + list(extra_cu or [])
    c_sources = C_SOURCES + list(extra_c or [])
    jobs = []
    cu_objs = []
    for src in cu_sources:
        s = os.path.join(CSRC, "cuda", src)
        o = os.path.join(BUILD, src + ".o")
        cu_objs.append(o)
        if _stale(o, [s] + hdrs):
            jobs.append([NVCC] + NVCC_FLAGS + ["-c", s, "-o", o])
    c_objs = {lt: [] for lt in LIBS}
    for lt in LIBS:
        for src in c_sources:
            s = os.path.join(CSRC, "host", src)
            o = os.path.join(BUILD, f"{src}.t{lt}.o")
            c_objs[lt].append(o)
            if _stale(o, [s] + hdrs):
                jobs.append(["gcc"] + CC_FLAGS + [f"-DLOG_TILE_DIM={lt}", "-c", s, "-o", o])
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 2)) as ex:
        for r in ex.map(_run, jobs):
            if verbose and (r.stdout or r.stderr):
                sys.stderr.write(r.stdout + r.stderr)
    outs = []
    for lt, name in LIBS.items():
        lib = os.path.join(PKG, name)
        objs = cu_objs + c_objs[lt]
        if _stale(lib, objs):
            _run([NVCC] + ARCH + ["-shared", "-o", lib] + objs + ["-Xlinker", "-Bsymbolic", "-lm"])
        outs.append(lib)
    return outs


if __name__ == "__main__":
    for p in build(verbose=True):
        print(p)
