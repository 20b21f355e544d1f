"""Builds libsurface_rt.so in-tree with nvcc for sm_100a.

    python -m surface_b200.build [--force]

Flags: -O3, -lineinfo, --fmad=false for the build and traversal sources (no
contraction, so float/double arithmetic rounds exactly like the reference's
x86-64 build), --fmad=true for the volume march (its parity bar is a
tolerance, and contraction shortens its arithmetic chains), static cudart,
hidden visibility except the extern "C" entry points of include/surface_rt.h.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
OBJDIR = os.path.join(ROOT, "_build", "surface_rt")
LIB = os.path.join(PKG, "libsurface_rt.so")

SOURCES = ["srt_build.cu", "srt_sort.cu", "srt_trace.cu", "srt_raysort.cu", "srt_volume.cu", "srt_batch.cu",
           "srt_spawn.cu", "srt_camera.cu", "srt_scene.cu", "srt_cache.cu", "srt_texture.cu",
           "srt_line.cu", "srt_solid.cu", "srt_isect.cu", "srt_capi.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC",
              "-Xcompiler", "-fvisibility=hidden", "-I" + INCLUDE]
FMAD = {"srt_volume.cu": "--fmad=true"}  # every other source: --fmad=false


def _nvcc():
    for c in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False):
    """Compile every translation unit whose sources changed, then link."""
    nvcc = _nvcc()
    os.makedirs(OBJDIR, exist_ok=True)
    headers = [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith((".cuh", ".h"))]
    headers.append(os.path.join(INCLUDE, "surface_rt.h"))
    objs = []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJDIR, src.replace(".cu", ".o"))
        objs.append(o)
        if force or _stale(o, [s] + headers):
            cmd = [nvcc, *NVCC_FLAGS, FMAD.get(src, "--fmad=false"), *ARCH, "-c", s, "-o", o]
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
    if force or _stale(LIB, objs):
        cmd = [nvcc, "-shared", *ARCH, "-cudart", "static", "-o", LIB, *objs]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
