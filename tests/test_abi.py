"""The C ABI library: loads, exports every entry point include/*.h declares,
record layouts agree with the header, and it fails loudly (no CPU fallback)
when no CUDA device is present."""
import ctypes as C
import glob
import os
import re
import subprocess

import numpy as np
import pytest

from surface_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = []
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names += re.findall(r"SRT_API\s+[\w\s\*]+?\b(srt_\w+)\s*\(", src)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    L = _lib.load()
    decl = declared_symbols()
    assert len(decl) >= 25
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.library_path()],
                         capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\sT\s+(srt_\w+)", out))
    missing = [n for n in decl if n not in exported]
    assert not missing, missing
    for n in decl:
        getattr(L, n)  # resolvable through ctypes
    # the Python binding declares exactly the header's entry points
    assert sorted(_lib.exported_symbols()) == decl


def test_record_layouts_match_header():
    assert _lib.RAY_DTYPE.itemsize == 32
    assert _lib.HIT_DTYPE.itemsize == 16
    assert C.sizeof(_lib.TraceOpts) == 6 * 8 + 8 + 8
    assert _lib.ISECT_DTYPE.itemsize == 80
    assert _lib.VOL_DTYPE.itemsize == 4 * 4 + 12 * 4 + 3 * 4
    from oracle import oracle as O
    assert O.RAY_DTYPE == _lib.RAY_DTYPE and O.HIT_DTYPE == _lib.HIT_DTYPE
    assert O.ISECT_DTYPE == _lib.ISECT_DTYPE
    assert O.VOL_DTYPE == _lib.VOL_DTYPE


def test_header_layouts_compile():
    """sizeof/offsetof of the header's records as a C compiler lays them out."""
    src = r"""
#include <stddef.h>
#include <stdio.h>
#include "surface_rt.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu\n", sizeof(srt_ray), sizeof(srt_hit), sizeof(srt_isect),
         sizeof(srt_trace_opts), offsetof(srt_trace_opts, isect), offsetof(srt_isect, d));
  return 0;
}
"""
    import tempfile
    with tempfile.TemporaryDirectory() as td:
        c = os.path.join(td, "l.c")
        open(c, "w").write(src)
        exe = os.path.join(td, "l")
        subprocess.run(["gcc", "-I" + os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()
    assert [int(x) for x in out] == [32, 16, 80, 64, 56, 64]


REF_RENDER = os.path.join(os.environ.get("SURFACE_REF", os.path.join(ROOT, "..", "reference")),
                          "render")


@pytest.mark.skipif(not os.path.exists(os.path.join(REF_RENDER, "render_accel_triangle.h")),
                    reason="reference tree absent")
def test_dropin_header_compiles_against_reference_headers():
    """include/surface_rt_accel.hpp (GpuTriangleAccel, GpuTetraAccel,
    GpuParticleAccel) compiles inside the reference's render/ headers, the way
    a SURFACE maintainer would include it, and its members have the reference
    accels' signatures."""
    src = r"""
#include "surface_rt_accel.hpp"
using namespace lsgl::render;
template <typename T, typename P, typename O> void sig() {
  bool (T::*b)(const P *, const O &) = &T::Build32;
  bool (T::*t)(Intersection &, Ray &) const = &T::Traverse;
  void (T::*x)(double *, double *) const = &T::BoundingBox;
  bool (T::*d)(const char *) = &T::Dump;
  (void)b; (void)t; (void)x; (void)d;
}
int main() {
  sig<GpuTriangleAccel, Mesh, TriangleBuildOptions>();
  sig<GpuTetraAccel, Tetrahedron, TetraBuildOptions>();
  sig<GpuParticleAccel, Particles, ParticleBuildOptions>();
  sig<TriangleAccel, Mesh, TriangleBuildOptions>();
  return 0;
}
"""
    import tempfile
    with tempfile.TemporaryDirectory() as td:
        c = os.path.join(td, "shim.cc")
        open(c, "w").write(src)
        subprocess.run(["g++", "-std=gnu++11", "-fsyntax-only", "-w", "-I" + REF_RENDER,
                        "-I" + os.path.join(ROOT, "include"), c], check=True)


def test_shim_check_library_loads():
    """The field-by-field checker of the drop-ins (oracle/_ref/libshim_check.so)
    loads with the product library and exports its entry points."""
    path = os.path.join(ROOT, "oracle", "_ref", "libshim_check.so")
    if not os.path.exists(path):
        pytest.skip("shim checker not built (reference tree absent)")
    L = C.CDLL(path)
    for n in ("shim_record_bytes", "shim_check_triangles", "shim_check_tetrahedra",
              "shim_check_spheres"):
        getattr(L, n)
    assert L.shim_record_bytes() == 148


def test_no_gpu_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    L = _lib.load()
    h = C.c_void_p()
    st = L.srt_ctx_create(0, C.byref(h))
    assert st == _lib.SRT_ERR_CUDA
    assert b"device" in L.srt_last_error()
    import surface_b200 as sb
    with pytest.raises(sb.SurfaceError):
        sb.TriangleAccel(sb.Context(0))


def test_null_arguments_are_rejected():
    L = _lib.load()
    assert L.srt_ctx_create(0, None) == _lib.SRT_ERR_INVALID
    assert L.srt_accel_create(None, 0, None) == _lib.SRT_ERR_INVALID
    assert L.srt_trace_closest(None, None, 0, None, None) == _lib.SRT_ERR_INVALID
    assert L.srt_ctx_synchronize(None) == _lib.SRT_ERR_INVALID
    assert L.srt_accel_destroy(None) == _lib.SRT_OK
    assert L.srt_ctx_launch_count(None) == 0
    # line, solid, texture and cache entry points
    assert L.srt_line_create(None, None) == _lib.SRT_ERR_INVALID
    assert L.srt_line_destroy(None) == _lib.SRT_OK
    assert L.srt_line_trace(None, None, 0, None, None, None) == _lib.SRT_ERR_INVALID
    assert L.srt_solid_create(None, None) == _lib.SRT_ERR_INVALID
    assert L.srt_solid_destroy(None) == _lib.SRT_OK
    assert L.srt_solid_trace(None, None, 0, None, None, None) == _lib.SRT_ERR_INVALID
    assert L.srt_texture3d_fetch(None, None, 0, None) == _lib.SRT_ERR_INVALID
    assert L.srt_cache_build_lines(None, None, 1, None, 0, None, 0.0, None, 0, 1,
                                   None) == _lib.SRT_ERR_INVALID
    assert L.srt_cache_build_solids(None, None, 1, 8, None, 0, None, 0, None) == \
        _lib.SRT_ERR_INVALID


def test_volume_camera_matches_oracle():
    """build_cameraframe (host code of the library) == the oracle's."""
    from oracle import oracle as O
    L = _lib.load()
    p = np.zeros(1, _lib.VOL_DTYPE)
    eye = np.array([0, 0, 3], np.float32)
    look = np.zeros(3, np.float32)
    up = np.array([0, 1, 0], np.float32)
    assert L.srt_volume_camera(512, 384, eye.ctypes.data, look.ctypes.data, up.ctypes.data,
                               C.c_float(45.0), p.ctypes.data) == 0
    q = O.volume_params(512, 384, eye, look, up, 45.0, 0.01, 1.0, 0.99, 100)
    for k in ("eye", "corner", "du", "dv"):
        assert np.array_equal(p[k].view(np.uint32), q[k].view(np.uint32)), k
