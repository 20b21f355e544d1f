"""AccelBuilder's accel cache (gles/gles_accel_builder.cc:34-117, 400-456,
1017-1037) over the GPU accels (srt_cache_*).

    cache = AccelBuilder()
    acc = cache.BuildTriangleAccel(Mesh(v, f), elembuf=1, arraybuf=2,
                                   count=nfaces * 3, static=True)
    ...                           # same key again: the same accel, a hit
    cache.Invalidate(2)           # buffer 2 changed: its accels are freed
    cache.EndFrame()              # dynamic entries are freed

Buffers are any integer ids of the caller (the reference uses the GL buffer
objects).  The cache owns the accels it returns.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import SRT_SPHERES, SRT_TETRAHEDRA, SRT_TRIANGLES, check
from .accel import (Context, Mesh, ParticleAccel, Particles, TetraAccel, Tetrahedron,
                    TriangleAccel, _View, torch)
from .lines import LineAccel, Lines
from .solids import Solid, SolidAccel

# Each Build* returns an accel object over the cached handle.


def _owned_by_cache(base):
    class Cached(base):
        """A cache-owned accel: queries and Traverse of the accel class; the
        handle is freed by the cache, not by this object."""

        def close(self):
            self.h = None

    Cached.__name__ = "Cached" + base.__name__
    return Cached


_LINES, _SOLIDS = 3, 4  # the cache's kinds beyond srt_kind
_CACHED = {SRT_TRIANGLES: _owned_by_cache(TriangleAccel),
           SRT_TETRAHEDRA: _owned_by_cache(TetraAccel),
           SRT_SPHERES: _owned_by_cache(ParticleAccel),
           _LINES: _owned_by_cache(LineAccel),
           _SOLIDS: _owned_by_cache(SolidAccel)}


class AccelBuilder:
    def __init__(self, maxCacheSize=8192 * 1024, ctx: Context | None = None, device=0):
        self.ctx = ctx or Context.default(device)
        self.L = self.ctx.L
        h = C.c_void_p()
        check(self.L.srt_cache_create(self.ctx.h, maxCacheSize, C.byref(h)))
        self.h = h
        self._keep = {}

    def _key(self, elembuf, arraybuf, position_offset, count, offset):
        return _lib.CacheKey(elembuf, arraybuf, position_offset, count, offset)

    def _finish(self, kind, out, keep, builds_before):
        v = out.value
        if self.info().builds != builds_before:  # built now: borrows these inputs
            self._keep[v] = keep
        obj = object.__new__(_CACHED[kind])
        obj.ctx, obj.L, obj.h, obj.built = self.ctx, self.L, C.c_void_p(v), True
        obj._keep = self._keep.get(v)
        return obj

    def BuildTriangleAccel(self, mesh: Mesh, elembuf, arraybuf, count, offset=0,
                           position_offset=0, static=True):
        key = self._key(elembuf, arraybuf, position_offset, count, offset)
        v = _View(mesh.vertices, np.float32, torch.float32)
        f = _View(mesh.faces, np.uint32, torch.int32)
        out = C.c_void_p()
        b0 = self.info().builds
        self.ctx.use_own_stream() if not v.device else self.ctx.use_torch_stream()
        check(self.L.srt_cache_build_triangles(self.h, C.byref(key), int(static), v.ptr,
                                               v.nbytes // 12, f.ptr, f.nbytes // 12,
                                               C.byref(out)))
        return self._finish(SRT_TRIANGLES, out, (v, f), b0)

    def BuildTetraAccel(self, tetras: Tetrahedron, elembuf, arraybuf, count, offset=0,
                        position_offset=0, static=True):
        key = self._key(elembuf, arraybuf, position_offset, count, offset)
        v = _View(tetras.vertices, np.float32, torch.float32)
        f = _View(tetras.faces, np.uint32, torch.int32)
        out = C.c_void_p()
        b0 = self.info().builds
        self.ctx.use_own_stream() if not v.device else self.ctx.use_torch_stream()
        check(self.L.srt_cache_build_tetrahedra(self.h, C.byref(key), int(static), v.ptr,
                                                v.nbytes // 12, f.ptr, f.nbytes // 16,
                                                C.byref(out)))
        return self._finish(SRT_TETRAHEDRA, out, (v, f), b0)

    def BuildParticleAccel(self, particles: Particles, elembuf, arraybuf, count, offset=0,
                           position_offset=0, static=True):
        key = self._key(elembuf, arraybuf, position_offset, count, offset)
        p = _View(particles.positions, np.float32, torch.float32)
        r = _View(particles.radius, np.float32, torch.float32)
        out = C.c_void_p()
        b0 = self.info().builds
        self.ctx.use_own_stream() if not p.device else self.ctx.use_torch_stream()
        check(self.L.srt_cache_build_spheres(self.h, C.byref(key), int(static), p.ptr, r.ptr,
                                             C.c_float(particles.constantRadius),
                                             p.nbytes // 12, C.byref(out)))
        return self._finish(SRT_SPHERES, out, (p, r), b0)

    def BuildLineAccel(self, lines: Lines, elembuf, arraybuf, count, offset=0,
                       position_offset=0, static=True, cap=True):
        """AccelBuilder::BuildLineAccel (gles/gles_accel_builder.cc:188)."""
        key = self._key(elembuf, arraybuf, position_offset, count, offset)
        p = _View(lines.positions, np.float32, torch.float32)
        s = _View(lines.segments, np.uint32, torch.int32)
        r = _View(lines.radius, np.float32, torch.float32)
        out = C.c_void_p()
        b0 = self.info().builds
        if p.device or s.device or (r.obj is not None and r.device):
            torch.cuda.current_stream().synchronize()
        self.ctx.use_own_stream()
        check(self.L.srt_cache_build_lines(self.h, C.byref(key), int(static), p.ptr,
                                           p.nbytes // 12, r.ptr,
                                           C.c_float(lines.constantRadius), s.ptr,
                                           s.nbytes // 8, int(cap), C.byref(out)))
        return self._finish(_LINES, out, (p, s, r), b0)

    def BuildSolidAccel(self, solids: Solid, elembuf, arraybuf, count, offset=0,
                        position_offset=0, static=True):
        """AccelBuilder::BuildSolidAccel (gles/gles_accel_builder.cc:328)."""
        key = self._key(elembuf, arraybuf, position_offset, count, offset)
        nv = int(solids.numVertsPerSolid)
        v = _View(solids.vertices, np.float32, torch.float32)
        ix = _View(solids.indices, np.uint32, torch.int32)
        out = C.c_void_p()
        b0 = self.info().builds
        if v.device or ix.device:
            torch.cuda.current_stream().synchronize()
        self.ctx.use_own_stream()
        check(self.L.srt_cache_build_solids(self.h, C.byref(key), int(static), nv, v.ptr,
                                            v.nbytes // 12, ix.ptr, ix.nbytes // (4 * nv),
                                            C.byref(out)))
        return self._finish(_SOLIDS, out, (v, ix), b0)

    def Invalidate(self, buffer):
        check(self.L.srt_cache_invalidate(self.h, buffer))
        self._prune()

    def EndFrame(self):
        check(self.L.srt_cache_end_frame(self.h))
        self._prune()

    def _prune(self):
        # a freed entry's handle may come back for a later build, which then
        # registers its own inputs; with no entries left nothing is borrowed
        info = self.info()
        if info.static_entries + info.dynamic_entries == 0:
            self._keep.clear()

    def info(self):
        i = _lib.CacheInfo()
        check(self.L.srt_cache_info_get(self.h, C.byref(i)))
        return i

    def GetCacheUsed(self):
        return self.info().bytes_used

    def GetCacheSize(self):
        return self.info().bytes_max

    def close(self):
        if getattr(self, "h", None):
            self.L.srt_cache_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass
