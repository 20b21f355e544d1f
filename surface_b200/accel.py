"""Host-side mirror of SURFACE's render/ accel classes over libsurface_rt.

The reference interface (render/render_accel_triangle.h:69-105,
render/render_accel_tetra.h:65-120, render/render_accel_particle.h:60-110):

    accel = TriangleAccel()
    accel.Build32(mesh, TriangleBuildOptions())   # -> True
    accel.Traverse(isect, ray)                    # one ray, -> bool
    accel.BoundingBox(bmin, bmax)
    accel.Dump(filename)

is kept with the same names and meaning.  ``Traverse`` is batched: it takes an
array of rays (numpy structured ``RAY_DTYPE``, or a float32 tensor of shape
(n, 8) laid out as srt_ray) and returns one hit per ray.  Host arrays give
host results (synchronous); CUDA tensors give CUDA tensors ordered on torch's
current stream (asynchronous).  Errors raise ``SurfaceError`` instead of the
reference's asserts; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import (HIT_DTYPE, ISECT_DTYPE, MISS, RAY_DTYPE, SRT_SPHERES, SRT_TETRAHEDRA,
                   SRT_TRIANGLES, AccelInfo, SurfaceError, TraceOpts, check)

try:  # torch is optional for the host API (numpy works alone)
    import torch
except Exception:  # noqa: BLE001
    torch = None


# ---------------------------------------------------------------- arrays
def _is_torch(x):
    return torch is not None and isinstance(x, torch.Tensor)


def _is_cuda(x):
    return _is_torch(x) and x.is_cuda


class _View:
    """Pointer to a contiguous array of the required dtype (keeps it alive)."""

    def __init__(self, x, np_dtype, torch_dtype=None):
        self.obj = None
        self.ptr = None
        self.device = False
        if x is None:
            return
        if _is_torch(x):
            t = x
            if torch_dtype is not None and t.dtype != torch_dtype:
                t = t.to(torch_dtype)
            t = t.contiguous()
            self.obj = t
            self.ptr = t.data_ptr()
            self.device = t.is_cuda
            self.nbytes = t.numel() * t.element_size()
        else:
            a = np.ascontiguousarray(x, dtype=np_dtype)
            self.obj = a
            self.ptr = a.ctypes.data
            self.nbytes = a.nbytes


# ---------------------------------------------------------------- context
class Context:
    """An srt_ctx: one device, one stream, reusable scratch buffers."""

    _defaults: dict = {}

    def __init__(self, device=0):
        L = _lib.load()
        h = C.c_void_p()
        check(L.srt_ctx_create(device, C.byref(h)))
        self.h = h
        self.device = device
        self.L = L

    @classmethod
    def default(cls, device=0):
        if device not in cls._defaults:
            cls._defaults[device] = Context(device)
        return cls._defaults[device]

    def use_torch_stream(self):
        """Order this context's work on torch's current stream."""
        if torch is not None and torch.cuda.is_available():
            s = torch.cuda.current_stream(self.device).cuda_stream
            # handle 0 is the legacy default stream; NULL would select the
            # context's own stream, so pass cudaStreamLegacy (1) instead
            check(self.L.srt_ctx_set_stream(self.h, C.c_void_p(s if s else 1)))

    def use_own_stream(self):
        check(self.L.srt_ctx_set_stream(self.h, None))

    def synchronize(self):
        check(self.L.srt_ctx_synchronize(self.h))

    def close(self):
        if getattr(self, "h", None):
            self.L.srt_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass


# ---------------------------------------------------------------- primitives
@dataclass
class Mesh:
    """render/render_prim_triangle.h:22-56 (float vertices, uint32 faces)."""
    vertices: object  # (V,3) float32
    faces: object     # (F,3) uint32


@dataclass
class Tetrahedron:
    """render/render_prim_tetra.h:30-37."""
    vertices: object  # (V,3) float32, or float64 for double positions (dvertices)
    faces: object     # (N,4) uint32


@dataclass
class Particles:
    """render/render_prim_particle.h:19-27."""
    positions: object            # (N,3) float32
    radius: object = None        # (N,) float32 or None
    constantRadius: float = 0.0


@dataclass
class TriangleBuildOptions:
    """render/render_accel_triangle.h:45-55; Build32 uses none of the fields."""
    debugPrint: bool = False
    costTaabb: float = 0.2
    minLeafPrimitives: int = 16
    maxTreeDepth: int = 256
    binSize: int = 64


@dataclass
class TetraBuildOptions(TriangleBuildOptions):
    minLeafPrimitives: int = 4


@dataclass
class ParticleBuildOptions(TriangleBuildOptions):
    pass


@dataclass
class TraceResult:
    hits: object
    subface: object = None
    scalar: object = None
    normal: object = None
    isect: object = None  # BuildIntersection's records (ISECT_DTYPE, or (n, 20) float32 CUDA)
    extra: dict = field(default_factory=dict)


# ---------------------------------------------------------------- accel
class _Accel:
    KIND = None

    def __init__(self, ctx: Context | None = None, device=0):
        self.ctx = ctx or Context.default(device)
        self.L = self.ctx.L
        h = C.c_void_p()
        check(self.L.srt_accel_create(self.ctx.h, self.KIND, C.byref(h)))
        self.h = h
        self._keep = ()
        self.built = False

    # -- build ------------------------------------------------------------
    def _sync_stream(self, *arrays):
        if any(_is_cuda(a) for a in arrays if a is not None):
            self.ctx.use_torch_stream()
        else:
            self.ctx.use_own_stream()

    # -- queries ----------------------------------------------------------
    def info(self) -> AccelInfo:
        inf = AccelInfo()
        check(self.L.srt_accel_info_get(self.h, C.byref(inf)))
        return inf

    def BoundingBox(self, bmin=None, bmax=None):
        """Root box of the tree (XxxAccel::BoundingBox)."""
        lo = np.zeros(3, np.float64)
        hi = np.zeros(3, np.float64)
        check(self.L.srt_accel_bbox(self.h, lo.ctypes.data, hi.ctypes.data))
        if bmin is not None:
            bmin[:3] = lo
        if bmax is not None:
            bmax[:3] = hi
        return lo, hi

    def export(self):
        """(raw device node records, sorted indices, sorted Morton codes)."""
        inf = self.info()
        raw = np.zeros(inf.num_nodes * inf.node_bytes, np.uint8)
        idx = np.zeros(inf.num_prims, np.uint32)
        codes = np.zeros(inf.num_prims, np.uint32)
        check(self.L.srt_accel_export(self.h, raw.ctypes.data, idx.ctypes.data,
                                      codes.ctypes.data))
        return raw, idx, codes

    def Dump(self, filename) -> bool:
        """Write the reference's Dump() format (render/render_accel_triangle.cc:1692)."""
        check(self.L.srt_accel_dump(self.h, str(filename).encode()))
        return True

    # -- traversal --------------------------------------------------------
    def Traverse(self, rays, hits=None, prev_normals=None, want_subface=False,
                 vertex_scalar=None, want_scalar=False, want_normal=False,
                 single_pass=False, sort_rays=False, want_isect=False, max_iter=0,
                 grid_launch=False):
        """Closest hit for every ray (batched XxxAccel::Traverse).

        single_pass=True walks the tree once in the reference's own order;
        the default two-pass walk returns the same hits with less work.
        sort_rays=True traverses in a coherent ray order (same hits).
        grid_launch=True runs the first pass one thread per ray over a full
        grid instead of persistent warps (same hits).
        want_isect=True also returns BuildIntersection's shading record per
        ray (position, normal, tangent, binormal, f0..f3, d0..d3).
        max_iter > 0 caps the steps of each ray's walk (SRT_ERR_LIMIT when a
        ray reaches it)."""
        if not self.built:
            raise SurfaceError(_lib.SRT_ERR_INVALID, "accel not built")
        cuda = _is_cuda(rays)
        if cuda:
            r = rays.contiguous()
            if r.dtype != torch.float32:
                raise TypeError("CUDA rays must be float32 (n, 8)")
            n = r.numel() // 8
            rv = _View(r, None)
            if hits is None:
                hits = torch.empty((n, 4), dtype=torch.float32, device=r.device)
            hv = _View(hits, None)

            def out(shape, dt=torch.float32):
                return torch.empty(shape, dtype=dt, device=r.device)
            sub = out((n,), torch.int32) if want_subface else None
            sca = out((n,)) if want_scalar else None
            nrm = out((n, 3)) if want_normal else None
            isx = out((n, 20)) if want_isect else None
            self.ctx.use_torch_stream()
        else:
            r = np.ascontiguousarray(rays, RAY_DTYPE)
            n = r.size
            rv = _View(r, RAY_DTYPE)
            if hits is None:
                hits = np.zeros(n, HIT_DTYPE)
            hv = _View(hits, HIT_DTYPE)
            sub = np.zeros(n, np.uint32) if want_subface else None
            sca = np.zeros(n, np.float32) if want_scalar else None
            nrm = np.zeros((n, 3), np.float32) if want_normal else None
            isx = np.zeros(n, ISECT_DTYPE) if want_isect else None
            self.ctx.use_own_stream()
        pn = _View(prev_normals, np.float32, torch.float32 if torch is not None else None)
        vs = _View(vertex_scalar, np.float32, torch.float32 if torch is not None else None)
        if want_scalar and not vs.device:
            raise SurfaceError(_lib.SRT_ERR_INVALID, "vertex_scalar must be a CUDA tensor")
        o = TraceOpts(pn.ptr, _View(sub, np.uint32).ptr if sub is not None else None,
                      vs.ptr, _View(sca, np.float32).ptr if sca is not None else None,
                      _View(nrm, np.float32).ptr if nrm is not None else None, None,
                      (_lib.SRT_TRACE_SINGLE_PASS if single_pass else 0)
                      | (_lib.SRT_TRACE_SORT_RAYS if sort_rays else 0)
                      | (_lib.SRT_TRACE_GRID if grid_launch else 0), int(max_iter),
                      _View(isx, ISECT_DTYPE if not cuda else None).ptr
                      if isx is not None else None)
        check(self.L.srt_trace_closest(self.h, rv.ptr, n, hv.ptr, C.byref(o)))
        if not (want_subface or want_scalar or want_normal or want_isect):
            return hits
        return TraceResult(hits, sub, sca, nrm, isx)

    def close(self):
        if getattr(self, "h", None):
            self.L.srt_accel_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass


class TriangleAccel(_Accel):
    KIND = SRT_TRIANGLES

    def Build32(self, mesh: Mesh, options: TriangleBuildOptions | None = None) -> bool:
        """LBVH build (render/render_accel_triangle.cc:1389-1690)."""
        v = _View(mesh.vertices, np.float32, torch.float32 if torch is not None else None)
        f = _View(mesh.faces, np.uint32, torch.int32 if torch is not None else None)
        nv = v.nbytes // 12
        nf = f.nbytes // 12
        self._sync_stream(mesh.vertices, mesh.faces)
        check(self.L.srt_accel_build_triangles(self.h, v.ptr, nv, f.ptr, nf))
        self._keep = (v, f)  # device inputs are borrowed for the accel's life
        self.built = True
        return True

    def Load(self, filename, mesh: Mesh) -> bool:
        """The accel of `mesh` from a Dump() file (no rebuild; no counterpart
        in the reference, which writes these files only)."""
        v = _View(mesh.vertices, np.float32, torch.float32 if torch is not None else None)
        f = _View(mesh.faces, np.uint32, torch.int32 if torch is not None else None)
        self._sync_stream(mesh.vertices, mesh.faces)
        check(self.L.srt_accel_load_triangles(self.h, str(filename).encode(), v.ptr,
                                              v.nbytes // 12, f.ptr, f.nbytes // 12))
        self._keep = (v, f)
        self.built = True
        return True


class TetraAccel(_Accel):
    KIND = SRT_TETRAHEDRA

    def Build32(self, tetras: Tetrahedron, options: TetraBuildOptions | None = None) -> bool:
        """LBVH build (render/render_accel_tetra.cc:1579-1850); float64
        vertices keep double precision (isDoublePrecisionPos)."""
        dbl = str(getattr(tetras.vertices, "dtype", "")) in ("float64", "torch.float64")
        if dbl:
            v = _View(tetras.vertices, np.float64, torch.float64 if torch is not None else None)
        else:
            v = _View(tetras.vertices, np.float32, torch.float32 if torch is not None else None)
        f = _View(tetras.faces, np.uint32, torch.int32 if torch is not None else None)
        self._sync_stream(tetras.vertices, tetras.faces)
        build = self.L.srt_accel_build_tetrahedra_double if dbl else self.L.srt_accel_build_tetrahedra
        check(build(self.h, v.ptr, v.nbytes // (24 if dbl else 12), f.ptr, f.nbytes // 16))
        self._keep = (v, f)
        self.built = True
        return True

    def Load(self, filename, tetras: Tetrahedron) -> bool:
        """The accel of `tetras` from a Dump() file (no rebuild)."""
        v = _View(tetras.vertices, np.float32, torch.float32 if torch is not None else None)
        f = _View(tetras.faces, np.uint32, torch.int32 if torch is not None else None)
        self._sync_stream(tetras.vertices, tetras.faces)
        check(self.L.srt_accel_load_tetrahedra(self.h, str(filename).encode(), v.ptr,
                                               v.nbytes // 12, f.ptr, f.nbytes // 16))
        self._keep = (v, f)
        self.built = True
        return True


class ParticleAccel(_Accel):
    KIND = SRT_SPHERES

    def Build32(self, particles: Particles, options: ParticleBuildOptions | None = None) -> bool:
        """LBVH build (render/render_accel_particle.cc:1560-1866)."""
        p = _View(particles.positions, np.float32, torch.float32 if torch is not None else None)
        r = _View(particles.radius, np.float32, torch.float32 if torch is not None else None)
        self._sync_stream(particles.positions, particles.radius)
        check(self.L.srt_accel_build_spheres(self.h, p.ptr, r.ptr,
                                             C.c_float(particles.constantRadius),
                                             p.nbytes // 12))
        self._keep = (p, r)
        self.built = True
        return True

    def Load(self, filename, particles: Particles) -> bool:
        """The accel of `particles` from a Dump() file (no rebuild)."""
        p = _View(particles.positions, np.float32, torch.float32 if torch is not None else None)
        r = _View(particles.radius, np.float32, torch.float32 if torch is not None else None)
        self._sync_stream(particles.positions, particles.radius)
        check(self.L.srt_accel_load_spheres(self.h, str(filename).encode(), p.ptr, r.ptr,
                                            C.c_float(particles.constantRadius),
                                            p.nbytes // 12))
        self._keep = (p, r)
        self.built = True
        return True


# ---------------------------------------------------------------- stages
def stage_morton(kind, vertices, prims=None, radius=None, constant_radius=0.0, ctx=None):
    """(codes, scene box) of the build's first two steps, in input order."""
    ctx = ctx or Context.default()
    v = np.ascontiguousarray(vertices, np.float32)
    p = None if prims is None else np.ascontiguousarray(prims, np.uint32)
    r = None if radius is None else np.ascontiguousarray(radius, np.float32)
    n = (p.size // (3 if kind == SRT_TRIANGLES else 4)) if p is not None else v.size // 3
    codes = np.zeros(n, np.uint32)
    box = np.zeros(6, np.float32)
    ctx.use_own_stream()
    check(ctx.L.srt_stage_morton(ctx.h, kind, v.ctypes.data, v.size // 3,
                                 None if p is None else p.ctypes.data,
                                 None if r is None else r.ctypes.data,
                                 C.c_float(constant_radius), n, codes.ctypes.data,
                                 box.ctypes.data))
    return codes, box


def stage_sort_pairs(codes, indices=None, ctx=None):
    ctx = ctx or Context.default()
    c = np.ascontiguousarray(codes, np.uint32).copy()
    i = (np.arange(c.size, dtype=np.uint32) if indices is None
         else np.ascontiguousarray(indices, np.uint32).copy())
    ctx.use_own_stream()
    check(ctx.L.srt_stage_sort_pairs(ctx.h, c.ctypes.data, i.ctypes.data, c.size))
    return c, i


def stage_karras(sorted_codes, ctx=None):
    ctx = ctx or Context.default()
    c = np.ascontiguousarray(sorted_codes, np.uint32)
    m = c.size - 1
    child = np.zeros(m, np.uint32)
    lt = np.zeros(m, np.uint8)
    rt = np.zeros(m, np.uint8)
    ctx.use_own_stream()
    check(ctx.L.srt_stage_karras(ctx.h, c.ctypes.data, c.size, child.ctypes.data,
                                 lt.ctypes.data, rt.ctypes.data))
    return child, lt, rt


# ---------------------------------------------------------------- rays
def spawn_secondary(rays, hits, normals, seed, ctx=None):
    """One hemisphere ray per hit (srt_spawn_secondary).  rays (n, 8), hits
    (n, 4) and normals (n, 3) are CUDA float32 tensors (the outputs of a
    Traverse with want_normal=True); returns (secondary rays (k, 8), their
    unit normals (k, 3)) for the k hit rays, in ray order, to be traced with
    prev_normals=normals."""
    if not (_is_cuda(rays) and _is_cuda(hits) and _is_cuda(normals)):
        raise SurfaceError(_lib.SRT_ERR_INVALID, "spawn_secondary takes CUDA tensors")
    ctx = ctx or Context.default(rays.device.index or 0)
    r, h, nrm = rays.contiguous(), hits.contiguous(), normals.contiguous().float()
    n = r.shape[0]
    out = torch.empty((n, 8), dtype=torch.float32, device=r.device)
    out_n = torch.empty((n, 3), dtype=torch.float32, device=r.device)
    cnt = C.c_uint32()
    ctx.use_torch_stream()
    check(ctx.L.srt_spawn_secondary(ctx.h, r.data_ptr(), h.data_ptr(), nrm.data_ptr(), n,
                                    C.c_uint64(seed), out.data_ptr(), out_n.data_ptr(),
                                    C.byref(cnt)))
    k = cnt.value
    return out[:k], out_n[:k]


__all__ = ["Context", "Mesh", "Tetrahedron", "Particles", "TriangleAccel", "TetraAccel",
           "ParticleAccel", "TriangleBuildOptions", "TetraBuildOptions",
           "ParticleBuildOptions", "stage_morton", "stage_sort_pairs", "stage_karras",
           "spawn_secondary",
           "RAY_DTYPE", "HIT_DTYPE", "ISECT_DTYPE", "MISS", "SurfaceError"]
