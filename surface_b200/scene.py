"""Several accels with transforms traced as one scene: RenderGraph
(gles/gles_render_graph.cc:104-314) on the GPU.

    scene = RenderGraph()
    scene.AddRenderElement(mesh_accel, T)        # T: 4x4, Matrixd layout
    scene.AddRenderElement(particle_accel, T2)
    scene.AddRenderElement(line_accel, T3)      # LineAccel / SolidAccel too
    scene.Build()
    hits, element = scene.Trace(rays)          # CUDA tensors in, CUDA out

Matrices are 4x4 doubles in Matrixd's layout: m[row][col] with points
transformed as p' = (p, 1) m, so the translation is the last row.
AddRenderElement derives invT, invT33 and the world box exactly as
RenderElement::Update does; add_element_matrices takes them from the caller.
Hit t is the world distance of the hit point; prim, u and v are the element's
own; element is the hit element's id (0, 1, ... in the order added) or MISS.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from ._lib import HIT_DTYPE, MISS, RAY_DTYPE, SurfaceError, check
from .accel import Context, _Accel
from .lines import LineAccel
from .solids import SolidAccel


def _mat(m):
    a = np.ascontiguousarray(m, np.float64).reshape(16)
    return a


def matrix_inverse(m):
    """Matrixd::Inverse (render/render_matrix.h:40-134) of a 4x4."""
    a = _mat(m).copy()
    _lib.load().srt_matrix_inverse(a.ctypes.data)
    return a.reshape(4, 4)


class RenderGraph:
    """Top-level tree over transformed accels (all of one Context)."""

    def __init__(self, ctx: Context | None = None, device=0):
        self.ctx = ctx or Context.default(device)
        self.L = self.ctx.L
        h = C.c_void_p()
        check(self.L.srt_scene_create(self.ctx.h, C.byref(h)))
        self.h = h
        self.elements = []

    def AddRenderElement(self, accel, T=None) -> int:
        """Add a built accel (triangles, tetrahedra, particles, LineAccel or
        SolidAccel) under transform T (identity when None); returns its
        element id."""
        if accel.ctx is not self.ctx and accel.ctx.h.value != self.ctx.h.value:
            raise SurfaceError(_lib.SRT_ERR_INVALID, "accel of another context")
        t = _mat(np.eye(4) if T is None else T)
        eid = C.c_uint32()
        if isinstance(accel, LineAccel):
            add = self.L.srt_scene_add_lines
        elif isinstance(accel, SolidAccel):
            add = self.L.srt_scene_add_solids
        else:
            add = self.L.srt_scene_add_element
        check(add(self.h, accel.h, t.ctypes.data, C.byref(eid)))
        self.elements.append(accel)
        return eid.value

    def add_element_matrices(self, accel: _Accel, T, invT, invT33, world_bmin,
                             world_bmax) -> int:
        """Add with the caller's own inverse matrices and world box."""
        t, it, it33 = _mat(T), _mat(invT), _mat(invT33)
        lo = np.ascontiguousarray(world_bmin, np.float64)
        hi = np.ascontiguousarray(world_bmax, np.float64)
        eid = C.c_uint32()
        check(self.L.srt_scene_add(self.h, accel.h, t.ctypes.data, it.ctypes.data,
                                   it33.ctypes.data, lo.ctypes.data, hi.ctypes.data,
                                   C.byref(eid)))
        self.elements.append(accel)
        return eid.value

    def Build(self) -> bool:
        """The top-level tree over the elements' world boxes."""
        self.ctx.use_torch_stream()
        check(self.L.srt_scene_build(self.h))
        return True

    def top_nodes(self):
        """(boxes (n, 6) float64 bmin|bmax, ints (n, 5) int32 child0, child1,
        axis, leaf, element) of the top-level tree, in BVHTree's node order."""
        n = self.L.srt_scene_top_nodes(self.h, None, None, 0)
        boxes = np.zeros((n, 6), np.float64)
        ints = np.zeros((n, 5), np.int32)
        self.L.srt_scene_top_nodes(self.h, boxes.ctypes.data, ints.ctypes.data, n)
        return boxes, ints

    def Trace(self, rays, prev_element=None, prev_normals=None, hits=None, element=None,
              stats=None):
        """Closest hit over all elements for every ray.

        rays: CUDA float32 (n, 8) tensor as srt_ray (or a RAY_DTYPE numpy
        array, copied to the device and the results back).  prev_element
        (n,) int32/uint32 and prev_normals (n, 3) float32 select the self-hit
        rule's element and sphere normal for secondary rays.  stats: optional
        CUDA int64 (5,) tensor the visit counters are added to (top-level
        nodes, element walks, branch nodes, leaves, primitives)."""
        host = not (isinstance(rays, torch.Tensor) and rays.is_cuda)
        dev = torch.device("cuda", self.ctx.device)
        if host:
            r = np.ascontiguousarray(rays, RAY_DTYPE)
            rt = torch.from_numpy(r.view(np.float32).reshape(-1, 8)).to(dev)
        else:
            rt = rays.contiguous()
            if rt.dtype != torch.float32:
                raise TypeError("CUDA rays must be float32 (n, 8)")
        n = rt.numel() // 8
        if hits is None:
            hits = torch.empty((n, 4), dtype=torch.float32, device=rt.device)
        if element is None:
            element = torch.empty((n,), dtype=torch.int32, device=rt.device)

        def dev_arr(x, dt):
            if x is None:
                return None
            if isinstance(x, torch.Tensor):
                return x.to(device=rt.device, dtype=dt).contiguous()
            return torch.from_numpy(np.ascontiguousarray(x).astype(
                np.int32 if dt == torch.int32 else np.float32)).to(rt.device)
        pe = prev_element
        if pe is not None and not isinstance(pe, torch.Tensor):
            pe = np.ascontiguousarray(pe, np.uint32).view(np.int32)
        pe = dev_arr(pe, torch.int32)
        pn = dev_arr(prev_normals, torch.float32)
        self.ctx.use_torch_stream()
        check(self.L.srt_scene_trace(self.h, rt.data_ptr(), n,
                                     None if pe is None else pe.data_ptr(),
                                     None if pn is None else pn.data_ptr(),
                                     hits.data_ptr(), element.data_ptr(),
                                     None if stats is None else stats.data_ptr()))
        if host:
            h = np.ascontiguousarray(hits.cpu().numpy()).view(HIT_DTYPE).reshape(-1)
            e = element.cpu().numpy().view(np.uint32).copy()
            return h, e
        return hits, element

    def close(self):
        if getattr(self, "h", None):
            self.L.srt_scene_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass


__all__ = ["RenderGraph", "matrix_inverse", "MISS"]
