"""Solid accel on the GPU (srt_solid_*): the reference's SolidAccel
(render/render_accel_solid.{h,cc}) over Solid (render/render_prim_solid.h)
-- pyramids (5 vertices), prisms (6) and hexahedra (8).

    acc = SolidAccel()
    acc.Build32(Solid(8, vertices, indices))
    hits = acc.Traverse(rays)                     # HIT_DTYPE (numpy) or (n, 4) CUDA
    hits, normals, positions = acc.Traverse(rays, want_point=True)
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from ._lib import HIT_DTYPE, RAY_DTYPE, SurfaceError, check
from .accel import Context, _is_cuda, _View
from .lines import LINE_NODE_DTYPE

SOLID_NODE_DTYPE = LINE_NODE_DTYPE  # SolidNode: the same 40-byte record


@dataclass
class Solid:
    """render/render_prim_solid.h: numVertsPerSolid (5, 6 or 8), vertices
    (V, 3) float32, or float64 for double-precision positions (dvertices,
    isDoublePrecisionPos), indices (N, numVertsPerSolid) uint32."""
    numVertsPerSolid: int
    vertices: object
    indices: object


class SolidAccel:
    def __init__(self, ctx: Context | None = None, device=0):
        self.ctx = ctx or Context.default(device)
        self.L = self.ctx.L
        h = C.c_void_p()
        check(self.L.srt_solid_create(self.ctx.h, C.byref(h)))
        self.h = h
        self.built = False

    def Build(self, solids: Solid, options=None) -> bool:
        """SolidAccel::Build (render/render_accel_solid.cc:1754): the binned-SAH
        build at every size, as the GLES accel builder runs it."""
        return self._build(solids, sah=True)

    def Build32(self, solids: Solid, options=None) -> bool:
        """SolidAccel::Build32 (render/render_accel_solid.cc:1795)."""
        return self._build(solids, sah=False)

    def _build(self, solids: Solid, sah: bool) -> bool:
        dbl = getattr(solids.vertices, "dtype", None) in (np.float64, torch.float64)
        v = (_View(solids.vertices, np.float64, torch.float64) if dbl
             else _View(solids.vertices, np.float32, torch.float32))
        ix = _View(solids.indices, np.uint32, torch.int32)
        nv = int(solids.numVertsPerSolid)
        # device inputs: in torch's stream order; host inputs: the context's stream
        if v.device or ix.device:
            self.ctx.use_torch_stream()
        else:
            self.ctx.use_own_stream()
        if sah:
            build = self.L.srt_solid_build_sah_double if dbl else self.L.srt_solid_build_sah
        else:
            build = self.L.srt_solid_build_double if dbl else self.L.srt_solid_build
        check(build(self.h, nv, v.ptr, v.nbytes // (24 if dbl else 12), ix.ptr,
                    ix.nbytes // (4 * nv)))
        self.built = True
        return True

    def info(self):
        """(solids, nodes)."""
        a, b = C.c_uint64(), C.c_uint64()
        check(self.L.srt_solid_info(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def export(self):
        n, nn = self.info()
        nodes = np.zeros(nn, SOLID_NODE_DTYPE)
        idx = np.zeros(n, np.uint32)
        check(self.L.srt_solid_export(self.h, nodes.ctypes.data, idx.ctypes.data))
        return nodes, idx

    def BoundingBox(self):
        lo = np.zeros(3)
        hi = np.zeros(3)
        check(self.L.srt_solid_bbox(self.h, lo.ctypes.data, hi.ctypes.data))
        return lo, hi

    def Dump(self, filename) -> bool:
        check(self.L.srt_solid_dump(self.h, str(filename).encode()))
        return True

    def Traverse(self, rays, hits=None, want_point=False):
        """Nearest entry or exit point per ray (batched SolidAccel::Traverse);
        want_point adds the normals and positions."""
        if not self.built:
            raise SurfaceError(_lib.SRT_ERR_INVALID, "accel not built")
        if _is_cuda(rays):
            r = rays.contiguous()
            n = r.numel() // 8
            if hits is None:
                hits = torch.empty((n, 4), dtype=torch.float32, device=r.device)
            nrm = pos = None
            if want_point:
                nrm = torch.empty((n, 3), dtype=torch.float32, device=r.device)
                pos = torch.empty((n, 3), dtype=torch.float32, device=r.device)
            self.ctx.use_torch_stream()
            ptrs = (r.data_ptr(), hits.data_ptr(), nrm.data_ptr() if nrm is not None else None,
                    pos.data_ptr() if pos is not None else None)
        else:
            r = np.ascontiguousarray(rays, RAY_DTYPE)
            n = r.size
            if hits is None:
                hits = np.zeros(n, HIT_DTYPE)
            nrm = np.zeros((n, 3), np.float32) if want_point else None
            pos = np.zeros((n, 3), np.float32) if want_point else None
            self.ctx.use_own_stream()
            ptrs = (r.ctypes.data, hits.ctypes.data, nrm.ctypes.data if nrm is not None else None,
                    pos.ctypes.data if pos is not None else None)
        check(self.L.srt_solid_trace(self.h, ptrs[0], n, ptrs[1], ptrs[2], ptrs[3]))
        return (hits, nrm, pos) if want_point else hits

    def close(self):
        if getattr(self, "h", None):
            self.L.srt_solid_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass
