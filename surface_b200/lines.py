"""Line (capped cylinder) accel on the GPU (srt_line_*): the reference's
LineAccel (render/render_accel_line.{h,cc}) over Lines
(render/render_prim_line.h).

    acc = LineAccel()
    acc.Build(Lines(positions, segments, radius), LineBuildOptions())
    hits = acc.Traverse(rays)                 # HIT_DTYPE (numpy in) or (n, 4) CUDA
    hits, normals = acc.Traverse(rays, want_normal=True)
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from ._lib import HIT_DTYPE, RAY_DTYPE, SurfaceError, check
from .accel import Context, _is_cuda, _View

LINE_NODE_DTYPE = np.dtype([("bmin", "<f4", 3), ("bmax", "<f4", 3), ("flag", "<i4"),
                            ("axis", "<i4"), ("data", "<u4", 2)])  # LineNode, 40 bytes


@dataclass
class Lines:
    """render/render_prim_line.h: vertex positions (V, 3) float32, segments
    (N, 2) uint32 vertex pairs, per-vertex radius (V,) or None for
    constantRadius.  numpy arrays or CUDA tensors."""
    positions: object
    segments: object
    radius: object = None
    constantRadius: float = 0.0


@dataclass
class LineBuildOptions:
    """render/render_accel_line.h:50-60 (defaults 4, 512, capped)."""
    minLeafPrimitives: int = 4
    maxTreeDepth: int = 512
    cap: bool = True


class LineAccel:
    def __init__(self, ctx: Context | None = None, device=0):
        self.ctx = ctx or Context.default(device)
        self.L = self.ctx.L
        h = C.c_void_p()
        check(self.L.srt_line_create(self.ctx.h, C.byref(h)))
        self.h = h
        self.built = False

    def Build(self, lines: Lines, options: LineBuildOptions | None = None) -> bool:
        """LineAccel::Build (render/render_accel_line.cc:298)."""
        o = options or LineBuildOptions()
        tdt = torch.float32
        p = _View(lines.positions, np.float32, tdt)
        s = _View(lines.segments, np.uint32, torch.int32)
        r = _View(lines.radius, np.float32, tdt)
        nv = p.nbytes // 12
        nl = s.nbytes // 8
        if any(v.device for v in (p, s, r) if v.obj is not None):
            torch.cuda.current_stream().synchronize()
        self.ctx.use_own_stream()
        check(self.L.srt_line_build(self.h, p.ptr, nv, r.ptr, C.c_float(lines.constantRadius),
                                    s.ptr, nl, o.minLeafPrimitives, o.maxTreeDepth, int(o.cap)))
        self.built = True
        return True

    def info(self):
        """(lines, nodes, tree depth)."""
        a, b, d = C.c_uint64(), C.c_uint64(), C.c_int32()
        check(self.L.srt_line_info(self.h, C.byref(a), C.byref(b), C.byref(d)))
        return a.value, b.value, d.value

    def export(self):
        """(nodes LINE_NODE_DTYPE in the Dump layout, line order)."""
        n, nn, _ = self.info()
        nodes = np.zeros(nn, LINE_NODE_DTYPE)
        idx = np.zeros(n, np.uint32)
        check(self.L.srt_line_export(self.h, nodes.ctypes.data, idx.ctypes.data))
        return nodes, idx

    def BoundingBox(self):
        lo = np.zeros(3)
        hi = np.zeros(3)
        check(self.L.srt_line_bbox(self.h, lo.ctypes.data, hi.ctypes.data))
        return lo, hi

    def Dump(self, filename) -> bool:
        check(self.L.srt_line_dump(self.h, str(filename).encode()))
        return True

    def Traverse(self, rays, hits=None, want_normal=False, stats=None):
        """Closest hit per ray (batched LineAccel::Traverse).  stats: a CUDA
        int64 tensor of 3 counters (branches, leaves, line tests) to add to."""
        if not self.built:
            raise SurfaceError(_lib.SRT_ERR_INVALID, "accel not built")
        if _is_cuda(rays):
            r = rays.contiguous()
            n = r.numel() // 8
            if hits is None:
                hits = torch.empty((n, 4), dtype=torch.float32, device=r.device)
            nrm = torch.empty((n, 3), dtype=torch.float32, device=r.device) if want_normal else None
            self.ctx.use_torch_stream()
            rp, hp = r.data_ptr(), hits.data_ptr()
            np_ = nrm.data_ptr() if nrm is not None else None
        else:
            r = np.ascontiguousarray(rays, RAY_DTYPE)
            n = r.size
            if hits is None:
                hits = np.zeros(n, HIT_DTYPE)
            nrm = np.zeros((n, 3), np.float32) if want_normal else None
            self.ctx.use_own_stream()
            rp, hp = r.ctypes.data, hits.ctypes.data
            np_ = nrm.ctypes.data if nrm is not None else None
        check(self.L.srt_line_trace(self.h, rp, n, hp, np_,
                                    None if stats is None else stats.data_ptr()))
        return (hits, nrm) if want_normal else hits

    def close(self):
        if getattr(self, "h", None):
            self.L.srt_line_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass
