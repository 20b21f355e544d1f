"""3D texture fetch on the GPU (srt_texture3d_*): Texture::Fetch of the
reference's GLES front end (gles/gles_common.h:344-399) for arrays of
coordinates -- dense textures (bytes, floats, doubles; repeat or
clamp-to-edge; per-axis remap tables of non-uniform volumes) and sparse
block volumes.

    tex = Texture3D()
    tex.set_dense(img, fmt=1)                 # img (D, H, W[, comps])
    tex.set_remap(1, table)                   # lsglTexCoordRemap(GL_COORDINATE_Y, ...)
    rgba = tex.Fetch(uvw)                     # (n, 3) -> (n, 4) float32
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from ._lib import check
from .accel import Context

FORMATS = {0: np.uint8, 1: np.float32, 2: np.float64}
BLOCK_DTYPE = np.dtype([("offset", "<i4", 3), ("extent", "<i4", 3), ("size", "<i4", 3),
                        ("level", "<i4"), ("data_offset", "<u8")])


class Texture3D:
    def __init__(self, ctx: Context | None = None, device=0):
        self.ctx = ctx or Context.default(device)
        self.L = self.ctx.L
        h = C.c_void_p()
        check(self.L.srt_texture3d_create(self.ctx.h, C.byref(h)))
        self.h = h

    def set_dense(self, img, fmt=1, components=None):
        """img: (D, H, W) or (D, H, W, comps), texels x fastest; fmt 0 bytes,
        1 float, 2 double."""
        a = np.ascontiguousarray(img, FORMATS[fmt])
        d, h, w = a.shape[:3]
        comps = components or (a.shape[3] if a.ndim == 4 else 1)
        self.ctx.use_own_stream()
        check(self.L.srt_texture3d_set_dense(self.h, fmt, w, h, d, comps, a.ctypes.data))

    def set_wrap(self, clamp_s=True, clamp_t=True, clamp_r=True):
        """Clamp-to-edge per axis (False: repeat)."""
        check(self.L.srt_texture3d_set_wrap(self.h, int(clamp_s), int(clamp_t), int(clamp_r)))

    def set_remap(self, axis, table):
        """Coordinate remap of a non-uniform volume for axis 0..2; None removes it."""
        t = None if table is None else np.ascontiguousarray(table, np.float32)
        self.ctx.use_own_stream()
        check(self.L.srt_texture3d_set_remap(self.h, axis, None if t is None else t.ctypes.data,
                                             0 if t is None else t.size))

    def set_sparse(self, blocks, pool, fmt, components, global_dim):
        """blocks: BLOCK_DTYPE array (offset, extent, size, level, data_offset
        into pool); pool: bytes of all blocks' voxels."""
        b = np.ascontiguousarray(blocks, BLOCK_DTYPE)
        p = np.frombuffer(bytes(pool), np.uint8)
        g = np.ascontiguousarray(global_dim, np.int32)
        self.ctx.use_own_stream()
        check(self.L.srt_texture3d_set_sparse(self.h, fmt, components, g.ctypes.data,
                                              b.ctypes.data, b.size, p.ctypes.data, p.size))

    def Fetch(self, uvw, out=None):
        """rgba (n, 4) float32 for coordinates uvw (n, 3): CUDA tensors in,
        CUDA out (numpy in, numpy out)."""
        host = not (isinstance(uvw, torch.Tensor) and uvw.is_cuda)
        dev = torch.device("cuda", self.ctx.device)
        u = (torch.from_numpy(np.ascontiguousarray(uvw, np.float32).reshape(-1, 3)).to(dev)
             if host else uvw.contiguous().float())
        n = u.numel() // 3
        if out is None:
            out = torch.empty((n, 4), dtype=torch.float32, device=u.device)
        self.ctx.use_torch_stream()
        check(self.L.srt_texture3d_fetch(self.h, u.data_ptr(), n, out.data_ptr()))
        return out.cpu().numpy() if host else out

    def close(self):
        if getattr(self, "h", None):
            self.L.srt_texture3d_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass
