"""Many triangle scenes built and traced in one pass (libsurface_rt srt_batch).

The reference builds one TriangleAccel per scene and traces it
(render/render_accel_triangle.cc:1389-1690 for Build32, :2511 for
Traverse); a batch of uneven scenes therefore costs one build and one trace
launch sequence per scene.  ``TriangleBatch`` does the same work for all scenes
at once: every build stage runs once over the concatenated primitives (scene
id as the top radix digit keeps the scenes apart) and one persistent kernel
traces every ray against its own scene's tree.  Results are identical to the
per-scene path, prim ids are face indices within the scene.

The first call autotunes the traversal launch shape, the second identical call
is captured in a CUDA graph and later identical calls replay it.  The batch
owns a context with its own stream (capturable) and orders it after torch's
current stream on entry and before it on return.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from ._lib import SurfaceError, check
from .accel import Context


class TriangleBatch:
    def __init__(self, device=0):
        self.ctx = Context(device)  # own stream: graph capture needs one
        self.L = self.ctx.L
        h = C.c_void_p()
        check(self.L.srt_batch_create(self.ctx.h, C.byref(h)))
        self.h = h
        self._stream = torch.cuda.ExternalStream(self.L.srt_ctx_get_stream(self.ctx.h),
                                                 device=torch.device("cuda", device))
        self._keep = ()

    def build_trace(self, vertices, faces, face_offsets, rays, ray_offsets, hits=None):
        """vertices (V,3) f32, faces (F,3) int32 vertex ids, rays (R,8) f32 as
        srt_ray -- CUDA tensors; face_offsets / ray_offsets: nscenes+1 host
        integers.  Returns hits (R,4) f32 laid out as srt_hit."""
        for name, t in (("vertices", vertices), ("faces", faces), ("rays", rays)):
            if not (isinstance(t, torch.Tensor) and t.is_cuda and t.is_contiguous()):
                raise SurfaceError(1, f"{name} must be a contiguous CUDA tensor")
        fo = np.ascontiguousarray(face_offsets, np.uint64)
        ro = np.ascontiguousarray(ray_offsets, np.uint64)
        if fo.size != ro.size or fo.size < 2:
            raise SurfaceError(1, "face_offsets and ray_offsets need nscenes+1 entries")
        if hits is None:
            hits = torch.empty((rays.shape[0], 4), dtype=torch.float32, device=rays.device)
        cur = torch.cuda.current_stream(rays.device)
        self._stream.wait_stream(cur)
        check(self.L.srt_batch_build_trace(self.h, fo.size - 1, vertices.data_ptr(),
                                           faces.data_ptr(), fo.ctypes.data, rays.data_ptr(),
                                           ro.ctypes.data, hits.data_ptr()))
        cur.wait_stream(self._stream)
        # the captured graph keeps raw pointers: hold the tensors it reads
        self._keep = (vertices, faces, rays, hits)
        return hits

    def config(self):
        """(block, rays_per_thread, graph_captured, kernels_per_call)."""
        blk = C.c_int32()
        r = C.c_int32()
        g = C.c_int32()
        k = C.c_uint64()
        check(self.L.srt_batch_config(self.h, C.byref(blk), C.byref(r), C.byref(g),
                                      C.byref(k)))
        return blk.value, r.value, bool(g.value), k.value

    def tuning(self):
        """The autotuned traversal point: {"block", "rays_per_grab",
        "stack_depth", "sort_bits"} (sort_bits 0: rays in array order)."""
        v = [C.c_int32() for _ in range(4)]
        check(self.L.srt_batch_tuning(self.h, *[C.byref(x) for x in v]))
        return dict(zip(("block", "rays_per_grab", "stack_depth", "sort_bits"),
                        (x.value for x in v)))

    def set_tuning(self, block=128, rays_per_grab=1, stack_depth=32, sort_bits=0):
        """Pin the traversal point instead of autotuning it."""
        check(self.L.srt_batch_set_tuning(self.h, int(block), int(rays_per_grab),
                                          int(stack_depth), int(sort_bits)))

    def launches(self):
        return self.L.srt_ctx_launch_count(self.ctx.h)

    def close(self):
        if getattr(self, "h", None):
            self.L.srt_batch_destroy(self.h)
            self.h = None
        if getattr(self, "ctx", None) is not None:
            self.ctx.close()
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass
