"""Eye rays and framebuffer writes of one frame (srt_camera_rays,
srt_framebuffer_write): RaytraceEngine::OnData's per-pixel loop
(gles/gles_raytrace_engine.cc:547-879) for one sample per pixel, on the GPU.

    cam = make_camera(512, 512, eye=(0, 0, 3), lookat=(0, 0, 0), fov=45)
    rays, pixel = camera_rays(cam)                 # CUDA tensors
    hits = accel.Traverse(rays)
    color, depth = framebuffer_write(cam, hits, pixel)

Rays follow Camera::buildFrame (render/render_camera.cc:17-63) and the
viewport conversion bit for bit; the write fills each hit pixel's
step x step block in the reference's Y-down layout.

Several samples per pixel (sampleCoverage) and the stereo environment camera
(lsglSetStereoEnvCamera): make_samples + camera_rays(..., samples=...) and
framebuffer_write(..., samples=...).  The sample jitter is the serial
renderer's random stream (TinyMT64 seeded 1234 with gles_common.cc's
parameters, drawn in pixel order), which the OpenMP renderer splits into
per-thread streams in scheduling order; the serial order is the one with a
fixed ray set.  Stereo rays use the C library's trigonometry as the reference
does; the GPU's agrees to an ulp or two.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _lib
from ._lib import check
from .accel import Context


def make_camera(width, height, eye=(0.0, 0.0, 3.0), lookat=(0.0, 0.0, 0.0),
                up=(0.0, 1.0, 0.0), fov=45.0, ortho=False, viewport=None, region=None,
                step=1):
    """srt_camera; viewport defaults to the framebuffer, region to the whole
    framebuffer."""
    c = _lib.Camera()
    c.eye[:], c.lookat[:], c.up[:] = list(eye), list(lookat), list(up)
    c.fov = fov
    c.ortho = 1 if ortho else 0
    c.width, c.height = width, height
    c.viewport[:] = list(viewport) if viewport is not None else [0, 0, width, height]
    c.region[:] = list(region) if region is not None else [0, 0, width, height]
    c.step = step
    return c


def camera_dict(c):
    """The same camera as the plain dict the CPU oracle takes."""
    return {"eye": list(c.eye), "lookat": list(c.lookat), "up": list(c.up), "fov": c.fov,
            "ortho": c.ortho, "width": c.width, "height": c.height,
            "viewport": list(c.viewport), "region": list(c.region), "step": c.step}


def _capacity(c):
    if c.step < 1:  # the library reports it; keep the sizing defined
        return 1
    nx = len(range(c.region[0], c.region[2], c.step))
    ny = len(range(c.region[1], c.region[3], c.step))
    return max(nx * ny, 1)


def make_samples(subsamples=1, stereo=None, jitter_seed=1234, jitter_offset=0):
    """srt_camera_samples: subsamples per axis; stereo = (zero_parallax,
    eye_separation) for the stereo environment camera; the jitter stream's
    seed and the draws earlier frames consumed."""
    s = _lib.CameraSamples()
    s.subsamples = int(subsamples)
    s.stereo_env = 1 if stereo else 0
    s.zero_parallax, s.eye_separation = stereo if stereo else (0.0, 0.0)
    s.jitter_seed = int(jitter_seed)
    s.jitter_offset = int(jitter_offset)
    return s


def camera_rays(cam, ctx: Context | None = None, device=0, samples=None):
    """(rays (n, 8) float32 as srt_ray, pixel (n,) int32 = (y << 16) | x of
    each ray's loop pixel), CUDA tensors on torch's current stream.  With
    samples (make_samples): subsamples^2 consecutive rays per loop pixel;
    the draws the frame consumed are then in the returned tensors' `draws`
    attribute of the rays (rays.draws)."""
    ctx = ctx or Context.default(device)
    cap = _capacity(cam)
    if samples is not None:
        cap *= samples.subsamples * samples.subsamples
    rays = torch.empty((cap, 8), dtype=torch.float32, device=f"cuda:{device}")
    pixel = torch.empty((cap,), dtype=torch.int32, device=f"cuda:{device}")
    cnt = C.c_uint32()
    ctx.use_torch_stream()
    if samples is None:
        check(ctx.L.srt_camera_rays(ctx.h, C.byref(cam), rays.data_ptr(), pixel.data_ptr(),
                                    C.byref(cnt)))
        n = cnt.value
        return rays[:n], pixel[:n]
    draws = C.c_uint64()
    check(ctx.L.srt_camera_rays_ex(ctx.h, C.byref(cam), C.byref(samples), rays.data_ptr(),
                                   pixel.data_ptr(), C.byref(cnt), C.byref(draws)))
    n = cnt.value
    out = rays[:n]
    out.draws = draws.value
    return out, pixel[:n]


def framebuffer_write(cam, hits, pixel, rgba=None, fmt=0, color=None, depth=None,
                      ctx: Context | None = None, samples=None):
    """Write the hit rays into (color, depth): color uint8 (H, W, 4) for
    fmt 0 (RGBA8) or float32 (H, W, 4) for fmt 1 (RGBA32F), depth float32
    (H, W); both created zeroed when not given."""
    dev = hits.device
    ctx = ctx or Context.default(dev.index or 0)
    if color is None:
        color = torch.zeros((cam.height, cam.width, 4),
                            dtype=torch.uint8 if fmt == 0 else torch.float32, device=dev)
    if depth is None:
        depth = torch.zeros((cam.height, cam.width), dtype=torch.float32, device=dev)
    h = hits.contiguous()
    p = pixel.contiguous()
    c = None if rgba is None else rgba.contiguous().float()
    ctx.use_torch_stream()
    if samples is None:
        check(ctx.L.srt_framebuffer_write(ctx.h, C.byref(cam), h.data_ptr(), p.data_ptr(),
                                          None if c is None else c.data_ptr(), h.shape[0],
                                          fmt, color.data_ptr(), depth.data_ptr()))
    else:
        check(ctx.L.srt_framebuffer_write_ex(ctx.h, C.byref(cam), C.byref(samples),
                                             h.data_ptr(), p.data_ptr(),
                                             None if c is None else c.data_ptr(), h.shape[0],
                                             fmt, color.data_ptr(), depth.data_ptr()))
    return color, depth
