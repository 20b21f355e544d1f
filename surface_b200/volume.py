"""Differentiable emission-absorption volume march (libsurface_rt).

The march keeps the reference shader's geometry
(examples/nonuniform_volume_render/input.frag: build_cameraframe with 3.14,
fragment-centre rays, the IntersectP slab test on [-1,1]^3, texture3D at
0.5*p + 0.5 with FilterTexture3DFloat's texel-corner trilinear weights) and
composites front to back:

    rgba  = transfer function, linearly interpolated at rho * (entries - 1)
    alpha = min(1 - exp(-sigma_scale * rgba.a * step), alpha_max)
    C    += T * alpha * rgba.rgb ;  T *= 1 - alpha ;  image = (C, 1 - T)

``VolumeMarch`` is a torch.autograd.Function whose backward is the hand-written
adjoint kernel: it rebuilds transmittance in reverse sample order from the
final transmittance saved by the forward pass (no per-sample state) and
returns gradients for the density grid and the transfer-function table.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from ._lib import VOL_DTYPE, check
from .accel import Context


def camera(width, height, eye=(0.0, 0.0, 3.0), lookat=(0.0, 0.0, 0.0), up=(0.0, 1.0, 0.0),
           fov_deg=45.0, step=None, res=256, sigma_scale=20.0, alpha_max=0.99,
           max_steps=8192):
    """srt_volume_params for the shader camera.  step defaults to half a voxel
    of a res^3 grid spanning [-1,1]^3 with texel-corner spacing 2/(res-1)."""
    L = _lib.load()
    p = np.zeros(1, VOL_DTYPE)
    e = np.asarray(eye, np.float32)
    la = np.asarray(lookat, np.float32)
    u = np.asarray(up, np.float32)
    check(L.srt_volume_camera(int(width), int(height), e.ctypes.data, la.ctypes.data,
                              u.ctypes.data, C.c_float(fov_deg), p.ctypes.data))
    p["max_steps"] = max_steps
    p["step"] = step if step is not None else 0.5 * 2.0 / (res - 1)
    p["sigma_scale"] = sigma_scale
    p["alpha_max"] = alpha_max
    return p


def _dims(density):
    d, h, w = density.shape
    return np.array([w, h, d], np.int32)


class Sampling:
    """The density texture's sampling state: per-axis remap tables of a
    non-uniform volume (lsglTexCoordRemap; None for none) and clamp-to-edge
    flags (False: GL's default repeat wrap).  Sampling() = clamp-to-edge, no
    remap, which is what march() uses without one."""

    def __init__(self, remap=(None, None, None), clamp=(True, True, True), device=0):
        self.tables = [None if t is None else
                       torch.as_tensor(np.ascontiguousarray(t, np.float32)).to(
                           torch.device("cuda", device)) for t in remap]
        self.clamp = tuple(bool(c) for c in clamp)

    def struct(self):
        sm = _lib.VolumeSampling()
        for k in range(3):
            t = self.tables[k]
            sm.remap[k] = None if t is None else t.data_ptr()
            sm.remap_n[k] = 0 if t is None else t.numel()
            sm.clamp[k] = int(self.clamp[k])
        return sm


def march(density, tf, params, ctx: Context | None = None, sampling: Sampling | None = None):
    """Forward march: (image (H, W, 4), final transmittance (H, W))."""
    ctx = ctx or Context.default(density.device.index or 0)
    density = density.contiguous().float()
    tf = tf.contiguous().float()
    H, W = int(params["height"][0]), int(params["width"][0])
    img = torch.empty((H, W, 4), dtype=torch.float32, device=density.device)
    trans = torch.empty((H, W), dtype=torch.float32, device=density.device)
    ctx.use_torch_stream()
    dims = _dims(density)
    sm = None if sampling is None else sampling.struct()
    check(ctx.L.srt_volume_march_fwd_ex(ctx.h, params.ctypes.data,
                                        None if sm is None else C.byref(sm),
                                        density.data_ptr(), dims.ctypes.data, tf.data_ptr(),
                                        tf.shape[0], img.data_ptr(), trans.data_ptr()))
    return img, trans


def march_backward(density, tf, params, trans, grad_image, ctx: Context | None = None,
                   sampling: Sampling | None = None):
    """Adjoint: (d loss / d density, d loss / d tf)."""
    ctx = ctx or Context.default(density.device.index or 0)
    density = density.contiguous().float()
    tf = tf.contiguous().float()
    gd = torch.zeros_like(density)
    gt = torch.zeros_like(tf)
    ctx.use_torch_stream()
    dims = _dims(density)
    g = grad_image.contiguous().float()
    sm = None if sampling is None else sampling.struct()
    check(ctx.L.srt_volume_march_bwd_ex(ctx.h, params.ctypes.data,
                                        None if sm is None else C.byref(sm),
                                        density.data_ptr(), dims.ctypes.data, tf.data_ptr(),
                                        tf.shape[0], None, trans.contiguous().data_ptr(),
                                        g.data_ptr(), gd.data_ptr(), gt.data_ptr()))
    return gd, gt


class VolumeMarch(torch.autograd.Function):
    @staticmethod
    def forward(ctx, density, tf, params, sampling=None):
        img, trans = march(density, tf, params, sampling=sampling)
        ctx.save_for_backward(density, tf, trans)
        ctx.params = params
        ctx.sampling = sampling
        return img

    @staticmethod
    def backward(ctx, grad_image):
        density, tf, trans = ctx.saved_tensors
        gd, gt = march_backward(density, tf, ctx.params, trans, grad_image,
                                sampling=ctx.sampling)
        return (gd if ctx.needs_input_grad[0] else None,
                gt if ctx.needs_input_grad[1] else None, None, None)


def render(density, tf, params, sampling: Sampling | None = None):
    """Differentiable image of `density` (D, H, W) through `tf` (entries, 4);
    `sampling` adds non-uniform remap tables and wrap modes."""
    return VolumeMarch.apply(density, tf, params, sampling)
