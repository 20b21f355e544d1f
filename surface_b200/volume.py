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


def march(density, tf, params, ctx: Context | None = None):
    """Forward march: (image (H, W, 4), final transmittance (H, W))."""
    ctx = ctx or Context.default(density.device.index or 0)
    density = density.contiguous().float()
    tf = tf.contiguous().float()
    H, W = int(params["height"][0]), int(params["width"][0])
    img = torch.empty((H, W, 4), dtype=torch.float32, device=density.device)
    trans = torch.empty((H, W), dtype=torch.float32, device=density.device)
    ctx.use_torch_stream()
    dims = _dims(density)
    check(ctx.L.srt_volume_march_fwd(ctx.h, params.ctypes.data, density.data_ptr(),
                                     dims.ctypes.data, tf.data_ptr(), tf.shape[0],
                                     img.data_ptr(), trans.data_ptr()))
    return img, trans


def march_backward(density, tf, params, trans, grad_image, ctx: Context | None = None):
    """Adjoint: (d loss / d density, d loss / d tf)."""
    ctx = ctx or Context.default(density.device.index or 0)
    density = density.contiguous().float()
    tf = tf.contiguous().float()
    gd = torch.zeros_like(density)
    gt = torch.zeros_like(tf)
    ctx.use_torch_stream()
    dims = _dims(density)
    g = grad_image.contiguous().float()
    check(ctx.L.srt_volume_march_bwd(ctx.h, params.ctypes.data, density.data_ptr(),
                                     dims.ctypes.data, tf.data_ptr(), tf.shape[0], None,
                                     trans.contiguous().data_ptr(), g.data_ptr(),
                                     gd.data_ptr(), gt.data_ptr()))
    return gd, gt


class VolumeMarch(torch.autograd.Function):
    @staticmethod
    def forward(ctx, density, tf, params):
        img, trans = march(density, tf, params)
        ctx.save_for_backward(density, tf, trans)
        ctx.params = params
        return img

    @staticmethod
    def backward(ctx, grad_image):
        density, tf, trans = ctx.saved_tensors
        gd, gt = march_backward(density, tf, ctx.params, trans, grad_image)
        return (gd if ctx.needs_input_grad[0] else None,
                gt if ctx.needs_input_grad[1] else None, None)


def render(density, tf, params):
    """Differentiable image of `density` (D, H, W) through `tf` (entries, 4)."""
    return VolumeMarch.apply(density, tf, params)
