"""The volume march oracle: FP32 forward agrees with the FP64 forward, and
the FP64 analytic adjoint (reverse-order transmittance recomputation) agrees
with FP64 central finite differences on density voxels and transfer-function
entries.  Geometry follows examples/nonuniform_volume_render/input.frag."""
import numpy as np
import pytest

from oracle import oracle as O
from surface_b200 import scenes as S


def small_case(res=24, img=20, seed=3):
    dens = S.volume_blobs(res, nblobs=6, seed=seed)
    target = S.volume_blobs(res, nblobs=6, seed=seed, shift_voxels=2.0)
    tf = S.transfer_function(256, seed=seed)
    step = 0.5 * 2.0 / (res - 1)
    P = O.volume_params(img, img, (0.3, 0.2, 3.0), (0, 0, 0), (0, 1, 0), 45.0, step, 20.0,
                        0.99, 4096)
    dims = (res, res, res)
    return P, dens, target, tf, dims


def test_fp32_forward_matches_fp64():
    P, dens, _, tf, dims = small_case()
    f32 = O.volume_fwd_f32(P, dens, dims, tf)
    _, f64, _, _ = O.volume_f64(P, dens, dims, tf, want_img=True)
    assert np.max(np.abs(f32 - f64)) < 1e-4
    assert np.max(f32[..., 3]) > 0.2  # the volume is visible


def test_fp64_adjoint_matches_finite_differences():
    P, dens, tgt_dens, tf, dims = small_case()
    target = O.volume_fwd_f32(P, tgt_dens, dims, tf)
    loss, _, gd, gt = O.volume_f64(P, dens, dims, tf, target=target, want_grad=True)
    assert loss > 0
    rng = np.random.default_rng(0)
    flat = gd.reshape(-1)
    cand = np.nonzero(np.abs(flat) > 1e-3 * np.abs(flat).max())[0]
    vox = rng.choice(cand, size=min(32, cand.size), replace=False)
    h = 1e-6
    d64 = dens.astype(np.float64)
    for v in vox:
        dp = d64.copy().reshape(-1)
        dm = d64.copy().reshape(-1)
        dp[v] += h
        dm[v] -= h
        lp = O.volume_f64(P, dp.reshape(dens.shape), dims, tf, target=target)[0]
        lm = O.volume_f64(P, dm.reshape(dens.shape), dims, tf, target=target)[0]
        fd = (lp - lm) / (2 * h)
        assert abs(fd - flat[v]) <= 1e-4 * max(abs(fd), 1e-3 * np.abs(flat).max()), (v, fd, flat[v])
    tflat = gt.reshape(-1)
    ent = np.argsort(-np.abs(tflat))[:16]
    t64 = tf.astype(np.float64)
    for e in ent:
        tp = t64.copy().reshape(-1)
        tm = t64.copy().reshape(-1)
        tp[e] += h
        tm[e] -= h
        lp = O.volume_f64(P, dens, dims, tp.reshape(tf.shape), target=target)[0]
        lm = O.volume_f64(P, dens, dims, tm.reshape(tf.shape), target=target)[0]
        fd = (lp - lm) / (2 * h)
        assert abs(fd - tflat[e]) <= 1e-4 * max(abs(fd), 1e-3 * np.abs(tflat).max()), (e, fd, tflat[e])


def test_nonuniform_sampling_fp32_vs_fp64_and_adjoint():
    """A non-uniform volume: y remapped through an exponential coordinate map
    with GL's repeat wrap (a coordinate remapped to 1.0 wraps to 0)."""
    P, dens, tgt_dens, tf, dims = small_case()
    remap = (None, S.exp_coord_map(dims[1] + 1), None)
    clamp = (0, 0, 0)
    f32 = O.volume_fwd_f32(P, dens, dims, tf, remap=remap, clamp=clamp)
    _, f64, _, _ = O.volume_f64(P, dens, dims, tf, want_img=True, remap=remap, clamp=clamp)
    plain = O.volume_fwd_f32(P, dens, dims, tf)
    assert np.max(np.abs(f32 - plain)) > 1e-2  # the remap changes the image
    # table indices and the wrap are taken in float vs double: compare the
    # images where both pick the same texels (all but a few pixels)
    err = np.abs(f32 - f64).max(axis=2)
    assert np.mean(err < 1e-4) > 0.99
    target = O.volume_fwd_f32(P, tgt_dens, dims, tf, remap=remap, clamp=clamp)
    loss, _, gd, gt = O.volume_f64(P, dens, dims, tf, target=target, want_grad=True,
                                   remap=remap, clamp=clamp)
    flat = gd.reshape(-1)
    vox = np.argsort(-np.abs(flat))[:12]
    h = 1e-6
    d64 = dens.astype(np.float64)
    for v in vox:
        dp = d64.copy().reshape(-1)
        dm = d64.copy().reshape(-1)
        dp[v] += h
        dm[v] -= h
        lp = O.volume_f64(P, dp.reshape(dens.shape), dims, tf, target=target, remap=remap,
                          clamp=clamp)[0]
        lm = O.volume_f64(P, dm.reshape(dens.shape), dims, tf, target=target, remap=remap,
                          clamp=clamp)[0]
        fd = (lp - lm) / (2 * h)
        assert abs(fd - flat[v]) <= 1e-4 * max(abs(fd), 1e-3 * np.abs(flat).max())
