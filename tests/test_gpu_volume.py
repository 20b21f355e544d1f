"""Volume march on the GPU: forward vs the FP32 oracle (1e-4 per channel),
adjoint vs the FP64 oracle gradient and FP64 central finite differences
(relative error <= 1e-3), and the torch.autograd.Function."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from surface_b200 import scenes as S
from surface_b200 import volume as V

pytestmark = pytest.mark.gpu

TOL_FWD = 1e-4   # per channel, FP32 image vs FP32 oracle
TOL_GRAD = 1e-3  # relative, FP32 adjoint vs FP64 reference gradient


def case(res, img, seed=3, nblobs=12):
    dens = S.volume_blobs(res, nblobs=nblobs, seed=seed)
    tgt = S.volume_blobs(res, nblobs=nblobs, seed=seed, shift_voxels=2.0)
    tf = S.transfer_function(256, seed=seed)
    p = V.camera(img, img, eye=(0.3, 0.2, 3.0), res=res)
    return p, dens, tgt, tf


def oracle_params(p):
    q = np.zeros(1, O.VOL_DTYPE)
    q[...] = p.view(O.VOL_DTYPE)
    return q


@pytest.mark.parametrize("res,img", [(32, 48), (64, 128)])
def test_forward_matches_oracle(res, img):
    p, dens, _, tf = case(res, img)
    im, tr = V.march(torch.as_tensor(dens).cuda(), torch.as_tensor(tf).cuda(), p)
    torch.cuda.synchronize()
    ref = O.volume_fwd_f32(oracle_params(p), dens, (res, res, res), tf)
    err = np.abs(im.cpu().numpy() - ref).max()
    assert err <= TOL_FWD, err
    assert np.allclose(tr.cpu().numpy(), 1.0 - ref[..., 3], atol=TOL_FWD)


def test_forward_full_size():
    """256^3 density, 512^2 rays, step 0.5 voxel."""
    p, dens, _, tf = case(256, 512, nblobs=32)
    im, _ = V.march(torch.as_tensor(dens).cuda(), torch.as_tensor(tf).cuda(), p)
    torch.cuda.synchronize()
    ref = O.volume_fwd_f32(oracle_params(p), dens, (256, 256, 256), tf)
    assert np.abs(im.cpu().numpy() - ref).max() <= TOL_FWD


def _gpu_grad(p, dens, tf, target):
    d = torch.as_tensor(dens).cuda().requires_grad_(True)
    t = torch.as_tensor(tf).cuda().requires_grad_(True)
    img = V.render(d, t, p)
    loss = ((img - torch.as_tensor(target).cuda()) ** 2).sum()
    loss.backward()
    torch.cuda.synchronize()
    return float(loss), d.grad.cpu().numpy().astype(np.float64), t.grad.cpu().numpy().astype(np.float64)


def test_adjoint_matches_fp64_reference_and_fd():
    res, img = 48, 64
    p, dens, tgt, tf = case(res, img)
    q = oracle_params(p)
    dims = (res, res, res)
    target = O.volume_fwd_f32(q, tgt, dims, tf)
    loss, gd, gt = _gpu_grad(p, dens, tf, target)
    rloss, _, rgd, rgt = O.volume_f64(q, dens, dims, tf, target=target, want_grad=True)
    assert abs(loss - rloss) <= 1e-4 * rloss
    # whole-array agreement with the FP64 analytic gradient
    assert np.linalg.norm(gd - rgd) <= TOL_GRAD * np.linalg.norm(rgd)
    assert np.linalg.norm(gt - rgt) <= TOL_GRAD * np.linalg.norm(rgt)
    # 64 voxels and 16 transfer-function entries against FP64 central FD
    rng = np.random.default_rng(1)
    flat = rgd.reshape(-1)
    sig = np.nonzero(np.abs(flat) > 1e-2 * np.abs(flat).max())[0]
    vox = rng.choice(sig, size=min(64, sig.size), replace=False)
    h = 1e-6
    d64 = dens.astype(np.float64).reshape(-1)
    worst = 0.0
    for v in vox:
        dp, dm = d64.copy(), d64.copy()
        dp[v] += h
        dm[v] -= h
        fd = (O.volume_f64(q, dp.reshape(dens.shape), dims, tf, target=target)[0]
              - O.volume_f64(q, dm.reshape(dens.shape), dims, tf, target=target)[0]) / (2 * h)
        worst = max(worst, abs(gd.reshape(-1)[v] - fd) / abs(fd))
    tflat = rgt.reshape(-1)
    ent = np.argsort(-np.abs(tflat))[:16]
    t64 = tf.astype(np.float64).reshape(-1)
    for e in ent:
        tp, tm = t64.copy(), t64.copy()
        tp[e] += h
        tm[e] -= h
        fd = (O.volume_f64(q, dens, dims, tp.reshape(tf.shape), target=target)[0]
              - O.volume_f64(q, dens, dims, tm.reshape(tf.shape), target=target)[0]) / (2 * h)
        worst = max(worst, abs(gt.reshape(-1)[e] - fd) / abs(fd))
    assert worst <= TOL_GRAD, worst


def test_adjoint_full_config():
    """The differentiable-volume configuration: 256^3 density of 32 blobs,
    256-entry transfer function, 512^2 rays, step 0.5 voxel, L2 loss against
    the image of the blobs shifted by 2 voxels.  The CUDA adjoint against the
    FP64 oracle gradient (whole arrays) and FP64 central finite differences on
    64 voxels (loss over the pixels whose rays pass near the voxel: the only
    ones a change there can reach) and 16 transfer-function entries (whole
    image); relative error <= 1e-3."""
    dens = S.volume_blobs(256, nblobs=32)
    tgt = S.volume_blobs(256, nblobs=32, shift_voxels=2.0)
    tf = S.transfer_function(256)
    p = V.camera(512, 512, eye=(0.0, 0.0, 3.0), res=256)
    q = oracle_params(p)
    dims = (256, 256, 256)
    target = O.volume_fwd_f32(q, tgt, dims, tf)
    loss, gd, gt = _gpu_grad(p, dens, tf, target)
    rloss, _, rgd, rgt = O.volume_f64(q, dens, dims, tf, target=target, want_grad=True)
    assert abs(loss - rloss) <= 1e-4 * rloss
    assert np.linalg.norm(gd - rgd) <= TOL_GRAD * np.linalg.norm(rgd)
    assert np.linalg.norm(gt - rgt) <= TOL_GRAD * np.linalg.norm(rgt)
    rng = np.random.default_rng(5)
    flat = rgd.reshape(-1)
    sig = np.nonzero(np.abs(flat) > 1e-2 * np.abs(flat).max())[0]
    vox = rng.choice(sig, size=64, replace=False)
    h = 1e-6
    d64 = dens.astype(np.float64).reshape(-1)
    worst = 0.0
    for v in vox:
        z, rem = divmod(int(v), 256 * 256)
        y, x = divmod(rem, 256)
        pix = O.volume_pixels_near(q, dims, (x, y, z), 1.5)
        assert pix.size > 0
        dp, dm = d64.copy(), d64.copy()
        dp[v] += h
        dm[v] -= h
        fd = (O.volume_f64_pixels(q, dp.reshape(dens.shape), dims, tf, target, pix)
              - O.volume_f64_pixels(q, dm.reshape(dens.shape), dims, tf, target, pix)) / (2 * h)
        worst = max(worst, abs(gd.reshape(-1)[v] - fd) / abs(fd))
    t64 = tf.astype(np.float64).reshape(-1)
    for e in np.argsort(-np.abs(rgt.reshape(-1)))[:16]:
        tp, tm = t64.copy(), t64.copy()
        tp[e] += h
        tm[e] -= h
        fd = (O.volume_f64(q, dens, dims, tp.reshape(tf.shape), target=target)[0]
              - O.volume_f64(q, dens, dims, tm.reshape(tf.shape), target=target)[0]) / (2 * h)
        worst = max(worst, abs(gt.reshape(-1)[e] - fd) / abs(fd))
    assert worst <= TOL_GRAD, worst


def test_autograd_function_matches_direct_adjoint():
    p, dens, tgt, tf = case(32, 40)
    d = torch.as_tensor(dens).cuda()
    t = torch.as_tensor(tf).cuda()
    target = V.march(torch.as_tensor(tgt).cuda(), t, p)[0]
    img, trans = V.march(d, t, p)
    gd, gt = V.march_backward(d, t, p, trans, 2 * (img - target))
    dd = d.clone().requires_grad_(True)
    tt = t.clone().requires_grad_(True)
    ((V.render(dd, tt, p) - target) ** 2).sum().backward()
    torch.cuda.synchronize()
    assert torch.allclose(dd.grad, gd, rtol=1e-4, atol=1e-7)
    assert torch.allclose(tt.grad, gt, rtol=1e-4, atol=1e-7)


def _nonuniform(res):
    """y remapped through an exponential coordinate map, GL's repeat wrap."""
    remap = (None, S.exp_coord_map(res + 1), None)
    return remap, (0, 0, 0)


def test_nonuniform_forward_matches_oracle():
    res, img = 48, 96
    p, dens, _, tf = case(res, img)
    remap, clamp = _nonuniform(res)
    smp = V.Sampling(remap=remap, clamp=[bool(c) for c in clamp])
    d, t = torch.as_tensor(dens).cuda(), torch.as_tensor(tf).cuda()
    im, tr = V.march(d, t, p, sampling=smp)
    # host tables are staged by the library
    host = V.Sampling(remap=remap, clamp=[bool(c) for c in clamp])
    host.tables = [None if x is None else x.cpu() for x in host.tables]
    im_h, _ = V.march(d, t, p, sampling=host)
    # clamp-to-edge without remap is the plain march
    im0, _ = V.march(d, t, p)
    im1, _ = V.march(d, t, p, sampling=V.Sampling())
    torch.cuda.synchronize()
    assert torch.equal(im0, im1) and torch.equal(im, im_h)
    ref = O.volume_fwd_f32(oracle_params(p), dens, (res,) * 3, tf, remap=remap, clamp=clamp)
    plain = O.volume_fwd_f32(oracle_params(p), dens, (res,) * 3, tf)
    assert np.abs(ref - plain).max() > 1e-2
    # a sample whose remap index sits on a table boundary may pick the next
    # entry when the position differs by an ulp; all other pixels agree
    err = np.abs(im.cpu().numpy() - ref).max(axis=2)
    assert np.mean(err <= TOL_FWD) >= 0.999, np.mean(err <= TOL_FWD)
    good = err <= TOL_FWD
    assert np.allclose(tr.cpu().numpy()[good], 1.0 - ref[..., 3][good], atol=TOL_FWD)


def test_nonuniform_adjoint_matches_fp64_reference_and_fd():
    res, img = 40, 64
    p, dens, tgt, tf = case(res, img)
    q = oracle_params(p)
    dims = (res,) * 3
    remap, clamp = _nonuniform(res)
    smp = V.Sampling(remap=remap, clamp=[bool(c) for c in clamp])
    target = O.volume_fwd_f32(q, tgt, dims, tf, remap=remap, clamp=clamp)
    dd = torch.as_tensor(dens).cuda().requires_grad_(True)
    tt = torch.as_tensor(tf).cuda().requires_grad_(True)
    out = V.render(dd, tt, p, sampling=smp)
    loss = ((out - torch.as_tensor(target).cuda()) ** 2).sum()
    loss.backward()
    torch.cuda.synchronize()
    gd = dd.grad.cpu().numpy().astype(np.float64)
    gt = tt.grad.cpu().numpy().astype(np.float64)
    rloss, _, rgd, rgt = O.volume_f64(q, dens, dims, tf, target=target, want_grad=True,
                                      remap=remap, clamp=clamp)
    assert abs(float(loss) - rloss) <= 1e-3 * rloss
    assert np.linalg.norm(gd - rgd) <= TOL_GRAD * np.linalg.norm(rgd)
    assert np.linalg.norm(gt - rgt) <= TOL_GRAD * np.linalg.norm(rgt)
    flat = rgd.reshape(-1)
    vox = np.argsort(-np.abs(flat))[:16]
    h = 1e-6
    d64 = dens.astype(np.float64).reshape(-1)
    worst = 0.0
    for v in vox:
        dp, dm = d64.copy(), d64.copy()
        dp[v] += h
        dm[v] -= h
        fd = (O.volume_f64(q, dp.reshape(dens.shape), dims, tf, target=target, remap=remap,
                           clamp=clamp)[0]
              - O.volume_f64(q, dm.reshape(dens.shape), dims, tf, target=target, remap=remap,
                             clamp=clamp)[0]) / (2 * h)
        worst = max(worst, abs(gd.reshape(-1)[v] - fd) / abs(fd))
    assert worst <= TOL_GRAD, worst


def test_adjoint_gradient_scale_and_non_finite():
    """The transfer-function gradient is summed per block in fixed point at
    a power-of-two scale taken from the block's image gradient: scaling the
    image gradient by 2^+-100 scales both gradients by the same factor, and
    a non-finite image gradient reaches the result (float path) instead of
    being rounded away."""
    p, dens, tgt, tf = case(32, 48)
    d = torch.as_tensor(dens).cuda()
    t = torch.as_tensor(tf).cuda()
    target = V.march(torch.as_tensor(tgt).cuda(), t, p)[0]
    img, trans = V.march(d, t, p)
    g = 2 * (img - target)
    gd, gt = V.march_backward(d, t, p, trans, g)
    assert gt.abs().max() > 0 and gd.abs().max() > 0
    for e in (-100, 100):
        f = 2.0 ** e
        gd2, gt2 = V.march_backward(d, t, p, trans, g * f)
        assert torch.allclose(gt2 / f, gt, rtol=1e-5, atol=1e-7 * float(gt.abs().max()))
        assert torch.allclose(gd2 / f, gd, rtol=1e-5, atol=1e-7 * float(gd.abs().max()))
    g_nan = g.clone()
    g_nan[24, 24, 0] = float("nan")
    _, gt3 = V.march_backward(d, t, p, trans, g_nan)
    assert torch.isnan(gt3).any()
