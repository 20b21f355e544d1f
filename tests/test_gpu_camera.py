"""Eye rays (srt_camera_rays) and framebuffer writes (srt_framebuffer_write)
on the GPU against the restated OnData loop of the CPU oracle (whose camera
frame is pinned to the reference's Camera::buildFrame): bit-exact rays,
pixels, colours and depths."""
import numpy as np
import pytest
import torch

import surface_b200 as sb
from oracle import oracle as O
from surface_b200 import camera as K
from surface_b200 import scenes as S

from conftest import bits

pytestmark = pytest.mark.gpu

CASES = [
    dict(width=512, height=512, eye=(0, 0, 3), lookat=(0, 0, 0), fov=45.0),
    dict(width=333, height=97, eye=(0.3, 0.2, 3), lookat=(0, 0.1, 0), fov=30.0, step=3),
    dict(width=200, height=150, eye=(1, 2, 3), lookat=(0, 0, 0), up=(0, 0, 1), ortho=True,
         step=2),
    dict(width=256, height=192, eye=(0, 0, 3), lookat=(0, 0, 0), fov=50.0,
         viewport=(16, -8, 240, 200), region=(10, 5, 250, 190), step=2),
]


def _scene():
    v, f = S.displaced_octasphere(6, seed=7)
    acc = sb.TriangleAccel()
    acc.Build32(sb.Mesh(torch.as_tensor(v).cuda(), torch.as_tensor(f.view(np.int32)).cuda()))
    return acc


@pytest.mark.parametrize("case", CASES)
def test_camera_rays_match_oracle(case):
    cam = K.make_camera(**case)
    rays, pix = K.camera_rays(cam)
    torch.cuda.synchronize()
    ref, rpix = O.camera_rays(K.camera_dict(cam))
    got = rays.cpu().numpy().reshape(-1).view(O.RAY_DTYPE)
    assert got.size == ref.size > 0
    for f in ("org", "dir", "prev_prim", "prev_t"):
        assert np.array_equal(bits(got[f]), bits(ref[f])), f
    assert np.array_equal(pix.cpu().numpy().view(np.uint32), rpix)


@pytest.mark.parametrize("case", CASES)
def test_framebuffer_write_matches_oracle(case):
    acc = _scene()
    cam = K.make_camera(**case)
    rays, pix = K.camera_rays(cam)
    hits = acc.Traverse(rays)
    gen = torch.Generator(device="cuda").manual_seed(3)
    rgba = torch.rand((rays.shape[0], 4), device="cuda", generator=gen) * 1.2 - 0.1
    torch.cuda.synchronize()
    h = hits.cpu().numpy().reshape(-1).view(O.HIT_DTYPE)
    p = pix.cpu().numpy().view(np.uint32)
    assert (h["prim"] != O.MISS).any() and (h["prim"] == O.MISS).any()
    d = K.camera_dict(cam)
    for fmt in (0, 1):
        for col in (None, rgba):
            c, dep = K.framebuffer_write(cam, hits, pix, rgba=col, fmt=fmt)
            torch.cuda.synchronize()
            rc, rd = O.framebuffer_write(d, h, p, None if col is None else col.cpu().numpy(),
                                         fmt)
            cg = c.cpu().numpy()
            assert np.array_equal(cg, rc) if fmt == 0 else np.array_equal(bits(cg), bits(rc))
            assert np.array_equal(bits(dep.cpu().numpy()), bits(rd))
    # the whole frame through the library equals the oracle's full OnData frame
    rays_o, pix_o = O.camera_rays(d)
    hits_o = O.OracleAccel(O.TRI, *S.displaced_octasphere(6, seed=7)).trace(rays_o)
    rc, rd = O.framebuffer_write(d, hits_o, pix_o, None, 0)
    c, dep = K.framebuffer_write(cam, hits, pix, fmt=0)
    assert np.array_equal(c.cpu().numpy(), rc)
    assert np.array_equal(bits(dep.cpu().numpy()), bits(rd))


def test_camera_arguments_are_checked():
    cam = K.make_camera(64, 64, step=0)
    with pytest.raises(sb.SurfaceError):
        K.camera_rays(cam)
    cam = K.make_camera(64, 64)
    rays, pix = K.camera_rays(cam)
    with pytest.raises(sb.SurfaceError):
        K.framebuffer_write(cam, rays.cpu()[:, :4].contiguous(), pix.cpu(), fmt=0)


# ------------------------------------------------- subsamples, stereo camera
SAMPLE_CASES = [
    (dict(width=160, height=120, eye=(0, 0, 3), lookat=(0, 0, 0), fov=45.0), 2, None, 0),
    (dict(width=97, height=61, eye=(0.3, 0.2, 3), lookat=(0, 0.1, 0), fov=30.0, step=2), 3,
     None, 12345),
    (dict(width=120, height=80, eye=(1, 2, 3), lookat=(0, 0, 0), up=(0, 0, 1), ortho=True,
          viewport=(8, -4, 110, 90), region=(4, 2, 116, 78)), 4, None, 7),
    (dict(width=256, height=128, eye=(0.1, 0.0, 0.2), lookat=(0, 0, -1), fov=45.0), 2,
     (1.5, 0.065), 0),
]
STEREO_TOL = 2e-6  # C library vs CUDA trigonometry, relative


@pytest.mark.parametrize("case,S,stereo,offset", SAMPLE_CASES)
def test_subsample_rays_match_oracle(case, S, stereo, offset):
    """subsamples^2 rays per pixel with the serial renderer's jitter stream
    (jumped to `offset` draws on the host, drawn per row on the GPU) and the
    stereo environment camera, against the restated OnData loop."""
    cam = K.make_camera(**case)
    smp = K.make_samples(S, stereo=stereo, jitter_offset=offset)
    rays, pix = K.camera_rays(cam, samples=smp)
    torch.cuda.synchronize()
    ref, rpix = O.camera_rays_ex(K.camera_dict(cam), S, stereo=stereo, offset=offset)
    got = rays.cpu().numpy().reshape(-1).view(O.RAY_DTYPE)
    assert got.size == ref.size > 0
    assert rays.draws == got.size // (S * S) * 2 * S * (S - 1)
    assert np.array_equal(pix.cpu().numpy().view(np.uint32), rpix)
    for f in ("prev_prim", "prev_t"):
        assert np.array_equal(bits(got[f]), bits(ref[f])), f
    if stereo is None:
        for f in ("org", "dir"):
            assert np.array_equal(bits(got[f]), bits(ref[f])), f
    else:
        for f in ("org", "dir"):
            d = np.abs(got[f].astype(np.float64) - ref[f].astype(np.float64))
            assert d.max() <= STEREO_TOL * max(1.0, np.abs(ref[f]).max()), (f, d.max())
        # nearly all bit-equal: the C library's float sine and cosine are
        # correctly rounded in all but rare cases
        same = np.all(bits(got["dir"]) == bits(ref["dir"]), axis=1).mean()
        assert same > 0.9, same


def test_jitter_offsets_continue_the_stream():
    """Two frames drawn one after the other equal one frame drawn from the
    draw count of the first (the stream's state carried across frames)."""
    cam = K.make_camera(64, 48, eye=(0, 0, 3), lookat=(0, 0, 0), fov=40.0)
    a, _ = K.camera_rays(cam, samples=K.make_samples(3))
    b, _ = K.camera_rays(cam, samples=K.make_samples(3, jitter_offset=a.draws))
    ref_b, _ = O.camera_rays_ex(K.camera_dict(cam), 3, offset=a.draws)
    got = b.cpu().numpy().reshape(-1).view(O.RAY_DTYPE)
    assert np.array_equal(bits(got["dir"]), bits(ref_b["dir"]))
    assert not np.array_equal(bits(a.cpu().numpy()), bits(b.cpu().numpy()))


@pytest.mark.parametrize("S", [2, 3])
def test_subsample_framebuffer_matches_oracle(S):
    """Per pixel the average of its subsamples' hits (colour and depth)."""
    acc = _scene()
    cam = K.make_camera(180, 140, eye=(0.2, 0.1, 2.6), lookat=(0, 0, 0), fov=45.0, step=2)
    smp = K.make_samples(S)
    rays, pix = K.camera_rays(cam, samples=smp)
    hits = acc.Traverse(rays)
    gen = torch.Generator(device="cuda").manual_seed(5)
    rgba = torch.rand((rays.shape[0], 4), device="cuda", generator=gen) * 1.2 - 0.1
    torch.cuda.synchronize()
    h = hits.cpu().numpy().reshape(-1).view(O.HIT_DTYPE)
    p = pix.cpu().numpy().view(np.uint32)
    d = K.camera_dict(cam)
    for fmt in (0, 1):
        col, dep = K.framebuffer_write(cam, hits, pix, rgba, fmt=fmt, samples=smp)
        rc, rd = O.framebuffer_write_ex(d, S, h, p, rgba.cpu().numpy(), fmt=fmt)
        assert col.cpu().numpy().tobytes() == rc.tobytes()
        assert np.array_equal(bits(dep.cpu().numpy()), bits(rd))
    # partial coverage: some pixels averaged over fewer hits than samples
    per = h["prim"].reshape(-1, S * S) != O.MISS
    assert ((per.sum(1) > 0) & (per.sum(1) < S * S)).any()
