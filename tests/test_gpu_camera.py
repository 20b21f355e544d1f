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
