"""srt_trace_closest_noalloc through the C ABI: the same hits as
srt_trace_closest (bit-exact, the tolerance of every trace test here) on two
calls in a row for triangles, tetrahedra and spheres; free device memory
unchanged by calls after the set-up call; the per-call ray limit."""
import ctypes as C

import numpy as np
import pytest
import torch

import surface_b200 as sb
from surface_b200 import _lib
from surface_b200 import scenes as S

from conftest import bits

pytestmark = pytest.mark.gpu

MAX_RAYS = 262144


def dev_rays(rays):
    return torch.as_tensor(rays.view(np.float32).reshape(-1, 8)).cuda()


def noalloc(acc, rays, hits):
    return acc.L.srt_trace_closest_noalloc(acc.h, C.c_void_p(rays.data_ptr()), rays.shape[0],
                                           C.c_void_p(hits.data_ptr()))


def scenes():
    v, f = S.displaced_octasphere(7)
    tri = sb.TriangleAccel()
    tri.Build32(sb.Mesh(torch.as_tensor(v).cuda(), torch.as_tensor(f.view(np.int32)).cuda()))
    vt, ft, _ = S.tet_grid(16, seed=5)
    tet = sb.TetraAccel()
    tet.Build32(sb.Tetrahedron(torch.as_tensor(vt).cuda(),
                               torch.as_tensor(ft.view(np.int32)).cuda()))
    pos, rad = S.particles(200000, seed=6)
    sph = sb.ParticleAccel()
    sph.Build32(sb.Particles(torch.as_tensor(pos).cuda(), torch.as_tensor(rad).cuda()))
    return [
        (tri, dev_rays(S.pinhole_rays(512, 512, (0, 0, 3), (0, 0, 0)))),  # exactly the limit
        (tet, dev_rays(S.ortho_rays(256, 256))),
        (sph, dev_rays(S.pinhole_rays(256, 256, (0.5, 0.5, 2.2), (0.5, 0.5, 0.5),
                                      fov_deg=30))),
    ]


def test_noalloc_matches_trace_closest_twice_and_allocates_nothing():
    cases = scenes()
    refs = [acc.Traverse(r) for acc, r in cases]
    outs = [(torch.full_like(h, float("nan")), torch.full_like(h, float("nan"))) for h in refs]
    # set-up call on this device, then measure
    for (acc, r), (h1, _) in zip(cases, outs):
        assert noalloc(acc, r, h1) == _lib.SRT_OK, _lib.load().srt_last_error()
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for (acc, r), (h1, h2) in zip(cases, outs):
        h1.fill_(float("nan"))
        assert noalloc(acc, r, h1) == _lib.SRT_OK
        assert noalloc(acc, r, h2) == _lib.SRT_OK
    for (acc, _), _ in zip(cases, outs):
        _lib.check(acc.L.srt_ctx_synchronize(acc.ctx.h))
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    for ref, (h1, h2) in zip(refs, outs):
        want = bits(ref.cpu().numpy())
        assert np.array_equal(bits(h1.cpu().numpy()), want)
        assert np.array_equal(bits(h2.cpu().numpy()), want)
        assert (ref[:, 3].view(torch.int32) != -1).any()


def test_noalloc_limits_and_arguments():
    acc, r = scenes()[0]
    L = acc.L
    big = torch.zeros((MAX_RAYS + 1, 8), device="cuda")
    hits = torch.zeros((MAX_RAYS + 1, 4), device="cuda")
    assert noalloc(acc, big, hits) == _lib.SRT_ERR_LIMIT
    assert b"262144" in L.srt_last_error()
    host_r = np.zeros((16, 8), np.float32)
    host_h = np.zeros((16, 4), np.float32)
    assert L.srt_trace_closest_noalloc(acc.h, host_r.ctypes.data, 16,
                                       host_h.ctypes.data) == _lib.SRT_ERR_INVALID
    assert L.srt_trace_closest_noalloc(acc.h, None, 0, None) == _lib.SRT_OK
    assert L.srt_trace_closest_noalloc(None, None, 0, None) == _lib.SRT_ERR_INVALID
