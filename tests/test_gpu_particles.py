"""The particle workload's frame on the GPU: advected frames, hemisphere
secondaries (srt_spawn_secondary) against their NumPy statement, and the
secondary trace with the self-hit rule against the CPU oracle (bit-exact)."""
import numpy as np
import pytest
import torch

import surface_b200 as sb
from oracle import oracle as O
from surface_b200 import scenes as S

from conftest import bits

pytestmark = pytest.mark.gpu


def _frame(n=200_000, seed=5, side=256, frame=0):
    pos, rad = S.particles(n, seed=seed)
    if frame:
        pos = S.particle_frames(pos, frame + 1, device="cuda")[frame].cpu().numpy()
    rays = S.pinhole_rays(side, side, (0.5, 0.5, 2.2), (0.5, 0.5, 0.5), fov_deg=30)
    return pos, rad, rays


def _gpu_primaries(pos, rad, rays):
    acc = sb.ParticleAccel()
    acc.Build32(sb.Particles(torch.as_tensor(pos).cuda(), torch.as_tensor(rad).cuda()))
    rt = torch.as_tensor(rays.view(np.float32).reshape(-1, 8)).cuda()
    res = acc.Traverse(rt, want_normal=True)
    return acc, rt, res


def test_spawn_matches_numpy_statement():
    pos, rad, rays = _frame()
    acc, rt, res = _gpu_primaries(pos, rad, rays)
    sec, sn = sb.spawn_secondary(rt, res.hits, res.normal, seed=11)
    torch.cuda.synchronize()
    hits = res.hits.cpu().numpy().reshape(-1).view(O.HIT_DTYPE)
    nrm = res.normal.cpu().numpy()
    ref, refn = S.spawn_secondary_np(rays, hits, nrm, 11)
    got = sec.cpu().numpy().reshape(-1).view(O.RAY_DTYPE)
    assert got.size == ref.size == int((hits["prim"] != O.MISS).sum()) > 1000
    assert np.array_equal(bits(got["org"]), bits(ref["org"]))  # float32 org + t * dir
    assert np.array_equal(got["prev_prim"], ref["prev_prim"])
    assert np.array_equal(bits(got["prev_t"]), bits(ref["prev_t"]))
    assert np.abs(got["dir"] - ref["dir"]).max() < 2e-6
    assert np.abs(sn.cpu().numpy() - refn).max() < 1e-6
    # unit length, in the hemisphere of the normal, cos(theta) ~ U[0, 1)
    d = got["dir"].astype(np.float64)
    assert np.abs(np.linalg.norm(d, axis=1) - 1).max() < 1e-5
    cos = np.einsum("ij,ij->i", d, refn.astype(np.float64))
    assert cos.min() > -1e-6
    assert abs(cos.mean() - 0.5) < 0.01
    # another seed gives other directions
    sec2, _ = sb.spawn_secondary(rt, res.hits, res.normal, seed=12)
    assert not torch.equal(sec2, sec)


def test_secondaries_match_oracle_with_self_hit_rule():
    pos, rad, rays = _frame(n=150_000, seed=9)
    pos[500:700] = pos[500]  # coincident centres
    acc, rt, res = _gpu_primaries(pos, rad, rays)
    sec, sn = sb.spawn_secondary(rt, res.hits, res.normal, seed=3)
    h2 = acc.Traverse(sec, prev_normals=sn)
    h2s = acc.Traverse(sec, prev_normals=sn, single_pass=True)
    torch.cuda.synchronize()
    o = O.OracleAccel(O.SPHERE, pos, None, rad)
    hits = res.hits.cpu().numpy().reshape(-1).view(O.HIT_DTYPE)
    oh = o.trace(rays)
    for f in ("t", "prim"):
        assert np.array_equal(bits(hits[f]), bits(oh[f]))
    sr = sec.cpu().numpy().reshape(-1).view(O.RAY_DTYPE)
    ref = o.trace(sr, prev_normals=sn.cpu().numpy())
    for h in (h2, h2s):
        g = h.cpu().numpy().reshape(-1).view(O.HIT_DTYPE)
        for f in ("t", "prim"):
            bad = np.nonzero(bits(g[f]) != bits(ref[f]))[0]
            assert bad.size == 0, (f, bad[:5])
    assert (ref["prim"] != O.MISS).any()


def test_advected_frame_builds_and_traces_exactly():
    pos, rad, rays = _frame(n=100_000, seed=4, side=128, frame=3)
    v = S.VelocityField(7)
    p = S.particles(100_000, seed=4)[0]
    for _ in range(3):
        p = v.advect(p)
    assert np.abs(p - pos).max() < 1e-5  # torch and NumPy frames agree
    acc, rt, res = _gpu_primaries(pos, rad, rays)
    o = O.OracleAccel(O.SPHERE, pos, None, rad)
    raw, idx, codes = acc.export()
    assert np.array_equal(O.canonicalize(O.generic_from_device(O.SPHERE, raw), 0),
                          o.canonical())
    g = res.hits.cpu().numpy().reshape(-1).view(O.HIT_DTYPE)
    oh = o.trace(rays)
    for f in ("t", "prim"):
        assert np.array_equal(bits(g[f]), bits(oh[f]))


def test_spawn_rejects_host_arrays_and_handles_no_hits():
    pos, rad, rays = _frame(n=20_000, seed=2, side=32)
    acc, rt, res = _gpu_primaries(pos, rad, rays)
    with pytest.raises(sb.SurfaceError):
        sb.spawn_secondary(rt.cpu(), res.hits, res.normal, seed=1)
    miss = torch.zeros_like(res.hits)
    miss.view(torch.int32)[:, 3] = -1  # prim = 0xFFFFFFFF everywhere
    sec, sn = sb.spawn_secondary(rt, miss, res.normal, seed=1)
    assert sec.shape == (0, 8) and sn.shape == (0, 3)
