"""The solid accel on the GPU (srt_solid_*) against the oracle's SolidAccel
Build32 / Traverse, bit for bit: the tree (same pre-order records) and solid
order, per ray the hit (t, solid), its normal and position -- pyramids,
prisms and hexahedra, grid-aligned, pinhole and interior rays, secondary
rays that skip the solid they leave; host and device inputs; Dump() bytes,
BoundingBox, small meshes and bad input."""
import numpy as np
import pytest
import torch

import surface_b200 as sb
from oracle import oracle as O
from surface_b200 import scenes as S
from surface_b200.solids import Solid, SolidAccel

from conftest import bits

pytestmark = pytest.mark.gpu

CASES = {"hexahedra": (8, 14), "prisms": (6, 11), "pyramids": (5, 8)}  # >= 1024 solids


def _check(nv, v, ix, rays, device_inputs=False):
    o = O.OracleSolids(nv, v, ix)
    acc = SolidAccel()
    if device_inputs:
        acc.Build32(Solid(nv, torch.as_tensor(v).cuda(),
                          torch.as_tensor(ix.astype(np.int32)).cuda()))
    else:
        acc.Build32(Solid(nv, v, ix))
    gn, gi = acc.export()
    on, oi = o.export()
    assert gn.tobytes() == on.tobytes()
    assert np.array_equal(gi, oi)
    want, wn, wp = o.trace(rays)
    got, gnrm, gpos = acc.Traverse(rays, want_point=True)
    assert np.array_equal(bits(got.view(np.float32).reshape(-1, 4)),
                          bits(want.view(np.float32).reshape(-1, 4)))
    assert np.array_equal(bits(gnrm), bits(wn)) and np.array_equal(bits(gpos), bits(wp))
    rt = torch.from_numpy(np.ascontiguousarray(rays).view(np.float32).reshape(-1, 8)).cuda()
    gd = acc.Traverse(rt).cpu().numpy()
    assert np.array_equal(bits(gd), bits(want.view(np.float32).reshape(-1, 4)))
    return acc, want, wp


@pytest.mark.parametrize("case", list(CASES))
def test_solids(case):
    nv, g = CASES[case]
    v, ix = S.solid_grid(nv, g, seed=9)
    rays = S.solid_rays(128, seed=nv)
    _, h, p = _check(nv, v, ix, rays, device_inputs=(nv == 6))
    assert 0.5 < (h["prim"] != O.MISS).mean() < 0.95
    ok = h["prim"] != O.MISS
    rng = np.random.default_rng(nv)
    d = rng.normal(size=(ok.sum(), 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays2 = S.make_rays(p[ok], d)
    rays2["prev_prim"] = h["prim"][ok]
    _, h2, _ = _check(nv, v, ix, rays2)
    assert (h2["prim"] != rays2["prev_prim"]).all()


@pytest.mark.parametrize("nsolids", [2, 3, 7, 40])
def test_small_meshes(nsolids):
    v, ix = S.solid_grid(8, 4, seed=2)
    ix = ix[:nsolids]
    _check(8, v, ix, S.solid_rays(32))


@pytest.mark.parametrize("nv,g,m", [(8, 9, 500), (6, 7, 686), (5, 5, 750), (8, 11, 1023)])
def test_sah_build_below_1024(nv, g, m):
    """Fewer than 1024 solids: the reference's binned-SAH Build (host build,
    uploaded tree): tree, order, hits, normals and positions equal the
    oracle's, from host and device inputs."""
    v, ix = S.solid_grid(nv, g, seed=3)
    ix = ix[:m]
    rays = S.solid_rays(64, seed=nv)
    _check(nv, v, ix, rays)
    _check(nv, v, ix, rays, device_inputs=True)


def test_dump_bbox_and_errors(tmp_path):
    v, ix = S.solid_grid(6, 6, seed=4)
    acc = SolidAccel()
    acc.Build32(Solid(6, v, ix))
    acc.Dump(tmp_path / "s.bin")
    nodes, idx = O.parse_solid_dump((tmp_path / "s.bin").read_bytes())
    on, oi = O.OracleSolids(6, v, ix).export()
    assert nodes.tobytes() == on.tobytes() and np.array_equal(idx, oi)
    lo, hi = acc.BoundingBox()
    assert np.array_equal(lo, on[0]["bmin"].astype(np.float64))
    assert np.array_equal(hi, on[0]["bmax"].astype(np.float64))
    bad = ix.copy()
    bad[3, 2] = v.shape[0]
    with pytest.raises(sb.SurfaceError):
        SolidAccel().Build32(Solid(6, v, bad))
    with pytest.raises(sb.SurfaceError):
        SolidAccel().Build32(Solid(7, v, ix))  # 7 vertices per solid


def test_against_reference_fixtures(golden):
    """The CUDA line and solid accels against the reference's own outputs
    (tests/golden/lines_solids.npz), bit for bit."""
    from surface_b200.lines import LineAccel, Lines
    g = golden("lines_solids.npz")
    for tag in ("line", "edge"):
        acc = LineAccel()
        acc.Build(Lines(g[f"{tag}_pos"], g[f"{tag}_seg"], g[f"{tag}_rad"]))
        h, n = acc.Traverse(g[f"{tag}_rays"], want_normal=True)
        assert np.array_equal(bits(h.view(np.float32).reshape(-1, 4)), bits(g[f"{tag}_hits"]))
        assert np.array_equal(bits(n), bits(g[f"{tag}_normals"]))
    for nv in (8, 6, 5):
        acc = SolidAccel()
        acc.Build32(Solid(nv, g[f"solid{nv}_verts"], g[f"solid{nv}_ix"]))
        nodes, idx = acc.export()
        assert O.tree_canonical(nodes) == O.tree_canonical(
            g[f"solid{nv}_nodes"].view(O.SOLID_NODE_DTYPE))
        assert np.array_equal(idx, g[f"solid{nv}_idx"])
        h, n, q = acc.Traverse(g[f"solid{nv}_rays"], want_point=True)
        assert np.array_equal(bits(h.view(np.float32).reshape(-1, 4)), bits(g[f"solid{nv}_hits"]))
        assert np.array_equal(bits(n), bits(g[f"solid{nv}_normals"]))
        assert np.array_equal(bits(q), bits(g[f"solid{nv}_positions"]))


def test_rebuild_and_trace_across_streams():
    """Builds from device arrays run in torch's stream order and the trace
    waits for the accel's latest build even when it is issued on another
    stream; the next build waits for the latest trace.  Every step's hits
    equal the oracle's."""
    v, ix = S.solid_grid(8, 24, seed=11)
    rays = S.pinhole_rays(192, 192, (1.7, 1.3, 2.1), (0.5, 0.5, 0.5), fov_deg=50)
    want, _, _ = O.OracleSolids(8, v, ix).trace(rays)
    acc = SolidAccel()
    dv = torch.as_tensor(v).cuda()
    dix = torch.as_tensor(ix.view(np.int32)).cuda()
    rt = torch.from_numpy(rays.view(np.float32).reshape(-1, 8)).cuda()
    s_build, s_trace = torch.cuda.Stream(), torch.cuda.Stream()
    torch.cuda.synchronize()  # the inputs' copies ran on the default stream
    outs = []
    for k in range(4):
        with torch.cuda.stream(s_build):
            acc.Build32(Solid(8, dv, dix))
        with torch.cuda.stream(s_trace):
            outs.append(acc.Traverse(rt))
    torch.cuda.synchronize()
    for h in outs:
        assert np.array_equal(bits(h.cpu().numpy()), bits(want.view(np.float32).reshape(-1, 4)))
    n, nn = acc.info()
    assert n == ix.shape[0] and nn > 1


@pytest.mark.parametrize("nv,g,m,shift", [(8, 11, None, 0.0), (6, 8, None, 100.0),
                                          (5, 6, None, 0.0), (8, 9, 400, 0.0)])
def test_double_positions(nv, g, m, shift):
    """Double-precision positions (float64 vertices: Solid::dvertices): the
    GPU Build32 (and the SAH Build below 1024 solids) and trace equal the
    oracle's, which equals the reference's, from host and device inputs."""
    v, ix = S.solid_grid(nv, g, seed=nv)
    rng = np.random.default_rng(nv + 100)
    v64 = v.astype(np.float64) + shift + rng.uniform(-1e-9, 1e-9, size=v.shape)
    if m is not None:
        ix = ix[:m]
    rays = S.solid_rays(64, seed=nv)
    rays["org"] += np.float32(shift)
    _check(nv, v64, ix, rays)
    _check(nv, v64, ix, rays, device_inputs=True)


def test_double_position_solids_in_a_scene():
    """A double-precision solid element beside a triangle element: the scene
    trace's per-ray loop walks it with the double records."""
    from surface_b200.scene import RenderGraph
    v, ix = S.solid_grid(8, 11, seed=4)
    v64 = v.astype(np.float64) - 0.5 + np.random.default_rng(3).uniform(-1e-9, 1e-9, v.shape)
    tv, tf = S.displaced_octasphere(3, seed=5)
    Ts = [S.affine((0, 0, 1), 30, (1.0, 1.2, 0.8), (-1.0, 0, 0)), S.affine(scale=(0.6,) * 3,
                                                                             translate=(1.2, 0, 0))]
    solid = SolidAccel()
    solid.Build32(Solid(8, v64, ix))
    tri = sb.TriangleAccel()
    tri.Build32(sb.Mesh(tv, tf))
    g = RenderGraph()
    g.AddRenderElement(solid, Ts[0])
    g.AddRenderElement(tri, Ts[1])
    g.Build()
    oacc = [O.OracleSolids(8, v64, ix), O.OracleAccel(O.TRI, tv, tf)]
    mats, wlo, whi = [], [], []
    for a, T in zip((solid, tri), Ts):
        lo, hi = a.BoundingBox()
        i1, i2, b0, b1 = O.element_update(T, lo, hi)
        mats.append((np.asarray(T).reshape(16), i1.reshape(16), i2.reshape(16)))
        wlo.append(b0)
        whi.append(b1)
    o = O.OracleScene(oacc, [m[0] for m in mats], [m[1] for m in mats], [m[2] for m in mats],
                      wlo, whi)
    wlo, whi = np.array(wlo), np.array(whi)
    rays = S.scene_rays(40_000, wlo.min(0), whi.max(0), seed=6, boxes=(wlo, whi))
    want, wel = o.trace(rays)
    assert set(wel[wel != S.MISS].tolist()) == {0, 1}
    got, gel = g.Trace(rays)
    assert np.array_equal(gel, wel)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


@pytest.mark.parametrize("nv,g,dbl", [(8, 14, False), (6, 11, True)])
def test_sah_build_at_every_size(nv, g, dbl):
    """SolidAccel::Build (binned SAH at every size, the GLES builder's
    choice): the uploaded tree, order and hits equal the oracle's."""
    v, ix = S.solid_grid(nv, g, seed=nv)
    if dbl:
        v = v.astype(np.float64) + np.random.default_rng(1).uniform(-1e-9, 1e-9, v.shape)
    o = O.OracleSolids(nv, v, ix, sah=True)
    acc = SolidAccel()
    acc.Build(Solid(nv, v, ix))
    gn, gi = acc.export()
    on, oi = o.export()
    assert gn.tobytes() == on.tobytes() and np.array_equal(gi, oi)
    rays = S.solid_rays(64, seed=nv)
    want, wn, wp = o.trace(rays)
    got, gnrm, gpos = acc.Traverse(rays, want_point=True)
    assert np.array_equal(bits(got.view(np.float32).reshape(-1, 4)),
                          bits(want.view(np.float32).reshape(-1, 4)))
    assert np.array_equal(bits(gnrm), bits(wn)) and np.array_equal(bits(gpos), bits(wp))
