"""Scenes of transformed accels (srt_scene_*, RenderGraph) on the GPU against
the oracle, bit for bit: the top-level tree, primary rays and secondary
rays that leave a hit element (self-hit rule inside prev_element only), for
triangle, tetrahedron, particle, line and solid elements."""
import numpy as np
import pytest
import torch

import surface_b200 as sb
from oracle import oracle as O
from surface_b200 import scenes as S
from surface_b200.scene import RenderGraph

from conftest import bits

pytestmark = pytest.mark.gpu

KIND = {0: (O.TRI, sb.TriangleAccel), 1: (O.TET, sb.TetraAccel), 2: (O.SPHERE, sb.ParticleAccel)}


def gpu_accel(e):
    if e["kind"] == 3:
        acc = sb.LineAccel()
        acc.Build(sb.Lines(e["verts"], e["segments"], e["radius"]))
        return acc
    if e["kind"] == 4:
        acc = sb.SolidAccel()
        acc.Build32(sb.Solid(e["nv"], e["verts"], e["faces"]))
        return acc
    cls = KIND[e["kind"]][1]
    acc = cls()
    if e["kind"] == 0:
        acc.Build32(sb.Mesh(e["verts"], e["faces"]))
    elif e["kind"] == 1:
        acc.Build32(sb.Tetrahedron(e["verts"], e["faces"]))
    else:
        acc.Build32(sb.Particles(e["verts"], e["radius"]))
    return acc


def oracle_accel(e):
    if e["kind"] == 3:
        return O.OracleLines(e["verts"], e["segments"], e["radius"])
    if e["kind"] == 4:
        return O.OracleSolids(e["nv"], e["verts"], e["faces"])
    k = KIND[e["kind"]][0]
    if e["kind"] == 2:
        return O.OracleAccel(k, e["verts"], None, e["radius"])
    return O.OracleAccel(k, e["verts"], e["faces"])


def make_pair(elems):
    gacc = [gpu_accel(e) for e in elems]
    oacc = [oracle_accel(e) for e in elems]
    g = RenderGraph()
    T, iT, iT33, wlo, whi = [], [], [], [], []
    for e, a in zip(elems, gacc):
        assert g.AddRenderElement(a, e["T"]) == len(T)
        lo, hi = a.BoundingBox()
        i1, i2, b0, b1 = O.element_update(e["T"], lo, hi)
        T.append(np.asarray(e["T"]).reshape(16))
        iT.append(i1.reshape(16))
        iT33.append(i2.reshape(16))
        wlo.append(b0)
        whi.append(b1)
    g.Build()
    o = O.OracleScene(oacc, T, iT, iT33, wlo, whi)
    return g, o, gacc, np.array(wlo), np.array(whi)


# Hits on sphere elements carry the spherical (u, v) of the element accel's
# Traverse, from double atan2 / acos (the C library's in the oracle, CUDA's
# here): equal to an ulp or two.  Everything else is bit for bit.
SPHERE_UV_TOL = 1e-6


def sphere_mask(gacc):
    return np.array([isinstance(a, sb.ParticleAccel) for a in gacc])


def assert_same(got, gel, want, wel, sph=None):
    h = got.cpu().numpy() if isinstance(got, torch.Tensor) else got.view(np.float32)
    e = gel.cpu().numpy().view(np.uint32) if isinstance(gel, torch.Tensor) else gel
    assert np.array_equal(e, wel)
    h = np.ascontiguousarray(h).reshape(-1, 4)
    w = np.ascontiguousarray(want.view(np.float32)).reshape(-1, 4)
    on_sphere = np.zeros(len(w), bool)
    if sph is not None:
        hit = wel != S.MISS
        on_sphere[hit] = sph[wel[hit]]
    # t and prim everywhere, u and v off spheres: bit for bit
    assert np.array_equal(bits(h[:, [0, 3]]), bits(w[:, [0, 3]]))
    assert np.array_equal(bits(h[~on_sphere][:, 1:3]), bits(w[~on_sphere][:, 1:3]))
    if on_sphere.any():
        d = np.abs(h[on_sphere][:, 1:3].astype(np.float64) - w[on_sphere][:, 1:3])
        assert d.max() <= SPHERE_UV_TOL, d.max()


@pytest.fixture(scope="module")
def mixed():
    elems = S.scene_elements(seed=31)
    return (elems,) + make_pair(elems)


def test_top_tree_matches_oracle(mixed):
    _, g, o, _, _, _ = mixed
    gb, gi = g.top_nodes()
    ob, oi = o.nodes()
    assert np.array_equal(gi, oi)
    assert np.array_equal(bits(gb), bits(ob))


def test_primary_rays_match_oracle(mixed):
    _, g, o, gacc, wlo, whi = mixed
    sph = sphere_mask(gacc)
    rays = S.scene_rays(200_000, wlo.min(0), whi.max(0), seed=9, boxes=(wlo, whi))
    want, wel = o.trace(rays)
    assert (wel != S.MISS).mean() > 0.2
    rt = torch.from_numpy(rays.view(np.float32).reshape(-1, 8)).cuda()
    hits, el = g.Trace(rt)
    torch.cuda.synchronize()
    assert_same(hits, el, want, wel, sph)
    # host arrays through the same entry point
    h2, e2 = g.Trace(rays[:5000])
    assert_same(h2, e2, want[:5000], wel[:5000], sph)


def test_secondary_rays_match_oracle(mixed):
    _, g, o, gacc, wlo, whi = mixed
    rays = S.scene_rays(100_000, wlo.min(0), whi.max(0), seed=12, boxes=(wlo, whi))
    want, wel = o.trace(rays)
    hit = np.nonzero(wel != S.MISS)[0]
    rng = np.random.default_rng(2)
    sec = np.zeros(hit.size, O.RAY_DTYPE)
    sec["org"] = rays["org"][hit] + want["t"][hit, None] * rays["dir"][hit]
    sec["dir"] = S._normalize(rng.normal(size=(hit.size, 3))).astype(np.float32)
    sec["prev_prim"] = want["prim"][hit]
    sec["prev_t"] = want["t"][hit]
    pe = wel[hit]
    pn = S._normalize(rng.normal(size=(hit.size, 3))).astype(np.float32)
    w2, we2 = o.trace(sec, pe, pn)
    st = torch.from_numpy(sec.view(np.float32).reshape(-1, 8)).cuda()
    hits, el = g.Trace(st, torch.from_numpy(pe.view(np.int32)).cuda(), torch.from_numpy(pn).cuda())
    torch.cuda.synchronize()
    assert_same(hits, el, w2, we2, sphere_mask(gacc))


@pytest.fixture(scope="module")
def with_lines_solids():
    elems = S.scene_elements(seed=43, ntri=1, nsph=1, ntet=1, nline=2, nsolid=3)
    return (elems,) + make_pair(elems)


def test_line_and_solid_elements_match_oracle(with_lines_solids):
    """Line and solid elements (walked by the per-ray loop) beside the
    accels of the rounds: primary rays, then secondary rays leaving the hit
    element (a solid skips the solid it leaves)."""
    elems, g, o, gacc, wlo, whi = with_lines_solids
    sph = sphere_mask(gacc)
    gb, gi = g.top_nodes()
    ob, oi = o.nodes()
    assert np.array_equal(gi, oi) and np.array_equal(bits(gb), bits(ob))
    rays = S.scene_rays(60_000, wlo.min(0), whi.max(0), seed=9, boxes=(wlo, whi))
    want, wel = o.trace(rays)
    kinds = np.array([e["kind"] for e in elems])
    got_kinds = set(kinds[wel[wel != S.MISS]].tolist())
    assert got_kinds == {0, 1, 2, 3, 4}
    hits, el = g.Trace(torch.from_numpy(rays.view(np.float32).reshape(-1, 8)).cuda())
    torch.cuda.synchronize()
    assert_same(hits, el, want, wel, sph)
    hit = np.nonzero(wel != S.MISS)[0]
    rng = np.random.default_rng(5)
    sec = np.zeros(hit.size, O.RAY_DTYPE)
    sec["org"] = rays["org"][hit] + want["t"][hit, None] * rays["dir"][hit]
    sec["dir"] = S._normalize(rng.normal(size=(hit.size, 3))).astype(np.float32)
    sec["prev_prim"] = want["prim"][hit]
    sec["prev_t"] = want["t"][hit]
    pe = wel[hit]
    pn = S._normalize(rng.normal(size=(hit.size, 3))).astype(np.float32)
    w2, we2 = o.trace(sec, pe, pn)
    h2, e2 = g.Trace(torch.from_numpy(sec.view(np.float32).reshape(-1, 8)).cuda(),
                     torch.from_numpy(pe.view(np.int32)).cuda(), torch.from_numpy(pn).cuda())
    torch.cuda.synchronize()
    assert_same(h2, e2, w2, we2, sph)


def test_many_instances_of_one_accel():
    """One accel under 40 transforms (instancing), touching and overlapping
    world boxes."""
    v, f = S.displaced_octasphere(4, seed=3)
    p, r = S.particles(3000, seed=4, median_radius=0.02)
    rng = np.random.default_rng(8)
    elems = []
    for j in range(40):
        T = S.affine(rng.normal(size=3), rng.uniform(0, 360), rng.uniform(0.3, 1.2, size=3),
                     rng.uniform(-6, 6, size=3))
        if j % 4 == 3:
            elems.append(dict(kind=2, verts=p, radius=r, T=T))
        else:
            elems.append(dict(kind=0, verts=v, faces=f, T=T))
    g, o, gacc, wlo, whi = make_pair(elems)
    gb, gi = g.top_nodes()
    ob, oi = o.nodes()
    assert np.array_equal(gi, oi) and np.array_equal(bits(gb), bits(ob))
    rays = S.scene_rays(100_000, wlo.min(0), whi.max(0), seed=3, boxes=(wlo, whi))
    want, wel = o.trace(rays)
    hits, el = g.Trace(torch.from_numpy(rays.view(np.float32).reshape(-1, 8)).cuda())
    torch.cuda.synchronize()
    assert_same(hits, el, want, wel, sphere_mask(gacc))


def test_explicit_matrices_and_errors(mixed):
    elems, g, o, gacc, wlo, whi = mixed
    g2 = RenderGraph()
    for e, a in zip(elems, gacc):
        lo, hi = a.BoundingBox()
        i1, i2, b0, b1 = O.element_update(e["T"], lo, hi)
        g2.add_element_matrices(a, e["T"], i1, i2, b0, b1)
    with pytest.raises(sb.SurfaceError):
        g2.Trace(np.zeros(4, O.RAY_DTYPE))  # not built
    g2.Build()
    assert np.array_equal(bits(g2.top_nodes()[0]), bits(g.top_nodes()[0]))
    rays = S.scene_rays(20_000, wlo.min(0), whi.max(0), seed=1, boxes=(wlo, whi))
    h1, e1 = g.Trace(rays)
    h2, e2 = g2.Trace(rays)
    assert np.array_equal(e1, e2) and np.array_equal(h1.view(np.uint32), h2.view(np.uint32))
    with pytest.raises(sb.SurfaceError):
        RenderGraph().Build()  # empty scene
    with pytest.raises(sb.SurfaceError):
        RenderGraph().AddRenderElement(sb.TriangleAccel(), np.eye(4))  # not built


def test_deep_line_element_in_a_scene():
    """A line element whose tree is 90 levels deep (a chain of segments at
    midpoints 2^-k, every split peels one off) beside a triangle element:
    the per-ray loop runs with the long walk stack and equals the oracle."""
    name, pos, seg, rad, constr, opts, rays = [c for c in S.line_cases() if c[0] == "chain"][0]
    lines = sb.LineAccel()
    lines.Build(sb.Lines(pos, seg, rad, constr), sb.LineBuildOptions(minLeafPrimitives=1))
    assert lines.info()[2] > 62
    tv, tf = S.displaced_octasphere(2, seed=8)
    tri = sb.TriangleAccel()
    tri.Build32(sb.Mesh(tv, tf))
    Ts = [np.eye(4), S.affine(scale=(0.3,) * 3, translate=(0.5, 0.8, 0.0))]
    g = RenderGraph()
    g.AddRenderElement(lines, Ts[0])
    g.AddRenderElement(tri, Ts[1])
    g.Build()
    oacc = [O.OracleLines(pos, seg, None, constr, min_leaf=1), O.OracleAccel(O.TRI, tv, tf)]
    mats, wlo, whi = [], [], []
    for a, T in zip((lines, tri), Ts):
        lo, hi = a.BoundingBox()
        i1, i2, b0, b1 = O.element_update(T, lo, hi)
        mats.append((np.asarray(T, np.float64).reshape(16), i1.reshape(16), i2.reshape(16)))
        wlo.append(b0)
        whi.append(b1)
    o = O.OracleScene(oacc, [m[0] for m in mats], [m[1] for m in mats], [m[2] for m in mats],
                      wlo, whi)
    want, wel = o.trace(rays)
    assert (wel == 0).sum() > 10
    got, gel = g.Trace(rays)
    assert np.array_equal(gel, wel)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
