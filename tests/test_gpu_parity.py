"""CUDA path vs the CPU oracle (and the reference's golden fixtures).

Bit-exact bar for integer/index work (Morton codes, sorted order, Karras tree,
canonical topology, leaf ranges) and for the boxes and hits, which the kernels
compute with the reference's own float/double operation order."""
import os
import tempfile

import numpy as np
import pytest

import surface_b200 as sb
from oracle import oracle as O
from surface_b200 import scenes as S

from conftest import bits

pytestmark = pytest.mark.gpu

KIND = {O.TRI: sb.TriangleAccel, O.TET: sb.TetraAccel, O.SPHERE: sb.ParticleAccel}


def gpu_build(kind, verts, faces=None, radius=None):
    acc = KIND[kind]()
    if kind == O.TRI:
        acc.Build32(sb.Mesh(verts, faces))
    elif kind == O.TET:
        acc.Build32(sb.Tetrahedron(verts, faces))
    else:
        acc.Build32(sb.Particles(verts, radius))
    return acc


def gpu_canonical(acc, kind):
    raw, idx, codes = acc.export()
    g = O.generic_from_device(kind, raw)
    return O.canonicalize(g, 0), idx, codes


def assert_hits_equal(h, ref, fields=("t", "u", "v", "prim")):
    for f in fields:
        a, b = bits(h[f]), bits(ref[f])
        bad = np.nonzero(a != b)[0]
        assert bad.size == 0, f"{f}: {bad.size} mismatches, first at {bad[:5]}"


# Sphere hits carry BuildIntersection's spherical (u, v): evaluated with the C
# library's double atan2 / acos in the reference and CUDA's on the GPU, which
# may differ in the last bits of the double; after rounding to float that is
# at most an ulp or two.  t and prim stay bit-exact.
SPHERE_UV_TOL = 1e-6


def assert_sphere_hits(h, ref):
    assert_hits_equal(h, ref, ("t", "prim"))
    hit = ref["prim"] != O.MISS
    for f in ("u", "v"):
        assert np.array_equal(bits(h[f][~hit]), bits(ref[f][~hit])), f
        d = np.abs(h[f][hit].astype(np.float64) - ref[f][hit].astype(np.float64))
        assert d.size == 0 or d.max() <= SPHERE_UV_TOL, f"{f}: max |diff| {d.max()}"


def trace_both(acc, rays, **kw):
    """Trace with the default two-pass walk, the single-pass walk in the
    reference's order, the default walk in sorted ray order and both walks
    launched over a full grid instead of persistent warps; all must agree bit
    for bit.  Returns the first."""
    a = acc.Traverse(rays, **kw)
    for other in (acc.Traverse(rays, single_pass=True, **kw),
                  acc.Traverse(rays, sort_rays=True, **kw),
                  acc.Traverse(rays, grid_launch=True, **kw),
                  acc.Traverse(rays, single_pass=True, grid_launch=True, **kw)):
        ha = a.hits if hasattr(a, "hits") else a
        hb = other.hits if hasattr(other, "hits") else other
        assert_hits_equal(ha, hb)
        if hasattr(a, "subface") and a.subface is not None:
            assert np.array_equal(a.subface, other.subface)
        if hasattr(a, "scalar") and a.scalar is not None:
            assert np.array_equal(bits(a.scalar), bits(other.scalar))
        if hasattr(a, "normal") and a.normal is not None:
            assert np.array_equal(bits(a.normal), bits(other.normal))
    return a


# ---------------------------------------------------------------- stages
def test_morton_stage_matches_oracle():
    v, f = S.displaced_octasphere(6, seed=11)
    codes, box = sb.stage_morton(sb.accel.SRT_TRIANGLES, v, f)
    lo = np.zeros(3, np.float32)
    hi = np.zeros(3, np.float32)
    O.lib().so_bbox_tris(O._ptr(v), O._ptr(f), f.shape[0], O._ptr(lo), O._ptr(hi))
    assert np.array_equal(bits(box), bits(np.concatenate([lo, hi])))
    ref = np.zeros(f.shape[0], np.uint32)
    O.lib().so_morton_tris(O._ptr(v), O._ptr(f), f.shape[0], O._ptr(lo), O._ptr(hi),
                           O._ptr(ref))
    assert np.array_equal(codes, ref)
    # tetrahedra and points
    vt, ft, _ = S.tet_grid(10, seed=2)
    codes, box = sb.stage_morton(sb.accel.SRT_TETRAHEDRA, vt, ft)
    O.lib().so_bbox_tets(O._ptr(vt), O._ptr(ft), ft.shape[0], O._ptr(lo), O._ptr(hi))
    ref = np.zeros(ft.shape[0], np.uint32)
    O.lib().so_morton_tets(O._ptr(vt), O._ptr(ft), ft.shape[0], O._ptr(lo), O._ptr(hi),
                           O._ptr(ref))
    assert np.array_equal(codes, ref)
    pos, rad = S.particles(50000, seed=3)
    codes, box = sb.stage_morton(sb.accel.SRT_SPHERES, pos, None, rad)
    O.lib().so_bbox_spheres(O._ptr(pos), O._ptr(rad), 0.0, pos.shape[0], O._ptr(lo),
                            O._ptr(hi))
    assert np.array_equal(bits(box), bits(np.concatenate([lo, hi])))
    assert np.array_equal(codes, O.morton_points(pos, lo, hi))


@pytest.mark.parametrize("n", [2, 8, 1023, 1024, 4097, 100_000, 3_456_663])
def test_sort_stage_is_stable_and_exact(n):
    rng = np.random.default_rng(n)
    codes = rng.integers(0, 1 << 30, size=n, dtype=np.uint32)
    codes[::3] = codes[0]  # many ties
    c, i = sb.stage_sort_pairs(codes)
    rc, ri = O.sort_pairs(codes)
    assert np.array_equal(c, rc)
    assert np.array_equal(i, ri)


@pytest.mark.parametrize("n", [131_071, 131_072, 131_073, 200_000, 262_144, 262_145])
def test_build_sort_paths_by_size(n):
    """The build sorts up to 2^18 codes with one look-back kernel per pass,
    more with the histogram / scan / scatter passes: sorted codes, order,
    tree and boxes exact on either side of the switch and at tile sizes."""
    v, f = S.octasphere_for_count(n, seed=n)
    f = f[:n]
    o, acc = _compare_build(O.TRI, v, f)
    rays = S.pinhole_rays(64, 64, (0, 0, 3), (0, 0, 0))
    assert_hits_equal(acc.Traverse(rays), o.trace(rays))


def test_karras_stage_matches_reference_fixture(golden):
    g = golden("prefix_tree.npz")
    for n in [8, 15, 31, 1023, 1000, 3211]:
        for pre in ("", "same_"):
            sc = np.sort(g[f"{pre}codes_{n}"])
            child, lt, rt = sb.stage_karras(sc)
            assert np.array_equal(child, g[f"{pre}child_{n}"])
            assert np.array_equal(lt, g[f"{pre}ltype_{n}"])
            assert np.array_equal(rt, g[f"{pre}rtype_{n}"])


def test_karras_stage_large():
    rng = np.random.default_rng(1)
    codes = np.sort(rng.integers(0, 1 << 30, size=2_000_000, dtype=np.uint32))
    codes[1000:5000] = codes[1000]
    codes = np.sort(codes)
    child, lt, rt = sb.stage_karras(codes)
    oc, olt, ort = O.karras(codes)
    assert np.array_equal(child, oc) and np.array_equal(lt, olt) and np.array_equal(rt, ort)


# ---------------------------------------------------------------- golden scenes
@pytest.mark.parametrize("tag,kind", [("tri", O.TRI), ("tet", O.TET), ("sph", O.SPHERE)])
def test_build_and_trace_match_reference_fixture(golden, tag, kind):
    g = golden("scenes_small.npz")
    if kind == O.TRI:
        acc = gpu_build(kind, g["tri_verts"], g["tri_faces"])
    elif kind == O.TET:
        acc = gpu_build(kind, g["tet_verts"], g["tet_faces"])
    else:
        acc = gpu_build(kind, g["sph_pos"], None, g["sph_rad"])
    can, idx, _ = gpu_canonical(acc, kind)
    assert np.array_equal(can, g[f"{tag}_canon"])
    assert np.array_equal(idx, g[f"{tag}_index"])
    lo, hi = acc.BoundingBox()
    assert np.array_equal(np.concatenate([lo, hi]), g[f"{tag}_bbox"])
    if kind == O.TET:
        res = trace_both(acc, g["tet_rays"], want_subface=True)
        assert_hits_equal(res.hits, g["tet_hits"])
        assert np.array_equal(res.subface, g["tet_subface"])
    elif kind == O.TRI:
        assert_hits_equal(trace_both(acc, g["tri_rays"]), g["tri_hits"])
    else:
        assert_sphere_hits(trace_both(acc, g["sph_rays"]), g["sph_hits"])
        h2 = trace_both(acc, g["sph_sec_rays"], prev_normals=g["sph_sec_normals"])
        assert_sphere_hits(h2, g["sph_sec_hits"])


# ---------------------------------------------------------------- vs oracle
def _compare_build(kind, verts, faces=None, radius=None):
    o = O.OracleAccel(kind, verts, faces, radius)
    acc = gpu_build(kind, verts, faces, radius)
    can, idx, codes = gpu_canonical(acc, kind)
    oc = o.canonical()
    assert can.shape == oc.shape, (can.shape, oc.shape)
    assert np.array_equal(can, oc)
    assert np.array_equal(idx, o.indices)
    assert np.array_equal(codes, o.codes)
    inf = acc.info()
    assert inf.num_prims == o.n
    return o, acc


@pytest.mark.parametrize("levels", [0, 1, 3, 5, 7])
def test_triangles_build_and_trace(levels):
    v, f = S.displaced_octasphere(levels, seed=100 + levels)
    o, acc = _compare_build(O.TRI, v, f)
    rays = S.pinhole_rays(128, 128, (0, 0, 3), (0, 0, 0))
    assert_hits_equal(trace_both(acc, rays), o.trace(rays))


@pytest.mark.parametrize("n", [2, 3, 17, 18, 1023, 1024, 1025, 5000])
def test_triangle_counts_at_boundaries(n):
    v, f = S.octasphere_for_count(max(n, 8), seed=n)
    f = f[:n]
    o, acc = _compare_build(O.TRI, v, f)
    rays = S.pinhole_rays(48, 48, (0, 0, 3), (0, 0, 0))
    assert_hits_equal(trace_both(acc, rays), o.trace(rays))


@pytest.mark.parametrize("cells", [2, 8, 20])
def test_tetra_build_and_trace(cells):
    v, f, sc = S.tet_grid(cells, seed=cells)
    o, acc = _compare_build(O.TET, v, f)
    for rays in (S.ortho_rays(96, 96),
                 S.pinhole_rays(64, 64, (1.7, 1.3, 2.1), (0.5, 0.5, 0.5), fov_deg=50)):
        import torch
        res = trace_both(acc, rays, want_subface=True)
        oh, osub, osc = o.trace(rays, want_subface=True, vertex_scalar=sc)
        assert_hits_equal(res.hits, oh)
        assert np.array_equal(res.subface, osub)
        # barycentric scalar at the entering point (needs the scalar on device)
        acc_t = torch.as_tensor(rays.view(np.float32).reshape(-1, 8)).cuda()
        r2 = acc.Traverse(acc_t, vertex_scalar=torch.as_tensor(sc).cuda(), want_scalar=True)
        torch.cuda.synchronize()
        assert np.array_equal(bits(r2.scalar.cpu().numpy()), bits(osc))


@pytest.mark.parametrize("cells,shift", [(12, 0.0), (24, 100.0)])
def test_tetra_double_positions(cells, shift):
    """Double-precision positions (float64 vertices: Tetrahedron::dvertices):
    tree, order and codes equal the oracle's, whose build and trace equal the
    reference's; hits, entering faces and the interpolated scalar bit for bit
    under every walk, and the shading records."""
    import torch
    v, f, sc = S.tet_grid(cells, seed=cells)
    v64 = v.astype(np.float64) + shift + np.random.default_rng(cells).uniform(-1e-9, 1e-9,
                                                                             v.shape)
    o, acc = _compare_build(O.TET, v64, f)
    for rays in (S.ortho_rays(96, 96),
                 S.pinhole_rays(64, 64, (1.7, 1.3, 2.1), (0.5, 0.5, 0.5), fov_deg=50)):
        rays["org"] += np.float32(shift)
        res = trace_both(acc, rays, want_subface=True)
        oh, osub, osc = o.trace(rays, want_subface=True, vertex_scalar=sc)
        assert_hits_equal(res.hits, oh)
        assert np.array_equal(res.subface, osub)
        rt = torch.as_tensor(rays.view(np.float32).reshape(-1, 8)).cuda()
        r2 = acc.Traverse(rt, vertex_scalar=torch.as_tensor(sc).cuda(), want_scalar=True,
                          want_isect=True, want_subface=True)
        torch.cuda.synchronize()
        assert np.array_equal(bits(r2.scalar.cpu().numpy()), bits(osc))
        rec = r2.isect.cpu().numpy().reshape(-1).view(O.ISECT_DTYPE)
        orec = o.isect(rays, oh, osub)
        for fld in rec.dtype.names:
            assert np.array_equal(bits(rec[fld]), bits(orec[fld])), fld
    # device-resident float64 inputs take the same path
    acc2 = sb.TetraAccel()
    acc2.Build32(sb.Tetrahedron(torch.as_tensor(v64).cuda(),
                                torch.as_tensor(f.astype(np.int32)).cuda()))
    rays = S.ortho_rays(96, 96)
    rays["org"] += np.float32(shift)
    assert_hits_equal(acc2.Traverse(rays), o.trace(rays))


def test_spheres_build_trace_and_self_hit_rule():
    pos, rad = S.particles(200_000, seed=5)
    pos[1000:1300] = pos[1000]  # coincident centres
    o, acc = _compare_build(O.SPHERE, pos, None, rad)
    rays = S.pinhole_rays(128, 128, (0.5, 0.5, 2.2), (0.5, 0.5, 0.5), fov_deg=30)
    res = trace_both(acc, rays, want_normal=True)
    oh = o.trace(rays)
    assert_sphere_hits(res.hits, oh)
    hit = oh["prim"] != O.MISS
    sec = np.zeros(int(hit.sum()), O.RAY_DTYPE)
    p = rays["org"][hit] + res.hits["t"][hit, None] * rays["dir"][hit]
    nrm = res.normal[hit]
    sec["org"] = p.astype(np.float32)
    sec["dir"] = S.hemisphere_dirs(nrm, seed=7)
    sec["prev_prim"] = oh["prim"][hit]
    sec["prev_t"] = oh["t"][hit]
    assert_sphere_hits(trace_both(acc, sec, prev_normals=nrm),
                      o.trace(sec, prev_normals=nrm))


def test_sphere_pole_hits_take_the_reference_walk():
    """Closest hits within rounding of their leaf box's entry with a second
    hit inside the same rounding window: the reference's pruning decides,
    and the GPU's second pass reproduces its walk."""
    import ctypes as C

    import torch
    from surface_b200 import _lib
    from test_walk_restatement import pole_pairs
    pos, rad, rays = pole_pairs()
    o, acc = _compare_build(O.SPHERE, pos, None, rad)
    assert_sphere_hits(trace_both(acc, rays), o.trace(rays))
    st = torch.zeros(4, dtype=torch.int64, device="cuda")
    rt = torch.as_tensor(rays.view(np.float32).reshape(-1, 8)).cuda()
    h = torch.empty((rays.size, 4), device="cuda")
    opts = _lib.TraceOpts(None, None, None, None, None, st.data_ptr(), 0, 0)
    acc.ctx.use_torch_stream()
    _lib.check(acc.L.srt_trace_closest(acc.h, rt.data_ptr(), rays.size, h.data_ptr(),
                                       C.byref(opts)))
    torch.cuda.synchronize()
    assert int(st[3]) > 0  # rays retraced by the reference's walk


def test_constant_radius_spheres():
    pos, _ = S.particles(30_000, seed=8)
    o = O.OracleAccel(O.SPHERE, pos, None, None, const_radius=0.004)
    acc = sb.ParticleAccel()
    acc.Build32(sb.Particles(pos, None, 0.004))
    can, idx, _ = gpu_canonical(acc, O.SPHERE)
    assert np.array_equal(can, o.canonical())
    rays = S.pinhole_rays(64, 64, (0.5, 0.5, 2.2), (0.5, 0.5, 0.5), fov_deg=30)
    assert_sphere_hits(acc.Traverse(rays), o.trace(rays))


def test_dump_is_reference_format():
    v, f = S.displaced_octasphere(5, seed=3)
    o = O.OracleAccel(O.TRI, v, f)
    acc = gpu_build(O.TRI, v, f)
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "a.bin")
        acc.Dump(path)
        with open(path, "rb") as fp:
            g, idx = O.parse_dump(O.TRI, fp.read())
    assert np.array_equal(O.canonicalize(g, 0), o.canonical())
    assert np.array_equal(idx, o.indices)
    # sequential depth-first emission: the node array equals the oracle's
    assert np.array_equal(g["d0"], o.nodes["d0"]) and np.array_equal(g["d1"], o.nodes["d1"])


def test_rebuild_reuses_accel():
    acc = sb.TriangleAccel()
    for lv in (6, 4, 6):
        v, f = S.displaced_octasphere(lv, seed=lv)
        acc.Build32(sb.Mesh(v, f))
        o = O.OracleAccel(O.TRI, v, f)
        can, idx, _ = gpu_canonical(acc, O.TRI)
        assert np.array_equal(can, o.canonical())


def test_torch_device_inputs_and_async_trace():
    import torch
    v, f = S.displaced_octasphere(6, seed=21)
    rays = S.pinhole_rays(128, 96, (0, 0, 3), (0, 0, 0))
    o = O.OracleAccel(O.TRI, v, f)
    acc = sb.TriangleAccel()
    vt = torch.as_tensor(v).cuda()
    ft = torch.as_tensor(f.astype(np.int32)).cuda()
    acc.Build32(sb.Mesh(vt, ft))
    rt = torch.as_tensor(rays.view(np.float32).reshape(-1, 8)).cuda()
    h = acc.Traverse(rt)
    torch.cuda.synchronize()
    hn = h.cpu().numpy().view(O.HIT_DTYPE).reshape(-1)
    assert_hits_equal(hn, o.trace(rays))


def _pinned(a, dt=np.float32):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a).view(dt).copy()).pin_memory()


def test_host_arrays_match_device_path():
    """Pageable host arrays (staged copies) and page-locked host arrays (read
    and written by the kernels in place) give the device path's results bit
    for bit, with every optional input and output."""
    import ctypes as C

    import torch
    from surface_b200 import _lib

    def dev(a, dt=np.float32):
        return torch.as_tensor(np.ascontiguousarray(a).view(dt)).cuda()

    v, f, sc = S.tet_grid(24, seed=41)
    acc = sb.TetraAccel()
    acc.Build32(sb.Tetrahedron(v, f))
    rays = S.ortho_rays(560, 560)  # 313,600 rays
    n = rays.size
    vs = torch.as_tensor(sc).cuda()
    d = acc.Traverse(dev(rays).reshape(-1, 8), want_subface=True, vertex_scalar=vs,
                     want_scalar=True)
    dh = d.hits.cpu().numpy().reshape(-1).view(O.HIT_DTYPE)
    h = acc.Traverse(rays, want_subface=True, vertex_scalar=vs, want_scalar=True)
    assert_hits_equal(h.hits, dh)
    assert np.array_equal(h.subface.view(np.int32), d.subface.cpu().numpy())
    assert np.array_equal(bits(h.scalar), bits(d.scalar.cpu().numpy()))
    assert (h.hits["prim"] != O.MISS).mean() > 0.5
    pr, ph = _pinned(rays), torch.zeros((n, 4)).pin_memory()
    psub, psc = torch.zeros(n, dtype=torch.int32).pin_memory(), torch.zeros(n).pin_memory()
    o = _lib.TraceOpts(None, psub.data_ptr(), vs.data_ptr(), psc.data_ptr(), None, None, 0, 0)
    _lib.check(acc.L.srt_trace_closest(acc.h, pr.data_ptr(), n, ph.data_ptr(), C.byref(o)))
    assert_hits_equal(ph.numpy().reshape(-1).view(O.HIT_DTYPE), dh)
    assert np.array_equal(psub.numpy(), d.subface.cpu().numpy())
    assert np.array_equal(bits(psc.numpy()), bits(d.scalar.cpu().numpy()))

    pos, rad = S.particles(100_000, seed=42)
    sp = sb.ParticleAccel()
    sp.Build32(sb.Particles(pos, rad))
    prim = S.pinhole_rays(600, 500, (0.5, 0.5, 2.2), (0.5, 0.5, 0.5), fov_deg=30)
    r1 = sp.Traverse(prim, want_normal=True)
    sec = prim.copy()
    hit = r1.hits["prim"] != O.MISS
    sec["org"][hit] = (prim["org"][hit] + r1.hits["t"][hit, None] * prim["dir"][hit])
    sec["dir"][hit] = S.hemisphere_dirs(r1.normal[hit], seed=43)
    sec["prev_prim"] = r1.hits["prim"]
    sec["prev_t"] = r1.hits["t"]
    nrm = np.ascontiguousarray(r1.normal, np.float32)
    d = sp.Traverse(dev(sec).reshape(-1, 8), prev_normals=torch.as_tensor(nrm).cuda(),
                    want_normal=True)
    dh = d.hits.cpu().numpy().reshape(-1).view(O.HIT_DTYPE)
    h = sp.Traverse(sec, prev_normals=nrm, want_normal=True)
    assert_hits_equal(h.hits, dh)
    assert np.array_equal(bits(h.normal), bits(d.normal.cpu().numpy()))
    n = sec.size
    pr, ph, pn = _pinned(sec), torch.zeros((n, 4)).pin_memory(), _pinned(nrm)
    pno = torch.zeros((n, 3)).pin_memory()
    o = _lib.TraceOpts(pn.data_ptr(), None, None, None, pno.data_ptr(), None, 0, 0)
    _lib.check(sp.L.srt_trace_closest(sp.h, pr.data_ptr(), n, ph.data_ptr(), C.byref(o)))
    assert_hits_equal(ph.numpy().reshape(-1).view(O.HIT_DTYPE), dh)
    assert np.array_equal(bits(pno.numpy()), bits(d.normal.cpu().numpy()))


# ---------------------------------------------------------------- full size
def test_full_size_triangle_workload():
    """131,072-triangle displaced octasphere, 512^2 pinhole rays."""
    v, f = S.displaced_octasphere(7)
    o, acc = _compare_build(O.TRI, v, f)
    rays = S.pinhole_rays(512, 512, (0, 0, 3), (0, 0, 0))
    h = trace_both(acc, rays)
    oh = o.trace(rays)
    assert_hits_equal(h, oh)
    assert acc.info().num_branches == len([1 for x in o.nodes if not x["leaf"]])


def test_full_size_tetra_workload():
    """1,310,720 tetrahedra (64^3 cells), 1024^2 orthographic rays."""
    v, f, sc = S.tet_grid(64)
    o, acc = _compare_build(O.TET, v, f)
    rays = S.ortho_rays(1024, 1024)
    res = trace_both(acc, rays, want_subface=True)
    oh, osub = o.trace(rays, want_subface=True)
    ids = np.mean(res.hits["prim"] == oh["prim"])
    assert ids >= 0.9999
    assert_hits_equal(res.hits, oh)
    assert np.array_equal(res.subface, osub)


def test_full_size_particle_frame():
    """The particle configuration's frame 3 (16,777,216 spheres advected three
    times): the build, all 2048^2 primaries and the hemisphere secondary of
    every hit (self-hit rule) against the oracle."""
    import torch
    pos0, rad = S.particles()
    pos = S.particle_frames(pos0, 4, device="cuda")[3].cpu().numpy()
    del pos0
    o, acc = _compare_build(O.SPHERE, pos, None, rad)
    rays = S.pinhole_rays(2048, 2048, (0.5, 0.5, 2.2), (0.5, 0.5, 0.5), fov_deg=30)
    rt = torch.as_tensor(rays.view(np.float32).reshape(-1, 8)).cuda()
    res = acc.Traverse(rt, want_normal=True)
    hits = res.hits.cpu().numpy().reshape(-1).view(O.HIT_DTYPE)
    assert_sphere_hits(hits, o.trace(rays))
    sec, sn = sb.spawn_secondary(rt, res.hits, res.normal, seed=3)
    h2 = acc.Traverse(sec, prev_normals=sn)
    torch.cuda.synchronize()
    sr = sec.cpu().numpy().reshape(-1).view(O.RAY_DTYPE)
    assert sr.size == int((hits["prim"] != O.MISS).sum()) > 1_000_000
    want = o.trace(sr, prev_normals=sn.cpu().numpy())
    assert_sphere_hits(h2.cpu().numpy().reshape(-1).view(O.HIT_DTYPE), want)
    assert (want["prim"] != O.MISS).any()


# The oracle against the reference's own build and trace (oracle/_ref) at the
# three full configurations.  No GPU is used; they run with the GPU suite for
# the box's host cores (minutes of CPU time on a small host).
need_ref = pytest.mark.skipif(not O.have_ref(), reason="reference build absent")


@need_ref
def test_oracle_vs_reference_full_triangles():
    v, f = S.displaced_octasphere(7)
    o, r = O.OracleAccel(O.TRI, v, f), O.RefAccel(O.TRI, v, f)
    rc, ridx = r.canonical()
    assert np.array_equal(o.canonical(), rc) and np.array_equal(o.indices, ridx)
    rays = S.pinhole_rays(512, 512, (0, 0, 3), (0, 0, 0))
    assert_hits_equal(o.trace(rays), r.trace(rays))


@need_ref
def test_oracle_vs_reference_full_tetrahedra():
    v, f, _ = S.tet_grid(64)
    o, r = O.OracleAccel(O.TET, v, f), O.RefAccel(O.TET, v, f)
    rc, ridx = r.canonical()
    assert np.array_equal(o.canonical(), rc) and np.array_equal(o.indices, ridx)
    rays = S.ortho_rays(1024, 1024)
    (ho, so), (hr, sr) = o.trace(rays, want_subface=True), r.trace(rays)
    assert_hits_equal(ho, hr)
    assert np.array_equal(so, sr)


@need_ref
def test_oracle_vs_reference_full_particles():
    pos, rad = S.particles()
    o, r = O.OracleAccel(O.SPHERE, pos, None, rad), O.RefAccel(O.SPHERE, pos, None, rad)
    rc, ridx = r.canonical()
    assert np.array_equal(o.canonical(), rc) and np.array_equal(o.indices, ridx)
    rays = S.pinhole_rays(2048, 2048, (0.5, 0.5, 2.2), (0.5, 0.5, 0.5), fov_deg=30)
    assert_hits_equal(o.trace(rays), r.trace(rays))


# ---------------------------------------------------------------- exact ties
def test_duplicate_triangles_tie_break():
    """Every face twice: each hit is an exact tie; the reference keeps the
    last one of its depth-first order (t <= current)."""
    v, f = S.displaced_octasphere(5, seed=31)
    f2 = np.concatenate([f, f[::-1]])
    o, acc = _compare_build(O.TRI, v, f2)
    rays = S.pinhole_rays(96, 96, (0, 0, 3), (0, 0, 0))
    h = trace_both(acc, rays)
    oh = o.trace(rays)
    assert_hits_equal(h, oh)
    assert np.any(oh["prim"] != O.MISS)


def test_duplicate_spheres_tie_break():
    pos, rad = S.particles(20_000, seed=32)
    pos2 = np.concatenate([pos, pos[::-1]])
    rad2 = np.concatenate([rad, rad[::-1]])
    o, acc = _compare_build(O.SPHERE, pos2, None, rad2)
    rays = S.pinhole_rays(96, 96, (0.5, 0.5, 2.2), (0.5, 0.5, 0.5), fov_deg=30)
    assert_sphere_hits(trace_both(acc, rays), o.trace(rays))


def test_duplicate_tetrahedra_tie_break():
    v, f, _ = S.tet_grid(10, seed=33)
    f2 = np.concatenate([f, f[::-1]])
    o, acc = _compare_build(O.TET, v, f2)
    for rays in (S.ortho_rays(80, 80),
                 S.pinhole_rays(64, 64, (1.7, 1.3, 2.1), (0.5, 0.5, 0.5), fov_deg=50)):
        res = trace_both(acc, rays, want_subface=True)
        oh, osub = o.trace(rays, want_subface=True)
        assert_hits_equal(res.hits, oh)
        assert np.array_equal(res.subface, osub)


def test_rays_from_inside_the_mesh():
    """Origins inside the tetrahedral mesh and the sphere cloud: entering
    distances near zero and negative."""
    v, f, _ = S.tet_grid(12, seed=34)
    o, acc = _compare_build(O.TET, v, f)
    rng = np.random.default_rng(3)
    rays = np.zeros(4096, O.RAY_DTYPE)
    rays["org"] = rng.uniform(0.05, 0.95, size=(4096, 3)).astype(np.float32)
    d = rng.normal(size=(4096, 3))
    rays["dir"] = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    rays["prev_prim"] = O.MISS
    res = trace_both(acc, rays, want_subface=True)
    oh, osub = o.trace(rays, want_subface=True)
    assert_hits_equal(res.hits, oh)
    assert np.array_equal(res.subface, osub)
