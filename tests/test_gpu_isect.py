"""Shading records on the GPU (srt_trace_opts.isect): every Intersection field
the reference's Traverse fills through BuildIntersection, checked against the
oracle's restatement (itself pinned to the reference by test_isect_oracle.py)
at the triangle and tetrahedron configurations' full sizes and on a sphere
cloud, through device, page-locked and pageable host arrays; and the C++
drop-ins of include/surface_rt_accel.hpp driven beside the reference's own
accels (oracle/_ref/libshim_check.so), comparing every Intersection field."""
import ctypes as C
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import surface_b200 as sb  # noqa: E402
from oracle import oracle as O  # noqa: E402
from surface_b200 import scenes as S  # noqa: E402

from conftest import ROOT, bits  # noqa: E402

pytestmark = pytest.mark.gpu

FIELDS = ("position", "f0", "normal", "f1", "tangent", "f2", "binormal", "f3", "d")
# Spheres' (u, v) come from double atan2 / acos: the C library's in the
# reference, CUDA's here; the float results agree to an ulp or two.
SPHERE_UV_TOL = 1e-6


def _check(kind, hits, sub, rec, rays, o):
    """GPU (hits, subface, records) against the oracle's trace + records."""
    if kind == O.TET:
        oh, osub = o.trace(rays, want_subface=True)
        assert np.array_equal(sub, osub)
    else:
        oh, osub = o.trace(rays), None
    for f in ("t", "prim") + (() if kind == O.SPHERE else ("u", "v")):
        bad = np.nonzero(bits(hits[f]) != bits(oh[f]))[0]
        assert bad.size == 0, (f, bad[:5])
    if kind == O.SPHERE:
        for f in ("u", "v"):
            d = np.abs(hits[f].astype(np.float64) - oh[f].astype(np.float64))
            assert d.max() <= SPHERE_UV_TOL, (f, d.max())
    orec = o.isect(rays, oh, osub)
    for f in FIELDS:
        a = bits(rec[f]).reshape(len(rec), -1)
        b = bits(orec[f]).reshape(len(rec), -1)
        bad = np.nonzero((a != b).any(1))[0]
        assert bad.size == 0, (f, bad.size, bad[:5])
    hit = oh["prim"] != O.MISS
    assert hit.sum() > len(rays) // 10
    assert not np.any(rec[~hit].view(np.uint8))
    return hit


def _gpu(kind, acc, rays_np, **kw):
    rt = torch.as_tensor(rays_np.view(np.float32).reshape(-1, 8), device="cuda")
    res = acc.Traverse(rt, want_isect=True, want_subface=(kind == O.TET), **kw)
    torch.cuda.synchronize()
    hits = res.hits.cpu().numpy().reshape(-1).view(O.HIT_DTYPE)
    rec = res.isect.cpu().numpy().reshape(-1).view(O.ISECT_DTYPE)
    sub = res.subface.cpu().numpy().view(np.uint32) if kind == O.TET else None
    return hits, sub, rec


def test_isect_triangles_full_config():
    """131,072-triangle octasphere, 512^2 pinhole rays: every record field."""
    v, f = S.displaced_octasphere(7)
    rays = S.pinhole_rays(512, 512, (0, 0, 3), (0, 0, 0))
    acc = sb.TriangleAccel()
    acc.Build32(sb.Mesh(torch.as_tensor(v, device="cuda"),
                        torch.as_tensor(f.astype(np.int32), device="cuda")))
    hits, sub, rec = _gpu(O.TRI, acc, rays)
    _check(O.TRI, hits, sub, rec, rays, O.OracleAccel(O.TRI, v, f))


def test_isect_tetrahedra_full_config():
    """1,310,720 tets, 1024^2 orthographic rays: entering-face normals and
    InterpolateTetra's weights bit for bit."""
    v, f, _ = S.tet_grid(64)
    rays = S.ortho_rays(1024, 1024)
    acc = sb.TetraAccel()
    acc.Build32(sb.Tetrahedron(torch.as_tensor(v, device="cuda"),
                               torch.as_tensor(f.astype(np.int32), device="cuda")))
    hits, sub, rec = _gpu(O.TET, acc, rays)
    hit = _check(O.TET, hits, sub, rec, rays, O.OracleAccel(O.TET, v, f))
    d = rec["d"][hit].astype(np.float64)
    assert np.allclose(d.sum(1), 1.0, atol=1e-5)


def test_isect_tetrahedra_oblique_rays():
    """Every entering face and Pluecker branch: oblique rays through a jittered grid."""
    v, f, _ = S.tet_grid(24, seed=5)
    rays = np.concatenate([
        S.pinhole_rays(256, 256, (1.7, 1.3, 2.1), (0.5, 0.5, 0.5), fov_deg=50),
        S.pinhole_rays(256, 256, (-0.7, -0.4, -1.2), (0.5, 0.5, 0.5), fov_deg=50),
        S.pinhole_rays(256, 256, (0.2, 2.2, 0.4), (0.5, 0.5, 0.5), fov_deg=50)])
    acc = sb.TetraAccel()
    acc.Build32(sb.Tetrahedron(v, f))
    hits, sub, rec = _gpu(O.TET, acc, rays)
    _check(O.TET, hits, sub, rec, rays, O.OracleAccel(O.TET, v, f))
    # the reference's Pluecker test reports faces 1, 2 and 3 as entering faces
    assert set(np.unique(sub[hits["prim"] != O.MISS])) == {1, 2, 3}


def test_isect_spheres_with_secondaries():
    pos, rad = S.particles(1_000_000, seed=17)
    rays = S.pinhole_rays(512, 512, (0.5, 0.5, 2.2), (0.5, 0.5, 0.5), fov_deg=30)
    acc = sb.ParticleAccel()
    acc.Build32(sb.Particles(pos, rad))
    o = O.OracleAccel(O.SPHERE, pos, None, rad)
    hits, sub, rec = _gpu(O.SPHERE, acc, rays)
    hit = _check(O.SPHERE, hits, sub, rec, rays, o)
    # secondaries with the self-hit rule (prev_prim / prev_t / prev normal)
    sec = np.zeros(int(hit.sum()), O.RAY_DTYPE)
    sec["org"] = rec["position"][hit]
    sec["dir"] = S.hemisphere_dirs(rec["normal"][hit], seed=5)
    sec["prev_prim"] = hits["prim"][hit]
    sec["prev_t"] = hits["t"][hit]
    pn = np.ascontiguousarray(rec["normal"][hit])
    res = acc.Traverse(sec, prev_normals=pn, want_isect=True)
    oh = o.trace(sec, prev_normals=pn)
    for f in ("t", "prim"):
        assert np.array_equal(bits(res.hits[f]), bits(oh[f])), f
    orec = o.isect(sec, oh)
    for f in FIELDS:
        assert np.array_equal(bits(res.isect[f]), bits(orec[f])), f


@pytest.mark.parametrize("how", ["pageable", "pinned"])
def test_isect_host_arrays(how):
    """Host rays and outputs: staged (pageable) and in place (page-locked)."""
    v, f, _ = S.tet_grid(16, seed=2)
    rays = S.pinhole_rays(200, 200, (-0.9, 1.6, 2.4), (0.5, 0.5, 0.5), fov_deg=40)
    acc = sb.TetraAccel()
    acc.Build32(sb.Tetrahedron(v, f))
    o = O.OracleAccel(O.TET, v, f)
    n = rays.size
    if how == "pageable":
        res = acc.Traverse(rays, want_isect=True, want_subface=True)
        hits, sub, rec = res.hits, res.subface, res.isect
    else:
        import surface_b200._lib as L_
        L = L_.load()
        pr = torch.from_numpy(rays.view(np.float32).reshape(-1, 8).copy()).pin_memory()
        ph = torch.empty((n, 4), dtype=torch.float32).pin_memory()
        pi = torch.empty((n, 20), dtype=torch.float32).pin_memory()
        opts = L_.TraceOpts(None, None, None, None, None, None, 0, 0, pi.data_ptr())
        L_.check(L.srt_trace_closest(acc.h, pr.data_ptr(), n, ph.data_ptr(), C.byref(opts)))
        hits = ph.numpy().reshape(-1).view(O.HIT_DTYPE)
        rec = pi.numpy().reshape(-1).view(O.ISECT_DTYPE)
        sub = o.trace(rays, want_subface=True)[1]
    _check(O.TET, hits, sub, rec, rays, o)


# ---------------------------------------------------------------- drop-in shim
SHIM = os.path.join(ROOT, "oracle", "_ref", "libshim_check.so")
REC = np.dtype([("hit", "<u4"), ("t", "<f4"), ("u", "<f4"), ("v", "<f4"), ("prim", "<u4"),
                ("subface", "<u4"), ("position", "<f4", 3), ("geometric", "<f4", 3),
                ("normal", "<f4", 3), ("tangent", "<f4", 3), ("binormal", "<f4", 3),
                ("f", "<u4", 8), ("d", "<f4", 8)])


def _shim():
    if not os.path.exists(SHIM):
        pytest.fail("oracle/_ref/libshim_check.so missing: build it with `make -C oracle` "
                    "where the reference tree is present")
    L = C.CDLL(SHIM)
    assert L.shim_record_bytes() == REC.itemsize
    P, Z = C.c_void_p, C.c_size_t
    L.shim_check_triangles.argtypes = [P, Z, P, Z, P, Z, C.c_int, P]
    L.shim_check_tetrahedra.argtypes = [P, P, Z, P, Z, C.c_int, P]
    L.shim_check_spheres.argtypes = [P, P, Z, P, P, Z, C.c_int, P]
    return L


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _run(L, tag, g, rays, mode, pn=None):
    out = np.zeros(rays.size, REC)
    if tag == "tri":
        v, f = g["tri_verts"], g["tri_faces"].astype(np.uint32)
        rc = L.shim_check_triangles(_ptr(v), v.shape[0], _ptr(f), f.shape[0], _ptr(rays),
                                    rays.size, mode, _ptr(out))
    elif tag == "tet":
        v, f = g["tet_verts"], g["tet_faces"].astype(np.uint32)
        rc = L.shim_check_tetrahedra(_ptr(v), _ptr(f), f.shape[0], _ptr(rays), rays.size,
                                     mode, _ptr(out))
    else:
        p, r = g["sph_pos"], g["sph_rad"]
        rc = L.shim_check_spheres(_ptr(p), _ptr(r), p.shape[0], _ptr(rays), _ptr(pn),
                                  rays.size, mode, _ptr(out))
    assert rc == 0
    return out


@pytest.mark.parametrize("tag", ["tri", "tet", "sph"])
def test_dropin_accels_fill_every_intersection_field(golden, tag):
    """GpuXxxAccel::Traverse (per ray) and ::TraverseBatch against the
    reference's XxxAccel::Traverse on the same primitives and rays: every
    field of Intersection, the untouched ones included, starts from the same
    bytes and must end equal."""
    L = _shim()
    g = golden("isect_small.npz")
    rays = np.ascontiguousarray(g[f"{tag}_rays"])
    ref = _run(L, tag, g, rays, 0)
    assert ref["hit"].sum() > 100
    for mode, sel in ((1, slice(0, 400)), (2, slice(None))):
        r = np.ascontiguousarray(rays[sel])
        got = _run(L, tag, g, r, mode)
        want = ref[sel]
        for f in REC.names:
            if tag == "sph" and f in ("u", "v"):
                d = np.abs(got[f].astype(np.float64) - want[f].astype(np.float64))
                assert d.max() <= SPHERE_UV_TOL, (mode, f, d.max())
                continue
            a = bits(got[f]).reshape(len(got), -1)
            b = bits(want[f]).reshape(len(want), -1)
            bad = np.nonzero((a != b).any(1))[0]
            assert bad.size == 0, (mode, f, bad[:5])
