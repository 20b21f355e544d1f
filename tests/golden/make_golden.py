"""Generates the golden fixtures in this directory from the reference itself.

    make -C oracle          # builds oracle/_ref/libsurface_ref.so from the reference tree
    python tests/golden/make_golden.py

Every array here is an output of the reference's own code (its render/ sources
linked by oracle/ref_harness.cc), on inputs drawn with the reference tests'
fixture generator (TinyMT64, seed 123456, test/cctest/test-prefix-tree.cc:10-23)
or with the seeded scene generators of surface_b200.scenes.  The tests check
the C restatement (oracle/) and the CUDA path against these files, so parity is
pinned even where the reference tree is absent.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from surface_b200 import scenes as S  # noqa: E402

PREFIX_NS = [8, 15, 31, 1023, 1000, 3211]  # test/cctest/test-prefix-tree.cc:500


def _ptr(a):
    return O._ptr(a)


def prefix_tree(L):
    """Morton codes (scalar and SSE paths) of the tests' point draws and the
    Karras arrays of the sorted codes, per size, drawn in the tests' order."""
    out = {}
    draws = O.tinymt64_doubles(3 * sum(PREFIX_NS), use_ref=True)
    off = 0
    lo = np.zeros(3, np.float32)
    hi = np.ones(3, np.float32)
    for n in PREFIX_NS:
        pts = draws[off:off + 3 * n].astype(np.float32).reshape(n, 3)
        off += 3 * n
        codes = np.zeros(n, np.uint32)
        codes_simd = np.zeros(n, np.uint32)
        L.ref_morton_points(_ptr(pts), n, _ptr(lo), _ptr(hi), _ptr(codes), 0)
        L.ref_morton_points(_ptr(pts), n, _ptr(lo), _ptr(hi), _ptr(codes_simd), 1)
        sc = np.sort(codes, kind="stable")
        child = np.zeros(n - 1, np.uint32)
        lt = np.zeros(n - 1, np.uint8)
        rt = np.zeros(n - 1, np.uint8)
        L.ref_karras(_ptr(sc), n, _ptr(child), _ptr(lt), _ptr(rt))
        out[f"pts_{n}"] = pts
        out[f"codes_{n}"] = codes
        out[f"codes_simd_{n}"] = codes_simd
        out[f"child_{n}"] = child.copy()
        out[f"ltype_{n}"] = lt.copy()
        out[f"rtype_{n}"] = rt.copy()
        # same-key variant (all points at 0.123458)
        same = np.full((n, 3), 0.123458, np.float32)
        cs = np.zeros(n, np.uint32)
        L.ref_morton_points(_ptr(same), n, _ptr(lo), _ptr(hi), _ptr(cs), 0)
        L.ref_karras(_ptr(cs), n, _ptr(child), _ptr(lt), _ptr(rt))
        out[f"same_codes_{n}"] = cs
        out[f"same_child_{n}"] = child.copy()
        out[f"same_ltype_{n}"] = lt.copy()
        out[f"same_rtype_{n}"] = rt.copy()
    # the radix sort of the largest case, from RadixSort30OMP itself
    n = 3211
    c = out[f"codes_{n}"].copy()
    i = np.arange(n, dtype=np.uint32)
    L.ref_radix_sort(_ptr(c), _ptr(i), n)
    out["sorted_codes_3211"] = c
    out["sorted_index_3211"] = i
    return out


def scene_fixtures():
    """Small scenes: canonical trees, sorted indices and closest hits from the
    reference's Build32 / Traverse."""
    out = {}
    # triangles: 2048-face displaced octasphere, 32x32 pinhole rays
    v, f = S.displaced_octasphere(4)
    R = O.RefAccel(O.TRI, v, f)
    can, idx = R.canonical()
    rays = S.pinhole_rays(32, 32, (0, 0, 3), (0, 0, 0))
    out.update(tri_verts=v, tri_faces=f, tri_canon=can, tri_index=idx, tri_rays=rays,
               tri_hits=R.trace(rays), tri_bbox=np.concatenate(R.bbox()))
    # tetrahedra: 8^3 grid (2560 tets), 32x32 orthographic rays
    vt, ft, sc = S.tet_grid(8)
    R = O.RefAccel(O.TET, vt, ft)
    can, idx = R.canonical()
    rays = S.ortho_rays(32, 32)
    hits, sub = R.trace(rays)
    out.update(tet_verts=vt, tet_faces=ft, tet_scalar=sc, tet_canon=can, tet_index=idx,
               tet_rays=rays, tet_hits=hits, tet_subface=sub,
               tet_bbox=np.concatenate(R.bbox()))
    # spheres: 4096 particles, 32x32 pinhole primaries + one secondary per hit
    pos, rad = S.particles(4096)
    R = O.RefAccel(O.SPHERE, pos, None, rad)
    can, idx = R.canonical()
    rays = S.pinhole_rays(32, 32, (0.5, 0.5, 2.2), (0.5, 0.5, 0.5), fov_deg=30)
    hits = R.trace(rays)
    hit = hits["prim"] != O.MISS
    p = rays["org"][hit] + hits["t"][hit, None] * rays["dir"][hit]
    nrm = p - pos[hits["prim"][hit]]
    nrm = (nrm / np.linalg.norm(nrm, axis=1, keepdims=True)).astype(np.float32)
    sec = np.zeros(int(hit.sum()), O.RAY_DTYPE)
    sec["org"] = p.astype(np.float32)
    sec["dir"] = S.hemisphere_dirs(nrm, seed=99)
    sec["prev_prim"] = hits["prim"][hit]
    sec["prev_t"] = hits["t"][hit]
    out.update(sph_pos=pos, sph_rad=rad, sph_canon=can, sph_index=idx, sph_rays=rays,
               sph_hits=hits, sph_sec_rays=sec, sph_sec_normals=nrm,
               sph_sec_hits=R.trace(sec, prev_normals=nrm),
               sph_bbox=np.concatenate(R.bbox()))
    return out


def isect_fixtures():
    """Every Intersection field the reference's Traverse fills (t/u/v/prim,
    subface_id and BuildIntersection's position, normal, tangent, binormal,
    f0..f3, d0..d3) for small scenes of the three kinds, with oblique rays."""
    out = {}
    v, f = S.displaced_octasphere(4, seed=7)
    rays = S.pinhole_rays(40, 40, (0.4, 0.3, 2.8), (0, 0, 0), fov_deg=50)
    h, _, rec = O.RefAccel(O.TRI, v, f).trace_isect(rays)
    out.update(tri_verts=v, tri_faces=f, tri_rays=rays, tri_hits=h, tri_isect=rec)
    vt, ft, _ = S.tet_grid(8, seed=11)
    rays = S.pinhole_rays(40, 40, (1.7, 1.3, 2.1), (0.5, 0.5, 0.5), fov_deg=50)
    h, sub, rec = O.RefAccel(O.TET, vt, ft).trace_isect(rays)
    out.update(tet_verts=vt, tet_faces=ft, tet_rays=rays, tet_hits=h, tet_subface=sub,
               tet_isect=rec)
    pos, rad = S.particles(4096, seed=13)
    rad = (rad * 30.0).astype(np.float32)  # most rays hit a sphere
    rays = S.pinhole_rays(40, 40, (0.5, 0.5, 2.2), (0.5, 0.5, 0.5), fov_deg=30)
    h, _, rec = O.RefAccel(O.SPHERE, pos, None, rad).trace_isect(rays)
    out.update(sph_pos=pos, sph_rad=rad, sph_rays=rays, sph_hits=h, sph_isect=rec)
    return out


def tex_fixture(L):
    rng = np.random.default_rng(5)
    w, h, d = 9, 7, 5
    img = rng.random((d, h, w), dtype=np.float32)
    uvw = rng.uniform(-0.5, 1.5, size=(300, 3)).astype(np.float32)
    out = {"tex_img": img, "tex_uvw": uvw}
    for mode in (0, 1):
        rgba = np.zeros((300, 4), np.float32)
        L.ref_tex3d(_ptr(img), w, h, d, 1, _ptr(uvw), 300, mode, mode, mode, _ptr(rgba))
        out[f"tex_out_clamp{mode}"] = rgba[:, 0].copy()
    return out


def dump_fixtures():
    """Files written by the reference's own XxxAccel::Dump() for small
    scenes of each kind, with the scenes: the accel loader must read them and
    the product's Dump() must write the same bytes."""
    import tempfile
    v, f = S.displaced_octasphere(4, seed=71)
    tv, tf, _ = S.tet_grid(6, seed=72)  # >= 1024 primitives: the LBVH path of Build32
    p, r = S.particles(3000, seed=73, median_radius=0.02)
    out = {"tri_verts": v, "tri_faces": f, "tet_verts": tv, "tet_faces": tf,
           "sph_pos": p, "sph_rad": r}
    for tag, acc in (("tri", O.RefAccel(O.TRI, v, f)), ("tet", O.RefAccel(O.TET, tv, tf)),
                     ("sph", O.RefAccel(O.SPHERE, p, None, r))):
        with tempfile.TemporaryDirectory() as td:
            path = os.path.join(td, "accel.bin")
            getattr(acc.L, f"ref_{acc.tag}_dump")(acc.h, path.encode())
            with open(path, "rb") as fp:
                out[f"{tag}_dump"] = np.frombuffer(fp.read(), np.uint8).copy()
    return out


def lines_solids_fixtures():
    """The reference's LineAccel and SolidAccel (Build32) on small scenes:
    their Dump() files and, per ray, the hit (t, u, v, prim) and normal (and
    for solids the position), plus a sparse volume's fetches with edge
    coordinates through the reference's SparseVolumeAccel."""
    out = {}
    pos, seg, rad = S.line_strands(300, 8, seed=81)
    lrays = S.pinhole_rays(48, 48, (0.2, 0.4, 3.1), (0, 0, 0), fov_deg=45)
    name, cp, cs, cr, cc, copts, crays = next(c for c in S.line_cases() if c[0] == "axes-cap1")
    out.update(line_pos=pos, line_seg=seg, line_rad=rad, line_rays=lrays,
               edge_pos=cp, edge_seg=cs, edge_rad=cr, edge_rays=crays)
    for tag, (p_, s_, r_, rays) in {"line": (pos, seg, rad, lrays),
                                   "edge": (cp, cs, cr, crays)}.items():
        acc = O.RefLines(p_, s_, r_)
        h, n = acc.trace(rays)
        out[f"{tag}_dump"] = np.frombuffer(acc.dump_bytes(), np.uint8).copy()
        out[f"{tag}_hits"] = h.view(np.float32).reshape(-1, 4).copy()
        out[f"{tag}_normals"] = n
    for nv, g in ((8, 11), (6, 8), (5, 6)):
        v, ix = S.solid_grid(nv, g, seed=83)
        rays = S.solid_rays(24, seed=nv)
        acc = O.RefSolids(nv, v, ix)
        h, n, q = acc.trace(rays)
        nodes, idx = acc.dump()
        out.update({f"solid{nv}_verts": v, f"solid{nv}_ix": ix, f"solid{nv}_rays": rays,
                    f"solid{nv}_nodes": nodes.view(np.uint8).copy(), f"solid{nv}_idx": idx,
                    f"solid{nv}_hits": h.view(np.float32).reshape(-1, 4).copy(),
                    f"solid{nv}_normals": n, f"solid{nv}_positions": q})
    blocks, pool, gdim = S.sparse_pages(ndiv=4, page=8, seed=5)
    uvw = S.sparse_edge_coords(blocks, gdim, 2000, 1)
    out.update(sp_blocks=blocks.view(np.uint8).copy(), sp_pool=np.frombuffer(pool, np.uint8).copy(),
               sp_gdim=np.array(gdim, np.int32), sp_uvw=uvw,
               sp_rgba=O.sparse_fetch(blocks, pool, 0, 1, gdim, uvw, use_ref=True))
    return out


def main():
    L = O.ref()
    if L is None:
        raise SystemExit("reference harness missing: run `make -C oracle` with the reference tree")
    only = sys.argv[1:]  # names of fixtures to write (default: all)
    jobs = {"prefix_tree": lambda: prefix_tree(L), "scenes_small": scene_fixtures,
            "texture3d": lambda: tex_fixture(L), "dumps_small": dump_fixtures,
            "lines_solids": lines_solids_fixtures, "isect_small": isect_fixtures}
    for name, make in jobs.items():
        if not only or name in only:
            np.savez_compressed(os.path.join(HERE, name + ".npz"), **make())
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))


if __name__ == "__main__":
    main()
