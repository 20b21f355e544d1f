"""Accels across frames and runs on the GPU: loading Dump() files
(srt_accel_load_*) and AccelBuilder's cache (srt_cache_*).

* dump -> load -> dump gives the same bytes, and the loaded accel traces
  bit-identically to the built one, for every kind;
* the reference's own Dump() files (tests/golden/dumps_small.npz) load into
  accels with the reference's tree and sorted order, the hits of the oracle
  and the Dump() bytes of a build;
* damaged files are refused before anything reaches the GPU;
* the cache finds static entries again, rebuilds dynamic ones, frees them at
  the end of the frame and on Invalidate, and counts bytes and hits."""
import os
import tempfile

import numpy as np
import pytest
import torch

import surface_b200 as sb
from oracle import oracle as O
from surface_b200 import scenes as S
from surface_b200.cache import AccelBuilder

from conftest import bits

pytestmark = pytest.mark.gpu


def _scene(kind, g=None):
    if kind == "tri":
        v, f = (g["tri_verts"], g["tri_faces"]) if g is not None else S.displaced_octasphere(5, 9)
        return sb.TriangleAccel, sb.Mesh(v, f), O.OracleAccel(O.TRI, v, f)
    if kind == "tet":
        v, f = (g["tet_verts"], g["tet_faces"]) if g is not None else S.tet_grid(12, 9)[:2]
        return sb.TetraAccel, sb.Tetrahedron(v, f), O.OracleAccel(O.TET, v, f)
    p, r = (g["sph_pos"], g["sph_rad"]) if g is not None else S.particles(20000, 9, 0.01)
    return sb.ParticleAccel, sb.Particles(p, r), O.OracleAccel(O.SPHERE, p, None, r)


def _build(cls, data):
    a = cls()
    a.Build32(data)
    return a


def _rays(kind, n=64):
    if kind == "tri":
        return S.pinhole_rays(n, n, (0, 0, 3), (0, 0, 0))
    if kind == "tet":
        return S.pinhole_rays(n, n, (1.7, 1.3, 2.1), (0.5, 0.5, 0.5), fov_deg=50)
    return S.pinhole_rays(n, n, (0.5, 0.5, 2.2), (0.5, 0.5, 0.5), fov_deg=30)


def _dump_bytes(acc):
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "a.bin")
        acc.Dump(path)
        with open(path, "rb") as fp:
            return fp.read()


def _hits(acc, rays):
    h = acc.Traverse(rays)
    return (h.hits if hasattr(h, "hits") else h).view(np.uint32)


@pytest.mark.parametrize("kind", ["tri", "tet", "sph"])
def test_dump_load_roundtrip(kind, tmp_path):
    cls, data, _ = _scene(kind)
    a = _build(cls, data)
    path = tmp_path / "accel.bin"
    a.Dump(path)
    b = cls()
    b.Load(path, data)
    assert _dump_bytes(b) == path.read_bytes()
    ia, ib = a.info(), b.info()
    for f in ("num_prims", "num_nodes", "num_branches", "num_leaves", "eps_scale"):
        assert getattr(ia, f) == getattr(ib, f)
    assert np.array_equal(bits(np.array(ia.scene_min[:] + ia.scene_max[:], np.float32)),
                          bits(np.array(ib.scene_min[:] + ib.scene_max[:], np.float32)))
    _, ia_idx, ia_codes = a.export()
    _, ib_idx, ib_codes = b.export()
    assert np.array_equal(ia_idx, ib_idx) and np.array_equal(ia_codes, ib_codes)
    rays = _rays(kind)
    assert np.array_equal(_hits(a, rays), _hits(b, rays))


@pytest.mark.parametrize("kind", ["tri", "tet", "sph"])
def test_load_reference_dump(kind, golden, tmp_path):
    g = golden("dumps_small.npz")
    cls, data, oracle = _scene(kind, g)
    path = tmp_path / "ref.bin"
    path.write_bytes(g[f"{kind}_dump"].tobytes())
    b = cls()
    b.Load(path, data)
    # the reference emits its nodes from OpenMP tasks, so its record order
    # varies from run to run; tree, boxes and sorted order do not
    okind = {"tri": O.TRI, "tet": O.TET, "sph": O.SPHERE}[kind]
    ref_nodes, ref_idx = O.parse_dump(okind, path.read_bytes())
    got_nodes, got_idx = O.parse_dump(okind, _dump_bytes(b))
    assert np.array_equal(O.canonicalize(got_nodes, 0), O.canonicalize(ref_nodes, 0))
    assert np.array_equal(got_idx, ref_idx)
    rays = _rays(kind, 48)
    want = oracle.trace(rays)
    want = want[0] if isinstance(want, tuple) else want
    assert np.array_equal(_hits(b, rays), want.view(np.uint32))
    # and it is the accel a build makes
    assert _dump_bytes(_build(cls, data)) == _dump_bytes(b)


def test_damaged_dumps_are_refused(golden, tmp_path):
    g = golden("dumps_small.npz")
    cls, data, _ = _scene("tri", g)
    raw = bytearray(g["tri_dump"].tobytes())
    nn = int(np.frombuffer(raw[:8], np.uint64)[0])
    cases = {
        "truncated": raw[:-4],
        "wrong kind": g["tet_dump"].tobytes(),
    }
    bad_child = bytearray(raw)
    bad_child[8 + 56:8 + 60] = np.uint32(nn + 5).tobytes()  # root's left child
    cases["child index"] = bad_child
    bad_perm = bytearray(raw)
    off = 8 + nn * 64 + 8
    bad_perm[off:off + 4] = bad_perm[off + 4:off + 8]  # duplicate sorted index
    cases["order"] = bad_perm
    bad_axis = bytearray(raw)
    bad_axis[8 + 52:8 + 56] = np.int32(3).tobytes()
    cases["axis"] = bad_axis
    for name, blob in cases.items():
        p = tmp_path / f"{name.replace(' ', '_')}.bin"
        p.write_bytes(bytes(blob))
        with pytest.raises(sb.SurfaceError):
            cls().Load(p, data)
    # another scene's file
    with pytest.raises(sb.SurfaceError):
        v, f = S.displaced_octasphere(5, 2)
        p = tmp_path / "good.bin"
        p.write_bytes(bytes(raw))
        sb.TriangleAccel().Load(p, sb.Mesh(v, f))


def test_cache_static_dynamic_invalidate():
    v, f = S.displaced_octasphere(5, 4)
    p, r = S.particles(20000, 5, 0.01)
    mesh = sb.Mesh(v, f)
    cache = AccelBuilder()
    a1 = cache.BuildTriangleAccel(mesh, elembuf=1, arraybuf=2, count=f.size)
    a2 = cache.BuildTriangleAccel(mesh, elembuf=1, arraybuf=2, count=f.size)
    info = cache.info()
    assert a1.h.value == a2.h.value and info.builds == 1 and info.hits == 1
    assert info.static_entries == 1 and info.bytes_used > 0
    # another key (offset) is another entry; the same key of another kind too
    cache.BuildTriangleAccel(mesh, elembuf=1, arraybuf=2, count=f.size, offset=3)
    sp = cache.BuildParticleAccel(sb.Particles(p, r), elembuf=1, arraybuf=2, count=f.size)
    assert cache.info().static_entries == 3
    # dynamic entries are rebuilt every time and freed at the end of the frame
    d1 = cache.BuildParticleAccel(sb.Particles(p, r), elembuf=7, arraybuf=8,
                                  count=p.shape[0], static=False)
    d2 = cache.BuildParticleAccel(sb.Particles(p, r), elembuf=7, arraybuf=8,
                                  count=p.shape[0], static=False)
    assert cache.info().dynamic_entries == 2 and d1.h.value != d2.h.value
    rays = _rays("sph")
    assert np.array_equal(_hits(d1, rays), _hits(sp, rays))
    used = cache.info().bytes_used
    cache.EndFrame()
    info = cache.info()
    assert info.dynamic_entries == 0 and info.bytes_used < used
    # cached accels trace like a direct build
    rays = _rays("tri")
    want = _hits(_build(sb.TriangleAccel, mesh), rays)
    assert np.array_equal(_hits(a1, rays), want)
    # Invalidate drops every entry built from the buffer (a1 is freed)
    cache.Invalidate(2)
    info = cache.info()
    assert info.static_entries == 0 and info.bytes_used == 0
    a3 = cache.BuildTriangleAccel(mesh, elembuf=1, arraybuf=2, count=f.size)
    assert cache.info().builds == 6 and np.array_equal(_hits(a3, rays), want)
    # device inputs are borrowed by the cached accel
    vt = torch.from_numpy(v).cuda()
    ft = torch.from_numpy(f.view(np.int32)).cuda()
    a4 = cache.BuildTriangleAccel(sb.Mesh(vt, ft), elembuf=11, arraybuf=12, count=f.size)
    del vt, ft
    torch.cuda.synchronize()
    assert np.array_equal(_hits(a4, rays), _hits(a3, rays))
    cache.close()


def test_cache_lines_and_solids():
    """AccelBuilder::BuildLineAccel / BuildSolidAccel: the same cache rules
    for the line and solid accels (a static hit returns the same accel, a
    different kind with the same key is another entry, EndFrame frees the
    dynamic ones, Invalidate the buffer's), and cached accels trace like
    direct builds."""
    from surface_b200.lines import LineAccel, Lines
    from surface_b200.solids import Solid, SolidAccel
    pos, seg, rad = S.line_strands(2000, 8, seed=2)
    v, ix = S.solid_grid(8, 11, seed=2)
    cache = AccelBuilder()
    l1 = cache.BuildLineAccel(Lines(pos, seg, rad), elembuf=1, arraybuf=2, count=seg.size)
    l2 = cache.BuildLineAccel(Lines(pos, seg, rad), elembuf=1, arraybuf=2, count=seg.size)
    s1 = cache.BuildSolidAccel(Solid(8, v, ix), elembuf=1, arraybuf=2, count=seg.size)
    info = cache.info()
    assert l1.h.value == l2.h.value and s1.h.value != l1.h.value
    assert info.builds == 2 and info.hits == 1 and info.static_entries == 2
    d = cache.BuildSolidAccel(Solid(8, v, ix), elembuf=5, arraybuf=6, count=ix.size,
                              static=False)
    assert cache.info().dynamic_entries == 1
    rays = S.pinhole_rays(96, 96, (0.2, 0.4, 3.1), (0, 0, 0))
    direct = LineAccel()
    direct.Build(Lines(pos, seg, rad))
    assert np.array_equal(bits(l1.Traverse(rays).view(np.float32).reshape(-1, 4)),
                          bits(direct.Traverse(rays).view(np.float32).reshape(-1, 4)))
    srays = S.solid_rays(48)
    ds = SolidAccel()
    ds.Build(Solid(8, v, ix))  # BuildSolidAccel runs SolidAccel::Build at every size
    assert s1.export()[0].tobytes() == O.OracleSolids(8, v, ix, sah=True).export()[0].tobytes()
    want = bits(ds.Traverse(srays).view(np.float32).reshape(-1, 4))
    assert np.array_equal(bits(s1.Traverse(srays).view(np.float32).reshape(-1, 4)), want)
    assert np.array_equal(bits(d.Traverse(srays).view(np.float32).reshape(-1, 4)), want)
    used = cache.info().bytes_used
    cache.EndFrame()
    assert cache.info().dynamic_entries == 0 and cache.info().bytes_used < used
    cache.Invalidate(2)
    assert cache.info().static_entries == 0 and cache.info().bytes_used == 0
    cache.close()
