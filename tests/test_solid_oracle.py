"""SolidAccel (render/render_accel_solid.cc): the oracle's restatement of
Build32 and Traverse against the reference's own code, bit for bit -- the
tree (compared in pre-order: the reference emits nodes from OpenMP tasks),
the solid order, and per ray the hit (t, solid), its position and normal --
for pyramids, prisms and hexahedra filling a jittered grid, with
grid-aligned rays, pinhole rays, rays starting inside the mesh and secondary
rays that skip the solid they leave (Ray::prev_prim_id)."""
import numpy as np
import pytest

from oracle import oracle as O
from surface_b200 import scenes as S

from conftest import bits

needs_ref = pytest.mark.skipif(not O.have_ref(), reason="reference harness not built")

# at least 1024 solids: below that the reference's Build32 falls back to its SAH Build
CASES = {"hexahedra": (8, 11), "prisms": (6, 8), "pyramids": (5, 6)}


def secondary(rays, hits, pos, seed):
    """Rays from each hit position in a random direction, skipping the hit solid."""
    ok = hits["prim"] != O.MISS
    rng = np.random.default_rng(seed)
    d = rng.normal(size=(ok.sum(), 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = S.make_rays(pos[ok], d)
    r["prev_prim"] = hits["prim"][ok]
    return r


@needs_ref
@pytest.mark.parametrize("case", list(CASES))
def test_solids_match_reference(case):
    nv, g = CASES[case]
    v, ix = S.solid_grid(nv, g, seed=7)
    o = O.OracleSolids(nv, v, ix)
    r = O.RefSolids(nv, v, ix)
    on, oi = o.export()
    rn, ri = r.dump()
    assert O.tree_canonical(on) == O.tree_canonical(rn)
    assert np.array_equal(oi, ri)
    lo, hi = r.bbox()
    assert np.array_equal(lo, on[0]["bmin"].astype(np.float64))
    assert np.array_equal(hi, on[0]["bmax"].astype(np.float64))
    rays = S.solid_rays(80, seed=nv)
    oh, onr, op = o.trace(rays)
    rh, rnr, rp = r.trace(rays)
    assert np.array_equal(bits(oh.view(np.float32).reshape(-1, 4)),
                          bits(rh.view(np.float32).reshape(-1, 4)))
    assert np.array_equal(bits(onr), bits(rnr)) and np.array_equal(bits(op), bits(rp))
    assert 0.5 < (rh["prim"] != O.MISS).mean() < 0.95
    rays2 = secondary(rays, rh, rp, nv)
    oh2, _, _ = o.trace(rays2)
    rh2, _, _ = r.trace(rays2)
    assert np.array_equal(bits(oh2.view(np.float32).reshape(-1, 4)),
                          bits(rh2.view(np.float32).reshape(-1, 4)))
    assert (rh2["prim"] != rays2["prev_prim"]).all()


def _raw(nodes):
    """Node bytes with the leaves' axis cleared (the reference leaves it unset)."""
    x = nodes.copy()
    x["axis"][x["flag"] == 1] = 0
    return x.tobytes()


def _sah_cases():
    out = []
    for nv, g in ((8, 9), (6, 7), (5, 5)):
        v, ix = S.solid_grid(nv, g, seed=3)
        for m in (2, 3, 4, 5, 17, 100, 500, ix.shape[0]):
            if m < 1024:
                out.append((f"nv{nv}-{m}", nv, v, ix[:m]))
    v, ix = S.solid_grid(8, 6, seed=5)
    out.append(("duplicates", 8, v, np.concatenate([ix[:50]] * 4)))
    flat = v.copy()
    flat[:, 2] = 0.5
    out.append(("flat", 8, flat, ix[:300]))
    return out


@needs_ref
@pytest.mark.parametrize("name,nv,v,ix", _sah_cases(), ids=[c[0] for c in _sah_cases()])
def test_sah_build_below_1024_matches_reference(name, nv, v, ix):
    """Below 1024 solids Build32 runs SolidAccel::Build (binned SAH,
    render/render_accel_solid.cc:1612-1793): the oracle's tree (node for
    node, in the reference's order), solid order and hits equal the
    reference's."""
    o = O.OracleSolids(nv, v, ix)
    r = O.RefSolids(nv, v, ix)
    on, oi = o.export()
    rn, ri = r.dump()
    assert _raw(on) == _raw(rn)
    assert np.array_equal(oi, ri)
    rays = S.solid_rays(48, seed=nv)
    oh, onr, op = o.trace(rays)
    rh, rnr, rp = r.trace(rays)
    assert np.array_equal(bits(oh.view(np.float32).reshape(-1, 4)),
                          bits(rh.view(np.float32).reshape(-1, 4)))
    assert np.array_equal(bits(onr), bits(rnr)) and np.array_equal(bits(op), bits(rp))
    rays2 = secondary(rays, rh, rp, nv)
    if rays2.size:
        oh2, _, _ = o.trace(rays2)
        rh2, _, _ = r.trace(rays2)
        assert np.array_equal(bits(oh2.view(np.float32).reshape(-1, 4)),
                              bits(rh2.view(np.float32).reshape(-1, 4)))


def _double_grid(nv, g, seed, shift=0.0):
    """A solid grid with double-precision positions that float does not
    hold: the float grid's vertices plus a seeded sub-ulp jitter, shifted."""
    v, ix = S.solid_grid(nv, g, seed=seed)
    rng = np.random.default_rng(seed + 100)
    v64 = v.astype(np.float64) + shift + rng.uniform(-1e-9, 1e-9, size=v.shape)
    return v64, ix


@needs_ref
@pytest.mark.parametrize("nv,g,m,shift", [(8, 11, None, 0.0), (6, 8, None, 100.0),
                                          (5, 6, None, 0.0), (8, 9, 400, 0.0),
                                          (6, 7, 600, 37.5)])
def test_double_positions_match_reference(nv, g, m, shift):
    """isDoublePrecisionPos: the oracle's Build32 (and SAH Build below 1024
    solids) and Traverse over double positions equal the reference's, node
    for node and hit for hit."""
    v64, ix = _double_grid(nv, g, seed=nv, shift=shift)
    if m is not None:
        ix = ix[:m]
    o = O.OracleSolids(nv, v64, ix)
    r = O.RefSolids(nv, v64, ix)
    assert o.verts.dtype == np.float64 and r.verts.dtype == np.float64
    on, oi = o.export()
    rn, ri = r.dump()
    if ix.shape[0] < 1024:
        assert _raw(on) == _raw(rn)
    else:
        assert O.tree_canonical(on) == O.tree_canonical(rn)
    assert np.array_equal(oi, ri)
    rays = S.solid_rays(48, seed=nv)
    rays["org"] += np.float32(shift)
    oh, onr, op = o.trace(rays)
    rh, rnr, rp = r.trace(rays)
    assert np.array_equal(bits(oh.view(np.float32).reshape(-1, 4)),
                          bits(rh.view(np.float32).reshape(-1, 4)))
    assert np.array_equal(bits(onr), bits(rnr)) and np.array_equal(bits(op), bits(rp))
    assert (rh["prim"] != O.MISS).mean() > 0.3
    # the double positions matter: the float build differs somewhere
    f = O.OracleSolids(nv, v64.astype(np.float32), ix)
    fh, _, fp = f.trace(rays)
    assert not (np.array_equal(fh.view(np.uint32), oh.view(np.uint32))
                and np.array_equal(fp.view(np.uint32), op.view(np.uint32)))


@needs_ref
@pytest.mark.parametrize("nv,g,dbl", [(8, 14, False), (6, 11, False), (5, 8, True)])
def test_sah_build_at_every_size_matches_reference(nv, g, dbl):
    """SolidAccel::Build, which the reference's GLES accel builder runs at
    every size (gles/gles_accel_builder.cc:967): the oracle's SAH tree over
    1024 solids or more equals the reference's node for node, float and
    double positions."""
    if dbl:
        v, ix = _double_grid(nv, g, seed=nv)
    else:
        v, ix = S.solid_grid(nv, g, seed=nv)
    o = O.OracleSolids(nv, v, ix, sah=True)
    r = O.RefSolids(nv, v, ix, sah=True)
    on, oi = o.export()
    rn, ri = r.dump()
    assert len(on) < 2 * ix.shape[0] and _raw(on) == _raw(rn)
    assert np.array_equal(oi, ri)
    rays = S.solid_rays(48, seed=nv)
    oh, _, op = o.trace(rays)
    rh, _, rp = r.trace(rays)
    assert np.array_equal(bits(oh.view(np.float32).reshape(-1, 4)),
                          bits(rh.view(np.float32).reshape(-1, 4)))
    assert np.array_equal(bits(op), bits(rp))
