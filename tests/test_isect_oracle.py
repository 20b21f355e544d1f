"""The oracle's BuildIntersection restatement (the shading record of a hit:
position, normal, tangent, binormal, f0..f3 and InterpolateTetra's d0..d3)
pinned against the reference: its stored outputs (tests/golden/isect_small.npz,
written by make_golden.py from the reference's own Traverse) and, when the
reference build is present, live runs on larger scenes."""
import numpy as np
import pytest

from oracle import oracle as O
from surface_b200 import scenes as S

from conftest import bits

FIELDS = ("position", "f0", "normal", "f1", "tangent", "f2", "binormal", "f3", "d")


def _same_records(a, b):
    for f in FIELDS:
        assert np.array_equal(bits(a[f]), bits(b[f])), f


def _same_hits(a, b):
    for f in ("t", "u", "v", "prim"):
        assert np.array_equal(bits(a[f]), bits(b[f])), f


@pytest.mark.parametrize("tag", ["tri", "tet", "sph"])
def test_isect_records_match_reference_fixture(golden, tag):
    g = golden("isect_small.npz")
    if tag == "tri":
        acc = O.OracleAccel(O.TRI, g["tri_verts"], g["tri_faces"])
    elif tag == "tet":
        acc = O.OracleAccel(O.TET, g["tet_verts"], g["tet_faces"])
    else:
        acc = O.OracleAccel(O.SPHERE, g["sph_pos"], None, g["sph_rad"])
    rays = g[f"{tag}_rays"]
    sub = None
    if tag == "tet":
        h, sub = acc.trace(rays, want_subface=True)
        assert np.array_equal(sub, g["tet_subface"])
    else:
        h = acc.trace(rays)
    _same_hits(h, g[f"{tag}_hits"])
    rec = acc.isect(rays, h, sub)
    _same_records(rec, g[f"{tag}_isect"])
    hit = h["prim"] != O.MISS
    assert hit.sum() > 100
    # a miss leaves an all-zero record
    assert not np.any(rec[~hit].view(np.uint8))
    if tag == "tet":
        # InterpolateTetra's weights are normalised to sum 1
        d = rec["d"][hit].astype(np.float64)
        assert np.allclose(d.sum(1), 1.0, atol=1e-5)


need_ref = pytest.mark.skipif(not O.have_ref(), reason="reference build absent")


@need_ref
def test_isect_oracle_vs_reference_live():
    v, f = S.displaced_octasphere(6, seed=21)
    rays = S.pinhole_rays(128, 128, (0.2, -0.4, 2.9), (0, 0, 0), fov_deg=45)
    hr, _, rr = O.RefAccel(O.TRI, v, f).trace_isect(rays)
    o = O.OracleAccel(O.TRI, v, f)
    ho = o.trace(rays)
    _same_hits(ho, hr)
    _same_records(o.isect(rays, ho), rr)

    vt, ft, _ = S.tet_grid(16, seed=23)
    rays = S.pinhole_rays(128, 128, (-0.9, 1.6, 2.4), (0.5, 0.5, 0.5), fov_deg=40)
    hr, sr, rr = O.RefAccel(O.TET, vt, ft).trace_isect(rays)
    o = O.OracleAccel(O.TET, vt, ft)
    ho, so = o.trace(rays, want_subface=True)
    _same_hits(ho, hr)
    assert np.array_equal(so, sr)
    _same_records(o.isect(rays, ho, so), rr)

    pos, rad = S.particles(30000, seed=25)
    rays = S.pinhole_rays(128, 128, (0.5, 0.5, 2.2), (0.5, 0.5, 0.5), fov_deg=30)
    hr, _, rr = O.RefAccel(O.SPHERE, pos, None, rad).trace_isect(rays)
    o = O.OracleAccel(O.SPHERE, pos, None, rad)
    ho = o.trace(rays)
    _same_hits(ho, hr)
    _same_records(o.isect(rays, ho), rr)
