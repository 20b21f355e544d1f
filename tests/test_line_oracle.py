"""LineAccel (render/render_accel_line.cc): the oracle's restatement against
the reference's own Build / Traverse / Dump / BoundingBox, bit for bit --
tree nodes, line order, hits (t, u, v, line) and BuildIntersection's normals
-- on hair-like strands, random segments and the edge cases of
scenes.line_cases (axis-parallel rays, rays along a line's axis through its
caps, zero-length lines, trees whose root is a leaf, a deep chain, leaf and
depth limits, caps off)."""
import numpy as np
import pytest

from oracle import oracle as O
from surface_b200 import scenes as S

from conftest import bits

needs_ref = pytest.mark.skipif(not O.have_ref(), reason="reference harness not built")

def _compare(pos, seg, rad, constr, opts, rays):
    o = O.OracleLines(pos, seg, rad, constr, **opts)
    r = O.RefLines(pos, seg, rad, constr, **opts)
    on, oi = o.export()
    rn, ri = r.dump()
    assert np.array_equal(O.line_nodes_masked(on).tobytes(), O.line_nodes_masked(rn).tobytes())
    assert np.array_equal(oi, ri)
    lo, hi = r.bbox()
    assert np.array_equal(lo, on[0]["bmin"].astype(np.float64))
    assert np.array_equal(hi, on[0]["bmax"].astype(np.float64))
    oh, onr = o.trace(rays)
    rh, rnr = r.trace(rays)
    assert np.array_equal(bits(oh.view(np.float32).reshape(-1, 4)),
                          bits(rh.view(np.float32).reshape(-1, 4)))
    assert np.array_equal(bits(np.nan_to_num(onr)), bits(np.nan_to_num(rnr)))
    assert np.array_equal(np.isnan(onr), np.isnan(rnr))
    return rh, o


@needs_ref
@pytest.mark.parametrize("cap", [True, False])
def test_strands_match_reference(cap):
    pos, seg, rad = S.line_strands(1500, 12, seed=3)
    rays = S.pinhole_rays(160, 160, (0.2, 0.4, 3.1), (0, 0, 0), fov_deg=45)
    h, _ = _compare(pos, seg, rad, 0.0, dict(cap=cap), rays)
    assert 0.2 < (h["prim"] != O.MISS).mean() < 0.95


@needs_ref
def test_segments_match_reference():
    pos, seg, rad = S.line_segments(12000, seed=9)
    rays = S.pinhole_rays(128, 128, (0.4, 0.2, 2.8), (0, 0, 0), fov_deg=50)
    h, o = _compare(pos, seg, rad, 0.0, {}, rays)
    assert (h["prim"] != O.MISS).mean() > 0.5
    assert o.depth() > 10


@needs_ref
@pytest.mark.parametrize("case", [c[0] for c in S.line_cases()])
def test_line_edge_cases_match_reference(case):
    name, pos, seg, rad, constr, opts, rays = next(c for c in S.line_cases() if c[0] == case)
    h, o = _compare(pos, seg, rad, constr, opts, rays)
    assert (h["prim"] != O.MISS).any()
    if name == "chain":
        assert o.depth() > 62  # deeper than the short traversal stack
