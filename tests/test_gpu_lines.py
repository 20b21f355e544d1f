"""The line accel on the GPU (srt_line_*) against the oracle's LineAccel,
bit for bit: the tree and line order, hits (t, u, v, line) and normals --
strands, random segments and the edge cases of scenes.line_cases (among
them a chain deeper than the short traversal stack); host and device
inputs; Dump() bytes and BoundingBox."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from surface_b200 import scenes as S
from surface_b200.lines import LineAccel, LineBuildOptions, Lines

from conftest import bits

pytestmark = pytest.mark.gpu


def _opts(d):
    return LineBuildOptions(minLeafPrimitives=d.get("min_leaf", 4),
                            maxTreeDepth=d.get("max_depth", 512), cap=d.get("cap", True))


def _check(pos, seg, rad, constr, opts, rays, device_inputs=False):
    o = O.OracleLines(pos, seg, rad, constr, **opts)
    acc = LineAccel()
    if device_inputs:
        lines = Lines(torch.as_tensor(pos).cuda(), torch.as_tensor(seg.astype(np.int32)).cuda(),
                      None if rad is None else torch.as_tensor(rad).cuda(), constr)
    else:
        lines = Lines(pos, seg, rad, constr)
    acc.Build(lines, _opts(opts))
    gn, gi = acc.export()
    on, oi = o.export()
    assert np.array_equal(O.line_nodes_masked(on).tobytes(), O.line_nodes_masked(gn).tobytes())
    assert np.array_equal(gi, oi)
    assert acc.info()[2] == o.depth()
    want, wn = o.trace(rays)
    got, gnrm = acc.Traverse(rays, want_normal=True)
    assert np.array_equal(bits(got.view(np.float32).reshape(-1, 4)),
                          bits(want.view(np.float32).reshape(-1, 4)))
    assert np.array_equal(np.isnan(gnrm), np.isnan(wn))
    assert np.array_equal(bits(np.nan_to_num(gnrm)), bits(np.nan_to_num(wn)))
    # device rays give the same hits
    rt = torch.from_numpy(np.ascontiguousarray(rays).view(np.float32).reshape(-1, 8)).cuda()
    gd = acc.Traverse(rt).cpu().numpy()
    assert np.array_equal(bits(gd), bits(want.view(np.float32).reshape(-1, 4)))
    return acc, want


@pytest.mark.parametrize("cap", [True, False])
def test_strands(cap):
    pos, seg, rad = S.line_strands(20000, 16, seed=4)
    rays = S.pinhole_rays(384, 384, (0.2, 0.4, 3.1), (0, 0, 0), fov_deg=45)
    _, h = _check(pos, seg, rad, 0.0, dict(cap=cap), rays, device_inputs=cap)
    assert 0.2 < (h["prim"] != O.MISS).mean() < 0.995


def test_segments():
    pos, seg, rad = S.line_segments(50000, seed=9)
    rays = S.pinhole_rays(256, 256, (0.4, 0.2, 2.8), (0, 0, 0), fov_deg=50)
    _check(pos, seg, rad, 0.0, {}, rays)


@pytest.mark.parametrize("case", [c[0] for c in S.line_cases()])
def test_edge_cases(case):
    name, pos, seg, rad, constr, opts, rays = next(c for c in S.line_cases() if c[0] == case)
    _check(pos, seg, rad, constr, opts, rays, device_inputs=(name == "chain"))


def test_dump_and_bbox(tmp_path):
    pos, seg, rad = S.line_strands(3000, 8, seed=6)
    acc = LineAccel()
    acc.Build(Lines(pos, seg, rad))
    acc.Dump(tmp_path / "lines.bin")
    nodes, idx = O.parse_line_dump((tmp_path / "lines.bin").read_bytes())
    o = O.OracleLines(pos, seg, rad)
    on, oi = o.export()
    assert np.array_equal(O.line_nodes_masked(nodes).tobytes(), O.line_nodes_masked(on).tobytes())
    assert np.array_equal(idx, oi)
    lo, hi = acc.BoundingBox()
    assert np.array_equal(lo, on[0]["bmin"].astype(np.float64))
    assert np.array_equal(hi, on[0]["bmax"].astype(np.float64))
    import surface_b200 as sb
    bad = seg.copy()
    bad[5, 1] = pos.shape[0]  # a vertex past the end
    with pytest.raises(sb.SurfaceError):
        LineAccel().Build(Lines(pos, bad, rad))


def test_bad_inputs_rejected():
    """A NaN position and a segment naming a vertex beyond nverts end the
    GPU build with SRT_ERR_INVALID (the build kernel flags them and reads
    no vertex out of range); the accel then builds and traces normally."""
    from surface_b200 import SurfaceError
    pos, seg, rad = S.line_strands(300, 4, seed=2)
    acc = LineAccel()
    bad = pos.copy()
    bad[7, 1] = np.nan
    with pytest.raises(SurfaceError):
        acc.Build(Lines(bad, seg, rad))
    seg2 = seg.copy()
    seg2[5, 1] = pos.shape[0] + 3
    with pytest.raises(SurfaceError):
        acc.Build(Lines(pos, seg2, rad))
    acc.Build(Lines(pos, seg, rad))
    gn, gi = acc.export()
    on, oi = O.OracleLines(pos, seg, rad).export()
    assert np.array_equal(O.line_nodes_masked(on).tobytes(), O.line_nodes_masked(gn).tobytes())
    assert np.array_equal(gi, oi)
