"""Scene (RenderGraph) oracle pinned to the reference's own code, on the CPU.

* Matrixd::Inverse: the oracle's and the product's host restatement against
  the reference's routine, bit for bit.
* BVHTree: the oracle's top-level tree (node boxes, children, axes, leaf
  ids) and per-ray candidate lists (entry distance and order) against the
  reference's BVHTree build and Trace.
* RenderGraph::Trace: the oracle's scene trace against a composition of the
  reference's own pieces -- its BVHTree candidates, its accels' Traverse on
  the local rays (triangles, tetrahedra, particles, lines, solids), and the
  world-distance rule of gles/gles_render_graph.cc:170-306 written out in
  numpy."""
import numpy as np
import pytest

from oracle import oracle as O
from surface_b200 import scenes as S

from conftest import bits

needs_ref = pytest.mark.skipif(not O.have_ref(), reason="reference harness not built")
FLT_MAX = np.float32(3.4028234663852886e38)


def _random_matrices(rng, n):
    out = []
    for i in range(n):
        if i % 3 == 0:
            out.append(rng.normal(size=(4, 4)))
        else:
            out.append(S.affine(rng.normal(size=3), rng.uniform(0, 360),
                                rng.uniform(0.2, 3.0, size=3), rng.uniform(-5, 5, size=3)))
    out.append(np.eye(4))
    out.append(S.affine(scale=(2.0, 0.5, 1.0)))
    return out


@needs_ref
def test_matrix_inverse_matches_reference():
    import surface_b200.scene as SC
    rng = np.random.default_rng(3)
    for m in _random_matrices(rng, 300):
        r = O.matrix_inverse(m, use_ref=True)
        assert np.array_equal(bits(O.matrix_inverse(m)), bits(r))
        assert np.array_equal(bits(SC.matrix_inverse(m)), bits(r))


def test_element_update_world_box():
    """TransformBoundingBox: min/max over the eight transformed corners."""
    rng = np.random.default_rng(4)
    for m in _random_matrices(rng, 50):
        lo = rng.uniform(-2, 0, size=3)
        hi = lo + rng.uniform(0, 3, size=3)
        iT, iT33, wlo, whi = O.element_update(m, lo, hi)
        c = np.array([[hi[0] if k & 1 else lo[0], hi[1] if k & 2 else lo[1],
                       hi[2] if k & 4 else lo[2]] for k in range(8)])
        x = ((m[0][None, :3] * c[:, :1] + m[1][None, :3] * c[:, 1:2])
             + m[2][None, :3] * c[:, 2:3]) + m[3][None, :3]
        assert np.array_equal(wlo, x.min(0)) and np.array_equal(whi, x.max(0))
        assert np.array_equal(bits(iT), bits(O.matrix_inverse(m)))
        m33 = m.copy()
        m33[3, :3] = 0.0
        assert np.array_equal(bits(iT33), bits(O.matrix_inverse(m33)))


def _boxes(rng, n, kind):
    if kind == "random":
        lo = rng.uniform(-10, 10, size=(n, 3))
        hi = lo + rng.uniform(0.01, 4, size=(n, 3))
    elif kind == "grid":  # touching boxes: shared faces, tied entry distances
        k = int(np.ceil(n ** (1 / 3)))
        idx = np.stack(np.unravel_index(np.arange(n), (k, k, k)), 1).astype(np.float64)
        lo, hi = idx, idx + 1.0
    elif kind == "dups":  # identical and nested boxes: no spatial split
        lo = np.repeat(rng.uniform(-1, 1, size=((n + 2) // 3, 3)), 3, 0)[:n]
        hi = lo + 1.0
        lo[1::4] += 0.25
    else:  # flat: zero extent on one axis
        lo = rng.uniform(-5, 5, size=(n, 3))
        lo[:, 1] = 0.0
        hi = lo + rng.uniform(0.1, 2, size=(n, 3))
        hi[:, 1] = 0.0
    return lo, hi


@needs_ref
@pytest.mark.parametrize("kind", ["random", "grid", "dups", "flat"])
@pytest.mark.parametrize("n", [1, 2, 3, 7, 16, 100, 1000])
def test_top_tree_matches_reference(kind, n):
    rng = np.random.default_rng(n * 7 + len(kind))
    lo, hi = _boxes(rng, n, kind)
    ref = O.RefTopTree(lo, hi)
    ours = O.OracleScene([None] * n, np.zeros((n, 16)), np.zeros((n, 16)), np.zeros((n, 16)),
                         lo, hi)
    rb, ri = ref.nodes()
    ob, oi = ours.nodes()
    assert rb.shape == ob.shape
    # BVHNode leaves axis unset on leaves and nodeID unset on branches
    leaf = ri[:, 3] == 1
    assert np.array_equal(leaf, oi[:, 3] == 1)
    assert np.array_equal(ri[:, :2], oi[:, :2])
    assert np.array_equal(ri[~leaf, 2], oi[~leaf, 2])
    assert np.array_equal(ri[leaf, 4], oi[leaf, 4])
    assert np.array_equal(bits(rb), bits(ob))
    # candidate lists: entry distance and order
    c = 0.5 * (lo.min(0) + hi.max(0))
    rad = np.linalg.norm(hi.max(0) - lo.min(0))
    for i in range(300):
        o = c + rad * rng.normal(size=3)
        d = (lo[rng.integers(n)] + rng.uniform(size=3) * (hi[0] - lo[0] + 1e-3)) - o
        if i % 5 == 0:
            d = np.zeros(3)
            d[i % 3] = 1.0 if i % 2 else -1.0
        d = d.astype(np.float32).astype(np.float64)
        o = o.astype(np.float32).astype(np.float64)
        rt, rid = ref.candidates(o, d)
        ot, oid = ours.candidates(o, d)
        if rt.size > 16:  # std::sort beyond 16 is not stable: compare as sets
            assert sorted(zip(rt.tolist(), rid.tolist())) == sorted(zip(ot.tolist(),
                                                                       oid.tolist()))
        else:
            assert np.array_equal(rid, oid)
            assert np.array_equal(bits(rt), bits(ot))


# ----------------------------------------------------------------- trace
def _multv(m, v):
    m = m.reshape(4, 4)
    return ((m[0][None, :3] * v[:, :1] + m[1][None, :3] * v[:, 1:2])
            + m[2][None, :3] * v[:, 2:3]) + m[3][None, :3]


def _ref_accel(e):
    if e["kind"] == 3:
        return O.RefLines(e["verts"], e["segments"], e["radius"])
    if e["kind"] == 4:
        return O.RefSolids(e["nv"], e["verts"], e["faces"])
    if e["kind"] == 0:
        return O.RefAccel(O.TRI, e["verts"], e["faces"])
    if e["kind"] == 1:
        return O.RefAccel(O.TET, e["verts"], e["faces"])
    return O.RefAccel(O.SPHERE, e["verts"], None, e["radius"])


def _oracle_accel(e):
    if e["kind"] == 3:
        return O.OracleLines(e["verts"], e["segments"], e["radius"])
    if e["kind"] == 4:
        return O.OracleSolids(e["nv"], e["verts"], e["faces"])
    if e["kind"] == 0:
        return O.OracleAccel(O.TRI, e["verts"], e["faces"])
    if e["kind"] == 1:
        return O.OracleAccel(O.TET, e["verts"], e["faces"])
    return O.OracleAccel(O.SPHERE, e["verts"], None, e["radius"])


def composed_reference_trace(refs, mats, tree, rays, prev_element=None, prev_normals=None):
    """RenderGraph::Trace from the reference's own BVHTree and accels."""
    n = rays.size
    ro = rays["org"].astype(np.float64)
    rd = rays["dir"].astype(np.float64)
    per = []
    for e, (acc, (T, iT, iT33)) in enumerate(zip(refs, mats)):
        lo, ld = _multv(iT, ro), _multv(iT33, rd)
        lr = rays.copy()
        lr["org"] = lo.astype(np.float32)
        lr["dir"] = ld.astype(np.float32)
        same = (np.zeros(n, bool) if prev_element is None
                else prev_element.astype(np.uint32) == e)
        lr["prev_prim"] = np.where(same, rays["prev_prim"], S.MISS)
        lr["prev_t"] = np.where(same, rays["prev_t"], np.float32(0))
        pn = np.zeros((n, 3), np.float32)
        if prev_normals is not None:
            pn[same] = prev_normals[same]
        if isinstance(acc, (O.RefLines, O.RefSolids)):  # no self-hit normal
            h = acc.trace(lr)[0]
        else:
            h = acc.trace(lr, pn)
        if isinstance(h, tuple):  # tetrahedra also return the sub-face
            h = h[0]
        with np.errstate(over="ignore", invalid="ignore"):  # misses carry FLT_MAX
            lp = (lo + h["t"].astype(np.float64)[:, None] * ld).astype(np.float32)
            wp = _multv(T, lp.astype(np.float64)).astype(np.float32)
            po = wp - rays["org"]
            tw = np.sqrt(po[:, 0] * po[:, 0] + po[:, 1] * po[:, 1] + po[:, 2] * po[:, 2])
        ok = (h["prim"] != S.MISS) & (h["t"] < FLT_MAX)
        per.append((h, tw, ok))
    hits = np.zeros(n, O.HIT_DTYPE)
    hits["t"] = FLT_MAX
    hits["prim"] = S.MISS
    el = np.full(n, S.MISS, np.uint32)
    for i in range(n):
        tm, ids = tree.candidates(ro[i], rd[i])
        tnear = np.finfo(np.float64).max
        for t0, e in zip(tm, ids):
            if tnear < t0:
                continue
            h, tw, ok = per[e]
            if ok[i] and np.float64(tw[i]) < tnear:
                tnear = np.float64(tw[i])
                hits[i] = h[i]
                hits[i]["t"] = tw[i]
                el[i] = e
    return hits, el


def build_scene_pair(elems, bboxes):
    """(oracle scene, reference accels, matrices, reference tree) from the
    elements and their local boxes."""
    mats, wlo, whi = [], [], []
    for e, (lo, hi) in zip(elems, bboxes):
        iT, iT33, a, b = O.element_update(e["T"], lo, hi)
        mats.append((e["T"].reshape(16), iT.reshape(16), iT33.reshape(16)))
        wlo.append(a)
        whi.append(b)
    return mats, np.array(wlo), np.array(whi)


@needs_ref
@pytest.mark.parametrize("mix", ["accels", "lines_solids"])
def test_scene_trace_matches_composed_reference(mix):
    elems = (S.scene_elements(seed=31) if mix == "accels" else
             S.scene_elements(seed=43, ntri=1, nsph=1, ntet=1, nline=2, nsolid=3))
    refs = [_ref_accel(e) for e in elems]
    orcs = [_oracle_accel(e) for e in elems]
    mats, wlo, whi = build_scene_pair(elems, [r.bbox() for r in refs])
    tree = O.RefTopTree(wlo, whi)
    scene = O.OracleScene(orcs, [m[0] for m in mats], [m[1] for m in mats],
                          [m[2] for m in mats], wlo, whi)
    rays = S.scene_rays(3000, wlo.min(0), whi.max(0), seed=9, boxes=(wlo, whi))
    want, wel = composed_reference_trace(refs, mats, tree, rays)
    got, gel = scene.trace(rays)
    assert np.array_equal(gel, wel)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    assert (wel != S.MISS).mean() > 0.2 and len(set(wel[wel != S.MISS].tolist())) == len(elems)
    # secondary rays leaving the hit element: the self-hit rule applies
    # only inside prev_element
    hit = np.nonzero(wel != S.MISS)[0]
    sec = np.zeros(hit.size, O.RAY_DTYPE)
    p = rays["org"][hit] + want["t"][hit, None] * rays["dir"][hit]
    rng = np.random.default_rng(2)
    sec["org"] = p
    sec["dir"] = S._normalize(rng.normal(size=(hit.size, 3))).astype(np.float32)
    sec["prev_prim"] = want["prim"][hit]
    sec["prev_t"] = want["t"][hit]
    pe = wel[hit]
    pn = S._normalize(rng.normal(size=(hit.size, 3))).astype(np.float32)
    want2, wel2 = composed_reference_trace(refs, mats, tree, sec, pe, pn)
    got2, gel2 = scene.trace(sec, pe, pn)
    assert np.array_equal(gel2, wel2)
    assert np.array_equal(got2.view(np.uint32), want2.view(np.uint32))


@needs_ref
def test_oracle_local_box_matches_reference():
    """XxxAccel::BoundingBox (the RenderElement's local box)."""
    for e in S.scene_elements(seed=31):
        a, r = _oracle_accel(e), _ref_accel(e)
        assert np.array_equal(bits(np.concatenate(a.bbox64())), bits(np.concatenate(r.bbox())))
