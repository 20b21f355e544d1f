"""The product's default traversal (front-to-back pass, reference-order
replay only for exact ties, reference walk when a candidate at the smallest
distance reports a distance before its leaf box's entry), restated in the oracle
(so_trace2), against the reference's Traverse (so_trace, itself pinned to the
reference build): identical hits on every ray."""
import numpy as np
import pytest

from oracle import oracle as O
from surface_b200 import scenes as S

from conftest import bits


def same(h1, h2, fields=("t", "u", "v", "prim")):
    for f in fields:
        assert np.array_equal(bits(h1[f]), bits(h2[f])), f


def test_triangles_and_exact_ties():
    v, f = S.displaced_octasphere(6, seed=41)
    o = O.OracleAccel(O.TRI, v, f)
    rays = S.pinhole_rays(192, 192, (0, 0, 3), (0, 0, 0))
    same(o.trace2(rays), o.trace(rays))
    dup = O.OracleAccel(O.TRI, v, np.concatenate([f, f[::-1]]))
    rays = S.pinhole_rays(96, 96, (0, 0, 3), (0, 0, 0))
    same(dup.trace2(rays), dup.trace(rays))


def test_tetrahedra_ortho_ties_and_oblique():
    v, f, _ = S.tet_grid(24, seed=42)
    o = O.OracleAccel(O.TET, v, f)
    for rays in (S.ortho_rays(192, 192),
                 S.pinhole_rays(96, 96, (1.7, 1.3, 2.1), (0.5, 0.5, 0.5), fov_deg=50)):
        (h2, s2), (h1, s1) = o.trace2(rays, want_subface=True), o.trace(rays, want_subface=True)
        same(h2, h1)
        assert np.array_equal(s2, s1)


def pole_pairs(n=48, z=0.5, dist=4.0, gap=5e-7, seed=45):
    """Sphere pairs hit at their poles: centres on an n x n grid at height z,
    each with a twin `gap` further down, and one orthographic ray down -z from
    z + dist through every centre.  A pole hit lies one leaf padding (16
    ulp(1)) behind its box face, less than the float error of a hit distance
    of ~4, so some hits report a distance below their box's entry, and the
    twin's hit lies within that error too -- the case where the reference's
    pruning decides which of the two it reports."""
    rng = np.random.default_rng(seed)
    g = (np.arange(n) + 0.5) / n
    X, Y = np.meshgrid(g, g)
    c = np.stack([X.ravel(), Y.ravel(), np.full(n * n, z)], 1).astype(np.float32)
    twin = c.copy()
    twin[:, 2] -= np.float32(gap)
    order = rng.permutation(2 * n * n)
    pos = np.concatenate([c, twin])[order]
    rad = np.full(2 * n * n, 0.004, np.float32)
    rays = np.zeros(n * n, O.RAY_DTYPE)
    rays["org"][:, :2] = c[:, :2]
    rays["org"][:, 2] = z + dist
    rays["dir"][:, 2] = -1.0
    rays["prev_prim"] = O.MISS
    return pos, rad, rays


def test_spheres_fallback_path():
    pos, rad = S.particles(300_000, seed=43)
    o = O.OracleAccel(O.SPHERE, pos, None, rad)
    rays = S.pinhole_rays(160, 160, (0.5, 0.5, 2.2), (0.5, 0.5, 0.5), fov_deg=30)
    h2, st = o.trace2(rays, want_stats=True)
    same(h2, o.trace(rays), ("t", "prim"))
    # pole hits with a twin inside the rounding window take the reference walk
    pp, pr, prays = pole_pairs()
    op = O.OracleAccel(O.SPHERE, pp, None, pr)
    hp, sp = op.trace2(prays, want_stats=True)
    same(hp, op.trace(prays), ("t", "prim"))
    assert sp[3] > 0
    if O.have_ref():
        same(hp, O.RefAccel(O.SPHERE, pp, None, pr).trace(prays), ("t", "prim"))
    # secondary rays with the self-hit rule
    hit = h2["prim"] != O.MISS
    p = rays["org"][hit] + h2["t"][hit, None] * rays["dir"][hit]
    n = p - pos[h2["prim"][hit]]
    n = (n / np.linalg.norm(n, axis=1, keepdims=True)).astype(np.float32)
    sec = np.zeros(int(hit.sum()), O.RAY_DTYPE)
    sec["org"] = p.astype(np.float32)
    sec["dir"] = S.hemisphere_dirs(n, seed=5)
    sec["prev_prim"] = h2["prim"][hit]
    sec["prev_t"] = h2["t"][hit]
    same(o.trace2(sec, prev_normals=n), o.trace(sec, prev_normals=n), ("t", "prim"))


@pytest.mark.skipif(not O.have_ref(), reason="reference build absent")
def test_restated_walk_vs_reference_build():
    v, f, _ = S.tet_grid(16, seed=44)
    rays = S.ortho_rays(128, 128)
    h2, s2 = O.OracleAccel(O.TET, v, f).trace2(rays, want_subface=True)
    hr, sr = O.RefAccel(O.TET, v, f).trace(rays)
    same(h2, hr)
    assert np.array_equal(s2, sr)


def _far_rays(rng, n, lo, hi, dist, scale):
    c = 0.5 * (lo + hi)
    rad = 0.5 * np.linalg.norm(hi - lo)
    o = c + (rad + dist) * S._normalize(rng.normal(size=(n, 3)))
    tgt = lo + rng.uniform(size=(n, 3)) * (hi - lo)
    rays = np.zeros(n, O.RAY_DTYPE)
    rays["org"] = o
    rays["dir"] = S._normalize(tgt - o) * scale
    rays["prev_prim"] = O.MISS
    return rays


@pytest.mark.parametrize("kind", ["tri", "tet", "sphere"])
def test_far_origins_and_scaled_directions(kind):
    """Rays from 10 and 100 units away with non-unit directions (the local
    rays of transformed scene elements): hit distances far above the leaf
    padding, where float distances round below their box's entry."""
    rng = np.random.default_rng({"tri": 1, "tet": 2, "sphere": 3}[kind])
    if kind == "tri":
        v, f = S.displaced_octasphere(5, seed=46)
        o, lo, hi = O.OracleAccel(O.TRI, v, f), -1.1 * np.ones(3), 1.1 * np.ones(3)
    elif kind == "tet":
        v, f, _ = S.tet_grid(20, seed=47)
        o, lo, hi = O.OracleAccel(O.TET, v, f), np.zeros(3), np.ones(3)
    else:
        p, r = S.particles(100_000, seed=48, median_radius=0.01)
        o, lo, hi = O.OracleAccel(O.SPHERE, p, None, r), np.zeros(3), np.ones(3)
    fell = 0
    for dist in (10.0, 100.0):
        for scale in (0.37, 2.9):
            rays = _far_rays(rng, 20_000, lo, hi, dist, scale)
            h2, st = o.trace2(rays, want_stats=True)
            h1 = o.trace(rays)
            same(h2, h1[0] if isinstance(h1, tuple) else h1)
            fell += int(st[3])
    if kind == "sphere":
        assert fell > 0  # the reference-walk fallback is exercised
