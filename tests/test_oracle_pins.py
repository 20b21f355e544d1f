"""The CPU oracle pinned against the reference: its own known answers and
invariants (test/cctest/test-prefix-tree.cc), golden fixtures generated from the
reference's code (tests/golden/make_golden.py), and -- when the reference build
is present -- direct differential runs against it."""
import numpy as np
import pytest

from oracle import oracle as O
from surface_b200 import scenes as S

from conftest import bits

NS = [8, 15, 31, 1023, 1000, 3211]


def test_tinymt64_restatement_matches_fixture(golden):
    g = golden("prefix_tree.npz")
    d = O.tinymt64_doubles(3 * sum(NS))
    off = 0
    for n in NS:
        pts = d[off:off + 3 * n].astype(np.float32).reshape(n, 3)
        off += 3 * n
        assert np.array_equal(bits(pts), bits(g[f"pts_{n}"]))


@pytest.mark.skipif(not O.have_ref(), reason="reference build absent")
def test_tinymt64_restatement_matches_reference():
    assert np.array_equal(O.tinymt64_doubles(5000), O.tinymt64_doubles(5000, use_ref=True))


def test_morton_known_answer():
    # test/cctest/test-prefix-tree.cc:27-41: (0.5,0.5,0.5) in the unit box, inv 1024
    c = O.morton_points(np.array([[0.5, 0.5, 0.5]], np.float32), [0, 0, 0], [1, 1, 1])
    assert int(c[0]) == (1 << 29) | (1 << 28) | (1 << 27)
    assert O.lib().so_morton_bits(512, 512, 512) == (1 << 29) | (1 << 28) | (1 << 27)


def test_morton_codes_match_reference_fixture(golden):
    g = golden("prefix_tree.npz")
    for n in NS:
        c = O.morton_points(g[f"pts_{n}"], [0, 0, 0], [1, 1, 1])
        assert np.array_equal(c, g[f"codes_{n}"])
        # the reference's SSE path agrees with its scalar path (:44-82)
        assert np.array_equal(c, g[f"codes_simd_{n}"])


def test_sort_is_stable_and_matches_reference(golden):
    g = golden("prefix_tree.npz")
    for n in NS:
        c, i = O.sort_pairs(g[f"codes_{n}"])
        assert np.all(c[:-1] <= c[1:])
        tie = c[:-1] == c[1:]
        assert np.all(i[:-1][tie] < i[1:][tie])
        assert np.array_equal(c, np.sort(g[f"codes_{n}"]))
    c, i = O.sort_pairs(g["codes_3211"])
    assert np.array_equal(c, g["sorted_codes_3211"])
    assert np.array_equal(i, g["sorted_index_3211"])


def _karras_invariants(child, lt, rt, n):
    # every leaf referenced exactly once, flat count (test-prefix-tree.cc:470-488)
    cnt = np.zeros(n, np.int64)
    np.add.at(cnt, child[lt == 1], 1)
    np.add.at(cnt, child[rt == 1] + 1, 1)
    assert np.all(cnt == 1)
    # ... and by a walk from the root, depth < 30 for distinct keys
    seen = np.zeros(n, np.int64)
    stack = [(0, 0)]
    maxd = 0
    while stack:
        i, d = stack.pop()
        maxd = max(maxd, d)
        g = int(child[i])
        for side, leaf in ((0, lt[i]), (1, rt[i])):
            c = g + side
            if leaf:
                seen[c] += 1
            else:
                stack.append((c, d + 1))
    assert np.all(seen == 1)
    return maxd


def test_karras_matches_reference_fixture(golden):
    g = golden("prefix_tree.npz")
    for n in NS:
        sc = np.sort(g[f"codes_{n}"])
        child, lt, rt = O.karras(sc)
        assert np.array_equal(child, g[f"child_{n}"])
        assert np.array_equal(lt, g[f"ltype_{n}"])
        assert np.array_equal(rt, g[f"rtype_{n}"])
        assert _karras_invariants(child, lt, rt, n) < 30
        # all keys equal (test-prefix-tree.cc:700-918)
        cs = g[f"same_codes_{n}"]
        assert np.all(cs == cs[0])
        child, lt, rt = O.karras(cs)
        assert np.array_equal(child, g[f"same_child_{n}"])
        assert np.array_equal(lt, g[f"same_ltype_{n}"])
        assert np.array_equal(rt, g[f"same_rtype_{n}"])
        _karras_invariants(child, lt, rt, n)


@pytest.mark.parametrize("tag,kind", [("tri", O.TRI), ("tet", O.TET), ("sph", O.SPHERE)])
def test_oracle_build_and_trace_match_reference_fixture(golden, tag, kind):
    g = golden("scenes_small.npz")
    if kind == O.TRI:
        acc = O.OracleAccel(kind, g["tri_verts"], g["tri_faces"])
    elif kind == O.TET:
        acc = O.OracleAccel(kind, g["tet_verts"], g["tet_faces"])
    else:
        acc = O.OracleAccel(kind, g["sph_pos"], None, g["sph_rad"])
    assert np.array_equal(acc.canonical(), g[f"{tag}_canon"])
    assert np.array_equal(acc.indices, g[f"{tag}_index"])
    if kind == O.TET:
        h, sub = acc.trace(g["tet_rays"], want_subface=True)
        assert np.array_equal(sub, g["tet_subface"])
    else:
        h = acc.trace(g[f"{tag}_rays"])
    ref = g[f"{tag}_hits"]
    for f in ("t", "u", "v", "prim"):
        assert np.array_equal(bits(h[f]), bits(ref[f])), f
    if kind == O.SPHERE:
        # secondaries (self-hit rule); u, v = BuildIntersection's spherical coordinates
        h2 = acc.trace(g["sph_sec_rays"], prev_normals=g["sph_sec_normals"])
        for f in ("t", "u", "v", "prim"):
            assert np.array_equal(bits(h2[f]), bits(g["sph_sec_hits"][f])), f


def test_tex3d_matches_reference_fixture(golden):
    g = golden("texture3d.npz")
    img = g["tex_img"]
    d, h, w = img.shape
    for mode in (0, 1):
        out = O.tex3d(img, (w, h, d), g["tex_uvw"], clamp=(mode, mode, mode))
        assert np.array_equal(bits(out), bits(g[f"tex_out_clamp{mode}"]))


# ---------------------------------------------------------------- direct runs
need_ref = pytest.mark.skipif(not O.have_ref(), reason="reference build absent")


@need_ref
@pytest.mark.parametrize("levels", [5, 6])
def test_oracle_vs_reference_triangles(levels):
    v, f = S.displaced_octasphere(levels, seed=levels)
    o = O.OracleAccel(O.TRI, v, f)
    r = O.RefAccel(O.TRI, v, f)
    rc, ridx = r.canonical()
    assert np.array_equal(o.canonical(), rc)
    assert np.array_equal(o.indices, ridx)
    rays = S.pinhole_rays(96, 96, (0, 0, 3), (0, 0, 0))
    ho, hr = o.trace(rays), r.trace(rays)
    for k in ("t", "u", "v", "prim"):
        assert np.array_equal(bits(ho[k]), bits(hr[k]))


@need_ref
def test_oracle_vs_reference_tetra():
    v, f, _ = S.tet_grid(12, seed=3)
    o = O.OracleAccel(O.TET, v, f)
    r = O.RefAccel(O.TET, v, f)
    rc, ridx = r.canonical()
    assert np.array_equal(o.canonical(), rc)
    rays = S.ortho_rays(96, 96)
    (ho, so), (hr, sr) = o.trace(rays, want_subface=True), r.trace(rays)
    assert np.array_equal(so, sr)
    for k in ("t", "u", "v", "prim"):
        assert np.array_equal(bits(ho[k]), bits(hr[k]))
    # oblique rays exercise all Pluecker branches
    obl = S.pinhole_rays(64, 64, (1.7, 1.3, 2.1), (0.5, 0.5, 0.5), fov_deg=50)
    ho, hr = o.trace(obl), r.trace(obl)[0]
    for k in ("t", "u", "v", "prim"):
        assert np.array_equal(bits(ho[k]), bits(hr[k]))


@need_ref
@pytest.mark.parametrize("shift", [0.0, 100.0])
def test_oracle_vs_reference_tetra_double_positions(shift):
    """isDoublePrecisionPos: tetrahedra over float64 positions that float
    does not hold (sub-ulp jitter, shifted away from the origin): the
    oracle's Build32 (double-padded boxes, Morton codes of the rounded
    positions) and Pluecker tests over the doubles equal the reference's,
    which differ from a build over the rounded positions."""
    v, f, _ = S.tet_grid(12, seed=3)
    rng = np.random.default_rng(9)
    v64 = v.astype(np.float64) + shift + rng.uniform(-1e-9, 1e-9, size=v.shape)
    o = O.OracleAccel(O.TET, v64, f)
    r = O.RefAccel(O.TET, v64, f)
    assert o.verts.dtype == np.float64 and r.verts.dtype == np.float64
    rc, ridx = r.canonical()
    assert np.array_equal(o.canonical(), rc)
    assert np.array_equal(o.indices, ridx)
    rays = S.ortho_rays(96, 96)
    rays["org"] += np.float32(shift)
    obl = S.pinhole_rays(64, 64, (1.7 + shift, 1.3 + shift, 2.1 + shift),
                         (0.5 + shift, 0.5 + shift, 0.5 + shift), fov_deg=50)
    for rr in (rays, obl):
        (ho, so), (hr, sr) = o.trace(rr, want_subface=True), r.trace(rr)
        assert np.array_equal(so, sr)
        for k in ("t", "u", "v", "prim"):
            assert np.array_equal(bits(ho[k]), bits(hr[k]))
        assert (hr["prim"] != O.MISS).mean() > 0.3
    f32 = O.OracleAccel(O.TET, v64.astype(np.float32), f)
    hf = f32.trace(obl)
    assert not all(np.array_equal(bits(hf[k]), bits(ho[k])) for k in ("t", "u", "v"))


@need_ref
def test_oracle_vs_reference_spheres_with_coincident_points():
    pos, rad = S.particles(20000, seed=4)
    pos[100:400] = pos[100]  # coincident centres (same Morton key)
    o = O.OracleAccel(O.SPHERE, pos, None, rad)
    r = O.RefAccel(O.SPHERE, pos, None, rad)
    rc, ridx = r.canonical()
    assert np.array_equal(o.canonical(), rc)
    assert np.array_equal(o.indices, ridx)
    rays = S.pinhole_rays(96, 96, (0.5, 0.5, 2.2), (0.5, 0.5, 0.5), fov_deg=30)
    ho, hr = o.trace(rays), r.trace(rays)
    for k in ("t", "u", "v", "prim"):
        assert np.array_equal(bits(ho[k]), bits(hr[k])), k


@need_ref
def test_oracle_vs_reference_flat_mesh():
    # a z-flat sheet: zero extent on one axis -> inf scale in the quantiser
    v, f = S.displaced_octasphere(5, seed=9)
    v[:, 2] = 0.25
    o = O.OracleAccel(O.TRI, v, f)
    r = O.RefAccel(O.TRI, v, f)
    rc, ridx = r.canonical()
    assert np.array_equal(o.canonical(), rc)
    assert np.array_equal(o.indices, ridx)


CAMERAS = [((0, 0, 3), (0, 0, 0), (0, 1, 0), 45.0, 0, 512, 512),
           ((0.3, 0.2, 3), (0, 0.1, 0), (0, 1, 0), 30.0, 0, 640, 480),
           ((1, 2, 3), (0, 0, 0), (0, 0, 1), 60.0, 1, 300, 200),
           ((0.5, 0.5, 2.2), (0.5, 0.5, 0.5), (0, 1, 0), 30.0, 0, 2048, 2048),
           ((-4, 1, -2), (0.2, -0.3, 0.9), (0.1, 1, 0), 75.0, 0, 333, 97)]


@pytest.mark.skipif(not O.have_ref(), reason="reference build absent")
@pytest.mark.parametrize("cam", CAMERAS)
def test_camera_frame_matches_reference(cam):
    """The restated Camera::buildFrame equals the reference's, bit for bit."""
    a = O.camera_frame(*cam)
    b = O.camera_frame(*cam, use_ref=True)
    for x, y in zip(a, b):
        assert np.array_equal(x.view(np.uint32), y.view(np.uint32))


@pytest.mark.skipif(not O.have_ref(), reason="reference build absent")
def test_stereo_env_ray_matches_reference():
    """The restated Camera::generateStereoEnvRay equals the reference's, bit
    for bit, over both eye halves of the image and random cameras."""
    rng = np.random.default_rng(11)
    for _ in range(400):
        eye = rng.uniform(-3, 3, 3).astype(np.float32)
        la = rng.uniform(-1, 1, 3).astype(np.float32)
        up = np.float32([0, 1, 0]) if rng.random() < 0.7 else rng.normal(size=3).astype(np.float32)
        W, H = int(rng.integers(8, 400)), int(rng.integers(8, 400))
        u, v = np.float32(rng.uniform(0, W)), np.float32(rng.uniform(0, H))
        zp, es = np.float32(rng.uniform(0.5, 5)), np.float32(rng.uniform(0.01, 0.2))
        a = O.stereo_env_ray(eye, la, up, zp, es, u, v, W, H)
        b = O.stereo_env_ray(eye, la, up, zp, es, u, v, W, H, use_ref=True)
        for x, y in zip(a, b):
            assert np.array_equal(x.view(np.uint32), y.view(np.uint32))


@pytest.mark.skipif(not O.have_ref(), reason="reference build absent")
def test_subsample_jitter_is_the_serial_stream():
    """The restated loop's jitter: pixel by pixel, subsample (vv, uu) lies at
    ((uu + ju) / S, (vv + jv) / S) with ju (uu != 0) then jv (vv != 0) taken
    in order from the reference's TinyMT64 stream (seed 1234,
    initialize_random's parameters) as floats.  Orthographic rays give the
    sample positions back exactly enough to read the jitter off them."""
    cam = {"eye": (0, 0, 3), "lookat": (0, 0, 0), "up": (0, 1, 0), "fov": 0.0,
           "ortho": 1, "width": 8, "height": 4, "viewport": (0, 0, 8, 4),
           "region": (0, 0, 8, 4), "step": 1}
    S = 3
    rays, pix = O.camera_rays_ex(cam, S, offset=5)
    D = 2 * S * (S - 1)
    draws = O.tinymt64_doubles(5 + 32 * D, seed=1234, use_ref=True)[5:].astype(np.float32)
    rays0, _ = O.camera_rays_ex(cam, 1)
    corner, u, v = O.camera_frame(*[cam[k] for k in ("eye", "lookat", "up", "fov", "ortho",
                                                     "width", "height")])
    k = 0
    for q in range(32):
        for vv in range(S):
            for uu in range(S):
                ju = draws[k] if uu else np.float32(0)
                k += 1 if uu else 0
                jv = draws[k] if vv else np.float32(0)
                k += 1 if vv else 0
                r = rays[q * S * S + vv * S + uu]
                su = np.float32(np.float32(uu) + ju) / np.float32(S)
                sv = np.float32(np.float32(vv) + jv) / np.float32(S)
                # offset from the pixel's first sample, along u and v
                off = r["org"].astype(np.float64) - rays[q * S * S]["org"].astype(np.float64)
                assert abs(off @ u / (u @ u) - su) < 1e-3
                assert abs(off @ v / (v @ v) - sv) < 1e-3
    assert k == 32 * D


def test_camera_rays_restatement_properties():
    """Eye rays of the restated OnData loop: unit directions, the pinhole
    rays pass through the eye, the viewport offset shifts pixels."""
    cam = {"eye": (0, 0, 3), "lookat": (0, 0, 0), "up": (0, 1, 0), "fov": 45.0,
           "ortho": 0, "width": 64, "height": 48, "viewport": (0, 0, 64, 48),
           "region": (0, 0, 64, 48), "step": 1}
    rays, pix = O.camera_rays(cam)
    assert rays.size == 64 * 48
    assert np.allclose(np.linalg.norm(rays["dir"], axis=1), 1, atol=1e-6)
    assert np.all(rays["org"] == np.float32([0, 0, 3]))
    sh, pix = O.camera_rays(dict(cam, viewport=(8, 0, 64, 48)))
    # pixels converted off screen are skipped; x = 7 converts to -0.5, which
    # the int conversion truncates to 0, so it stays
    assert sh.size == (64 - 7) * 48
    assert (pix & 0xFFFF).min() == 7


def test_reference_dump_fixtures_match_oracle(golden):
    """The Dump() files written by the reference (tests/golden/dumps_small.npz)
    hold the oracle's tree and sorted order for the same scenes."""
    g = golden("dumps_small.npz")
    for tag, kind, acc in (("tri", O.TRI, lambda: O.OracleAccel(O.TRI, g["tri_verts"],
                                                                g["tri_faces"])),
                           ("tet", O.TET, lambda: O.OracleAccel(O.TET, g["tet_verts"],
                                                                g["tet_faces"])),
                           ("sph", O.SPHERE, lambda: O.OracleAccel(O.SPHERE, g["sph_pos"],
                                                                   None, g["sph_rad"]))):
        nodes, idx = O.parse_dump(kind, g[f"{tag}_dump"].tobytes())
        o = acc()
        assert np.array_equal(idx, o.indices)
        assert np.array_equal(O.canonicalize(nodes, 0), o.canonical())


def test_lines_solids_sparse_fixtures(golden):
    """The oracle's LineAccel, SolidAccel (Build32) and sparse-volume fetch
    against the reference's own outputs stored in lines_solids.npz (made by
    tests/golden/make_golden.py): trees, hits, normals, positions, texels."""
    g = golden("lines_solids.npz")
    for tag in ("line", "edge"):
        o = O.OracleLines(g[f"{tag}_pos"], g[f"{tag}_seg"], g[f"{tag}_rad"])
        nodes, idx = O.parse_line_dump(g[f"{tag}_dump"].tobytes())
        on, oi = o.export()
        assert O.line_nodes_masked(on).tobytes() == O.line_nodes_masked(nodes).tobytes()
        assert np.array_equal(oi, idx)
        h, n = o.trace(g[f"{tag}_rays"])
        assert np.array_equal(bits(h.view(np.float32).reshape(-1, 4)), bits(g[f"{tag}_hits"]))
        assert np.array_equal(bits(n), bits(g[f"{tag}_normals"]))
    for nv in (8, 6, 5):
        o = O.OracleSolids(nv, g[f"solid{nv}_verts"], g[f"solid{nv}_ix"])
        on, oi = o.export()
        ref_nodes = g[f"solid{nv}_nodes"].view(O.SOLID_NODE_DTYPE)
        assert O.tree_canonical(on) == O.tree_canonical(ref_nodes)
        assert np.array_equal(oi, g[f"solid{nv}_idx"])
        h, n, q = o.trace(g[f"solid{nv}_rays"])
        assert np.array_equal(bits(h.view(np.float32).reshape(-1, 4)), bits(g[f"solid{nv}_hits"]))
        assert np.array_equal(bits(n), bits(g[f"solid{nv}_normals"]))
        assert np.array_equal(bits(q), bits(g[f"solid{nv}_positions"]))
    blocks = g["sp_blocks"].view(O.BLOCK_DTYPE)
    got = O.sparse_fetch(blocks, g["sp_pool"].tobytes(), 0, 1, tuple(g["sp_gdim"]), g["sp_uvw"])
    assert np.array_equal(bits(got), bits(g["sp_rgba"]))
