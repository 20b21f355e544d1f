"""Texture::Fetch for 3D textures: the oracle's restatement against the
reference's own code, bit for bit (dense FilterTexture3D{Byte,Float,Double}
with wrap modes and non-uniform coordinate remaps; sparse volumes through
SparseVolumeAccel)."""
import numpy as np
import pytest

from oracle import oracle as O
from surface_b200 import scenes as S

from conftest import bits

needs_ref = pytest.mark.skipif(not O.have_ref(), reason="reference harness not built")


def coords(n, seed, lo=-0.3, hi=1.3, dims=(9, 7, 5)):
    rng = np.random.default_rng(seed)
    c = rng.uniform(lo, hi, size=(n, 3)).astype(np.float32)
    # texel-aligned and boundary coordinates
    k = rng.integers(0, 12, size=(n // 4, 3))
    c[: n // 4] = (k / (np.array(dims) - 1.0)).astype(np.float32)
    c[n // 4: n // 4 + 8] = np.array([0.0, 1.0, -1.0])[np.arange(24).reshape(8, 3) % 3]
    # NaN, infinite and out-of-int-range coordinates (x86 conversions)
    c[-4:] = [[np.nan, 0.5, 0.5], [3e9, 0.5, 0.5], [-3e9, 0.2, 0.1], [0.5, np.inf, 0.5]]
    return c


@needs_ref
@pytest.mark.parametrize("fmt", [0, 1, 2])
@pytest.mark.parametrize("comps", [1, 3, 4])
def test_dense_fetch_matches_reference(fmt, comps):
    img = S.dense_texture(fmt, comps=comps, seed=fmt * 10 + comps)
    uvw = coords(4000, fmt + 7 * comps)
    for clamp in ((1, 1, 1), (0, 0, 0), (1, 0, 1)):
        for remap in ((None, None, None), (None, S.remap_table(8), None),
                      (S.remap_table(5, 3), S.remap_table(17, 4), S.remap_table(2, 5))):
            got = O.tex_fetch(fmt, img, comps, uvw, clamp, remap)
            want = O.tex_fetch(fmt, img, comps, uvw, clamp, remap, use_ref=True)
            assert np.array_equal(bits(got), bits(want)), (clamp, remap)


@needs_ref
@pytest.mark.parametrize("fmt", [0, 1, 2])
@pytest.mark.parametrize("comps", [1, 2, 4])
@pytest.mark.parametrize("overlap", [False, True])
def test_sparse_fetch_matches_reference(fmt, comps, overlap):
    blocks, pool, gdim = S.sparse_blocks(fmt, comps, seed=fmt + 3 * comps, overlap=overlap)
    rng = np.random.default_rng(comps)
    uvw = rng.uniform(-0.05, 1.05, size=(6000, 3)).astype(np.float32)
    # points on block faces and corners
    b = blocks[rng.integers(0, blocks.size, size=500)]
    face = b["offset"] + b["extent"] * rng.integers(0, 2, size=(500, 3))
    uvw[:500] = (face / np.array(gdim)).astype(np.float32)
    got = O.sparse_fetch(blocks, pool, fmt, comps, gdim, uvw)
    want = O.sparse_fetch(blocks, pool, fmt, comps, gdim, uvw, use_ref=True)
    assert np.array_equal(bits(got), bits(want))
    assert (want[:, 3] != 0).mean() > 0.05  # a share of the samples lands in blocks


@needs_ref
@pytest.mark.parametrize("case", ("pages",) + S.LOCATE_CASES)
def test_sparse_locate_edge_cases_match_reference(case):
    """Points on block faces, edges and corners, ulps and the tree's 1e-6
    widening off them, for layouts that stress BVHTree::Locate."""
    for fmt, comps in ((0, 1), (1, 3)):
        if case == "pages":
            blocks, pool, gdim = S.sparse_pages(ndiv=4, page=8, seed=5)
            fmt, comps = 0, 1
        else:
            blocks, pool, gdim = S.sparse_locate_case(case, fmt, comps)
        uvw = S.sparse_edge_coords(blocks, gdim, 8000, fmt, spread=(-1.5, 1.5))
        got = O.sparse_fetch(blocks, pool, fmt, comps, gdim, uvw)
        want = O.sparse_fetch(blocks, pool, fmt, comps, gdim, uvw, use_ref=True)
        assert np.array_equal(bits(got), bits(want))
        assert (want[:, 3] != 0).mean() > 0.2
