"""3D texture fetch on the GPU (srt_texture3d_*) against the oracle, bit for
bit: dense bytes/floats/doubles with 1-4 components, repeat and
clamp-to-edge, non-uniform remap tables; sparse block volumes (touching and
overlapping blocks, all formats)."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from surface_b200 import scenes as S
from surface_b200.texture import Texture3D

from conftest import bits

pytestmark = pytest.mark.gpu


def same(got, want):
    """Bit-exact, except that a NaN's encoding is the hardware's (x86 writes
    the default NaN 0xffc00000, the GPU 0x7fffffff): NaNs must sit at the
    same places."""
    got, want = np.asarray(got), np.asarray(want)
    ng, nw = np.isnan(got), np.isnan(want)
    return np.array_equal(ng, nw) and np.array_equal(bits(np.where(ng, 0, got)),
                                                     bits(np.where(nw, 0, want)))


def coords(n, seed, lo=-0.3, hi=1.3, dims=(9, 7, 5)):
    rng = np.random.default_rng(seed)
    c = rng.uniform(lo, hi, size=(n, 3)).astype(np.float32)
    k = rng.integers(0, 12, size=(n // 4, 3))
    c[: n // 4] = (k / (np.array(dims) - 1.0)).astype(np.float32)
    c[n // 4: n // 4 + 8] = np.array([0.0, 1.0, -1.0])[np.arange(24).reshape(8, 3) % 3]
    c[-4:] = [[np.nan, 0.5, 0.5], [3e9, 0.5, 0.5], [-3e9, 0.2, 0.1], [0.5, np.inf, 0.5]]
    return c


@pytest.mark.parametrize("fmt", [0, 1, 2])
@pytest.mark.parametrize("comps", [1, 2, 4])
def test_dense_fetch_matches_oracle(fmt, comps):
    img = S.dense_texture(fmt, comps=comps, seed=fmt * 10 + comps)
    uvw = coords(20000, fmt + 7 * comps)
    t = Texture3D()
    t.set_dense(img, fmt)
    for clamp in ((1, 1, 1), (0, 0, 0), (1, 0, 1)):
        t.set_wrap(*clamp)
        for remap in ((None, None, None), (None, S.remap_table(8), None),
                      (S.remap_table(5, 3), S.remap_table(17, 4), S.remap_table(2, 5))):
            for axis in range(3):
                t.set_remap(axis, remap[axis])
            got = t.Fetch(uvw)
            want = O.tex_fetch(fmt, img, comps, uvw, clamp, remap)
            assert same(got, want), (clamp, remap)


@pytest.mark.parametrize("fmt", [0, 1, 2])
@pytest.mark.parametrize("comps", [1, 3, 4])
@pytest.mark.parametrize("overlap", [False, True])
def test_sparse_fetch_matches_oracle(fmt, comps, overlap):
    blocks, pool, gdim = S.sparse_blocks(fmt, comps, seed=fmt + 3 * comps, overlap=overlap)
    rng = np.random.default_rng(comps)
    uvw = rng.uniform(-0.05, 1.05, size=(30000, 3)).astype(np.float32)
    b = blocks[rng.integers(0, blocks.size, size=3000)]
    uvw[:3000] = ((b["offset"] + b["extent"] * rng.integers(0, 2, size=(3000, 3)))
                  / np.array(gdim)).astype(np.float32)
    t = Texture3D()
    t.set_sparse(blocks, pool, fmt, comps, gdim)
    got = t.Fetch(torch.from_numpy(uvw).cuda()).cpu().numpy()
    want = O.sparse_fetch(blocks, pool, fmt, comps, gdim, uvw)
    assert same(got, want)
    assert (want[:, 3] != 0).mean() > 0.05


def test_large_texture_and_errors():
    img = S.dense_texture(1, dims=(160, 128, 96), comps=1, seed=3)
    t = Texture3D()
    t.set_dense(img, 1)
    t.set_wrap(True, True, True)  # repeat by default, as Texture's constructor sets
    t.set_remap(2, S.remap_table(97))
    uvw = coords(200_000, 11, 0.0, 1.0, dims=(160, 128, 96))
    want = O.tex_fetch(1, img, 1, uvw, (1, 1, 1), (None, None, S.remap_table(97)))
    assert same(t.Fetch(uvw), want)
    import surface_b200 as sb
    with pytest.raises(sb.SurfaceError):
        t.set_dense(img, 1, components=5)  # at most four components
    blocks, pool, gdim = S.sparse_blocks(1, 1)
    blocks["data_offset"][0] = len(pool)  # voxels outside the pool
    with pytest.raises(sb.SurfaceError):
        t.set_sparse(blocks, pool, 1, 1, gdim)



def _check_sparse(blocks, pool, fmt, comps, gdim, uvw):
    t = Texture3D()
    t.set_sparse(blocks, pool, fmt, comps, gdim)
    got = t.Fetch(torch.from_numpy(uvw).cuda()).cpu().numpy()
    want = O.sparse_fetch(blocks, pool, fmt, comps, gdim, uvw)
    assert same(got, want)
    return want


def test_sparse_pages_faces_and_widening():
    """A page checkerboard: neighbours meet at edges, so points on an edge
    or within the widening of one belong to the first page in tree order."""
    blocks, pool, gdim = S.sparse_pages(ndiv=4, page=8, seed=5)
    want = _check_sparse(blocks, pool, 0, 1, gdim, S.sparse_edge_coords(blocks, gdim, 60000, 1))
    assert (want[:, 3] != 0).mean() > 0.3


@pytest.mark.parametrize("case", S.LOCATE_CASES)
def test_sparse_locate_edge_cases(case):
    for fmt, comps in ((0, 1), (1, 3)):
        blocks, pool, gdim = S.sparse_locate_case(case, fmt, comps)
        uvw = S.sparse_edge_coords(blocks, gdim, 30000, fmt, spread=(-1.5, 1.5))
        want = _check_sparse(blocks, pool, fmt, comps, gdim, uvw)
        assert (want[:, 3] != 0).mean() > 0.2


def test_fetch_host_arrays_through_the_c_abi():
    """srt_texture3d_fetch with host coordinate and output arrays (staged by
    the library) gives the device path's result."""
    blocks, pool, gdim = S.sparse_pages(ndiv=4, page=8, seed=5)
    t = Texture3D()
    t.set_sparse(blocks, pool, 0, 1, gdim)
    uvw = S.sparse_edge_coords(blocks, gdim, 5000, 3)
    dev = t.Fetch(torch.from_numpy(uvw).cuda()).cpu().numpy()
    host = np.zeros((uvw.shape[0], 4), np.float32)
    u = np.ascontiguousarray(uvw)
    from surface_b200._lib import check
    check(t.L.srt_texture3d_fetch(t.h, u.ctypes.data, u.shape[0], host.ctypes.data))
    assert same(host, dev)
    assert same(host, O.sparse_fetch(blocks, pool, 0, 1, gdim, uvw))
