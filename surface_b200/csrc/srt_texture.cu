// srt_texture.cu -- Texture::Fetch of 3D textures on the GPU
// (gles/gles_common.h:344-399), for a whole array of coordinates.
//
// Dense textures: the per-axis coordinate remap of non-uniform volumes
// (local::remap, gles/gles_common.h:264-269, set by lsglTexCoordRemap), then
// FilterTexture3D{Byte,Float,Double} (render/render_texture.cc:832-1175):
// repeat wrap by fasterfloorf unless clamp-to-edge, vox = u * (dim - 1),
// texel-corner trilinear interpolation with the reference's Lerp (dlerp in
// double for double textures), bytes read as v / 255.5f, a single component
// replicated to rgba.
//
// Sparse volumes: position = u * globalDim, the first block that
// BVHTree::Locate reaches (render/render_bvh_tree.cc:587-655; the tree is
// built on the host like the scene's top level), then
// SparseVolumeAccel::Sample (render/render_accel_volume.cc:61-139): the
// nearest texel of the block, the local offset scaled by size/extent of x on
// all three axes as the reference does, bytes as v / 255.0f, doubles through
// float, alpha 1 below four components, (0, 0, 0, 0) outside every block.
//
// Locate is answered through a cell grid built with the tree: Locate's
// answer is the first leaf in depth-first (left first) order whose box holds
// the point, because every node's box holds its children's (the 1e-6
// widening grows with the extent).  Each cell of an integer lattice over the
// blocks keeps the first leaf whose box holds the whole cell (its owner), the
// earlier leaves that reach into the cell (tested in order) and a core box
// clear of them; a point inside the core takes the owner (or no block, in a
// cell without one) with no box test.
// Cells with more than kCellList candidates walk the tree.
//
// Float-to-int conversions follow x86 (NaN and out-of-range values give
// INT_MIN), so every coordinate gives the reference's texel.  Compiled without
// FMA contraction: each expression rounds as in the reference.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "srt_internal.cuh"

using namespace srt;

struct srt_texture3d {
  srt_ctx *ctx = nullptr;
  bool sparse = false;
  int format = 1, comps = 1;
  int dim[3] = {0, 0, 0};   // dense: width, height, depth; sparse: globalDim
  int clamp[3] = {0, 0, 0};  // clamp-to-edge per axis (else repeat)
  DevBuf data;               // dense texels or the sparse data pool
  size_t data_bytes = 0;
  DevBuf remap[3];
  uint32_t nremap[3] = {0, 0, 0};
  DevBuf tree, blocks;       // sparse: BVHTree over the blocks, block table
  uint32_t nblocks = 0, ntree = 0;
  DevBuf cells, leaves, list;  // sparse: the tree's cell grid (cells.p null: none)
  float ulo[3], uhi[3];
  int org[3], shift[3], g[3];
};

namespace srt {
namespace {

__device__ __forceinline__ int clampi(int v, int lo, int hi) {
  return min(max(v, lo), hi);
}

__device__ __forceinline__ float lerp_ref(float t, float a, float b) {
  return (1.f - t) * a + t * b;
}
__device__ __forceinline__ double dlerp_ref(double t, double a, double b) {
  return (1.0 - t) * a + t * b;
}

struct DenseTex {
  const void *data;
  const float *remap[3];
  uint32_t nremap[3];
  int dim[3], clamp[3], comps, format;
};

template <int FMT>
__device__ __forceinline__ float texel_f(const void *d, size_t k) {
  if (FMT == 0) return (float)static_cast<const unsigned char *>(d)[k] / 255.5f;
  return __ldg(&static_cast<const float *>(d)[k]);
}

template <int FMT>
__global__ void __launch_bounds__(256)
dense_fetch_kernel(DenseTex t, const float *__restrict__ uvw, size_t n,
                   float4 *__restrict__ rgba) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    float c[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
      c[k] = __ldg(&uvw[3 * i + k]);
      if (t.nremap[k]) {  // local::remap
        const int nk = (int)t.nremap[k];
        int idx = f2i_x86(c[k] * (float)nk);
        idx = max(min(nk - 1, idx), 0);
        c[k] = __ldg(&t.remap[k][idx]);
      }
      if (!t.clamp[k]) c[k] = c[k] - (float)floor_ref(c[k]);
    }
    float vox[3];
    int v0[3], v1[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
      vox[k] = c[k] * ((float)t.dim[k] - 1.0f);
      v0[k] = clampi(f2i_x86(vox[k]), 0, t.dim[k] - 1);
      v1[k] = min(v0[k] + 1, t.dim[k] - 1);
    }
    const size_t sx = (size_t)t.comps, sy = sx * t.dim[0], sz = sy * t.dim[1];
    const size_t b000 = v0[2] * sz + v0[1] * sy + v0[0] * sx;
    const size_t ox = (size_t)(v1[0] - v0[0]) * sx, oy = (size_t)(v1[1] - v0[1]) * sy,
                 oz = (size_t)(v1[2] - v0[2]) * sz;
    float vals[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    for (int ch = 0; ch < t.comps && ch < 4; ch++) {
      const size_t b = b000 + ch;
      if (FMT == 2) {
        const double *d = static_cast<const double *>(t.data);
        const double dx = (double)(vox[0] - (float)v0[0]), dy = (double)(vox[1] - (float)v0[1]),
                     dz = (double)(vox[2] - (float)v0[2]);
        const double d00 = dlerp_ref(dx, __ldg(&d[b]), __ldg(&d[b + ox]));
        const double d10 = dlerp_ref(dx, __ldg(&d[b + oy]), __ldg(&d[b + oy + ox]));
        const double d01 = dlerp_ref(dx, __ldg(&d[b + oz]), __ldg(&d[b + oz + ox]));
        const double d11 = dlerp_ref(dx, __ldg(&d[b + oz + oy]), __ldg(&d[b + oz + oy + ox]));
        const double d0 = dlerp_ref(dy, d00, d10), d1 = dlerp_ref(dy, d01, d11);
        vals[ch] = (float)dlerp_ref(dz, d0, d1);
      } else {
        const float dx = vox[0] - (float)v0[0], dy = vox[1] - (float)v0[1],
                    dz = vox[2] - (float)v0[2];
        const float d00 = lerp_ref(dx, texel_f<FMT>(t.data, b), texel_f<FMT>(t.data, b + ox));
        const float d10 =
            lerp_ref(dx, texel_f<FMT>(t.data, b + oy), texel_f<FMT>(t.data, b + oy + ox));
        const float d01 =
            lerp_ref(dx, texel_f<FMT>(t.data, b + oz), texel_f<FMT>(t.data, b + oz + ox));
        const float d11 = lerp_ref(dx, texel_f<FMT>(t.data, b + oz + oy),
                                   texel_f<FMT>(t.data, b + oz + oy + ox));
        const float d0 = lerp_ref(dy, d00, d10), d1 = lerp_ref(dy, d01, d11);
        vals[ch] = lerp_ref(dz, d0, d1);
      }
    }
    rgba[i] = (t.comps == 1) ? make_float4(vals[0], vals[0], vals[0], vals[0])
                             : make_float4(vals[0], vals[1], vals[2], vals[3]);
  }
}

// A leaf of the block tree in depth-first order: its (widened) box and block.
struct SparseLeaf {
  double bmin[3], bmax[3];
  int32_t block, pad;
};
// A block as the sample reads it: size[0] / extent[0] (the reference scales
// all three axes by x's ratio), the texels' byte offset, offset and size.
// fast != 0: size[0] == extent[0], offsets >= 0 and offset + extent <= 2^22,
// where trunc((p - offset) * 1.0) in double is floor(p) - offset for every p
// in the block (a float p below an integer k >= 1 is at least 2^-24 k away
// from it, more than the double rounding of p - offset < 2^22 can bridge).
struct alignas(16) BlockRec {
  double sx;
  uint64_t data_off;
  int32_t off[3], size0;
  int32_t size1, size2, fast, pad;
};
static_assert(sizeof(BlockRec) == 48, "three 16-byte loads");
// One lattice cell: `owner` (the block of the first leaf holding the whole
// cell, -1 if none) with its sample record, the leaves to test in order
// before the owner (with no owner: every leaf reaching into the cell), and
// the cell's open core clear of those leaves, where the answer is `owner`.
// list = first << 5 | count; count kWalk: walk the tree.
struct alignas(16) SparseCell {
  float core_lo[3];
  int32_t owner;
  float core_hi[3];
  uint32_t list;
  BlockRec rec;
};
static_assert(sizeof(SparseCell) == 80, "five 16-byte loads");
constexpr uint32_t kCellList = 16;
constexpr uint32_t kWalk = 31;

struct SparseTex {
  const TopNode *tree;
  const BlockRec *blocks;
  const unsigned char *pool;
  int gdim[3], comps, format;
  uint32_t max_iter;
  // cell grid (cells == nullptr: walk the tree for every point)
  const SparseCell *cells;
  const SparseLeaf *leaves;
  const uint32_t *list;
  float ulo[3], uhi[3];  // the union of the leaf boxes, rounded out to floats
  int org[3], shift[3], g[3];  // lattice origin, log2 cell size, cells
};

__device__ __forceinline__ bool in_box(const TopNode &t, const double p[3]) {
  return p[0] >= t.bmin[0] && p[0] <= t.bmax[0] && p[1] >= t.bmin[1] && p[1] <= t.bmax[1] &&
         p[2] >= t.bmin[2] && p[2] <= t.bmax[2];
}

// BVHTree::Locate's first leaf: depth first, the left child first.
__device__ int locate(const TopNode *__restrict__ tree, const double p[3], uint32_t max_iter,
                      uint32_t *err) {
  int stk[64];
  int sp = 0, node = 0;
  for (uint32_t g = 0; g < max_iter; g++) {
    const TopNode &t = tree[node];
    if (t.leaf) {
      if (in_box(t, p)) return (int)t.id;
      if (sp < 1) return -1;
      node = stk[--sp];
      continue;
    }
    const bool h0 = t.child[0] > 0 && in_box(tree[t.child[0]], p);
    const bool h1 = t.child[1] > 0 && in_box(tree[t.child[1]], p);
    if (!h0 && !h1) {
      if (sp < 1) return -1;
      node = stk[--sp];
    } else if (h0 && h1) {
      if (sp >= 64) {
        atomicOr(err, kErrStack);
        return -1;
      }
      stk[sp++] = t.child[1];
      node = t.child[0];
    } else {
      node = h0 ? t.child[0] : t.child[1];
    }
  }
  atomicOr(err, kErrIter);
  return -1;
}

__device__ __forceinline__ BlockRec unpack_rec(int4 a, int4 b, int4 d) {
  BlockRec r;
  r.sx = __hiloint2double(a.y, a.x);
  r.data_off = ((uint64_t)(uint32_t)a.w << 32) | (uint32_t)a.z;
  r.off[0] = b.x;
  r.off[1] = b.y;
  r.off[2] = b.z;
  r.size0 = b.w;
  r.size1 = d.x;
  r.size2 = d.y;
  r.fast = d.z;
  return r;
}

__device__ __forceinline__ BlockRec load_rec(const BlockRec *r) {
  const int4 *q = reinterpret_cast<const int4 *>(r);
  return unpack_rec(__ldg(q), __ldg(q + 1), __ldg(q + 2));
}

// The cell of p, clamped to the grid: floor((p - org) / 2^shift) is
// (floor(p) - org) >> shift for an integer origin (NaN maps to cell 0 and
// then fails the union test).
__device__ __forceinline__ size_t cell_of(const SparseTex &t, const int fl[3]) {
  int c[3];
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const long long d = ((long long)fl[k] - t.org[k]) >> t.shift[k];
    c[k] = (int)(d < 0 ? 0 : (d >= t.g[k] ? t.g[k] - 1 : d));
  }
  return ((size_t)c[2] * t.g[1] + c[1]) * t.g[0] + c[0];
}

// SparseVolumeAccel::Sample of block record r at p: the nearest texel.  The
// reference stores each component as a double and the caller reads it as a
// float, so bytes give (float)b / 255.0f (lut), floats themselves and
// doubles (float)d.
__device__ __forceinline__ float4 sample_rec(const SparseTex &t, const BlockRec &r,
                                             const float pf[3], const int fl[3],
                                             const float *lut) {
  const int size[3] = {r.size0, r.size1, r.size2};
  int ix[3];
  if (r.fast) {
#pragma unroll
    for (int k = 0; k < 3; k++) ix[k] = max(min(size[k] - 1, fl[k] - r.off[k]), 0);
  } else {
#pragma unroll
    for (int k = 0; k < 3; k++) {
      const double x = ((double)pf[k] - (double)r.off[k]) * r.sx;  // x's ratio on every axis
      ix[k] = max(min(size[k] - 1, d2i_x86(x)), 0);
    }
  }
  const size_t idx =
      ((size_t)ix[2] * size[1] + (size_t)ix[1]) * (size_t)size[0] + (size_t)ix[0];
  const unsigned char *base = t.pool + r.data_off;
  const int nc = t.comps >= 4 ? 4 : t.comps;
  float v[4] = {0.f, 0.f, 0.f, 1.f};
  for (int c = 0; c < nc; c++) {
    const size_t k = (size_t)nc * idx + c;  // the stride is the clamped count
    if (t.format == 0)
      v[c] = lut[__ldg(base + k)];
    else if (t.format == 1)
      v[c] = __ldg(reinterpret_cast<const float *>(base) + k);
    else
      v[c] = (float)__ldg(reinterpret_cast<const double *>(base) + k);
  }
  return make_float4(v[0], v[1], v[2], v[3]);
}

// One fetch through the cell grid; the block is the one locate() finds for
// every point.  The cell's first 32 bytes decide; its owner's record (the
// last 48) is read only when the point is in the owner.
__device__ __forceinline__ float4 fetch_cells(const SparseTex &t, const float pf[3],
                                              const float *lut, uint32_t *err) {
  int fl[3];
#pragma unroll
  for (int k = 0; k < 3; k++) fl[k] = __float2int_rd(pf[k]);
  const int4 *q = reinterpret_cast<const int4 *>(t.cells + cell_of(t, fl));
  const int4 c0 = __ldg(q), c1 = __ldg(q + 1);
  // outside the union of the leaf boxes: in no leaf (NaN included).  p is a
  // float, so p >= lo exactly when p >= lo rounded up to a float.
  int id = -1;
  bool own = false;
  if (pf[0] >= t.ulo[0] && pf[0] <= t.uhi[0] && pf[1] >= t.ulo[1] && pf[1] <= t.uhi[1] &&
      pf[2] >= t.ulo[2] && pf[2] <= t.uhi[2]) {
    id = c0.w;
    const bool core = pf[0] > __int_as_float(c0.x) && pf[0] < __int_as_float(c1.x) &&
                      pf[1] > __int_as_float(c0.y) && pf[1] < __int_as_float(c1.y) &&
                      pf[2] > __int_as_float(c0.z) && pf[2] < __int_as_float(c1.z);
    if (!core) {
      const uint32_t first = (uint32_t)c1.w >> 5, n = (uint32_t)c1.w & 31u;
      const double p[3] = {(double)pf[0], (double)pf[1], (double)pf[2]};
      if (n == kWalk) {
        id = locate(t.tree, p, t.max_iter, err);
      } else {
        for (uint32_t j = 0; j < n; j++) {
          const SparseLeaf &L = t.leaves[__ldg(&t.list[first + j])];
          if (p[0] >= L.bmin[0] && p[0] <= L.bmax[0] && p[1] >= L.bmin[1] &&
              p[1] <= L.bmax[1] && p[2] >= L.bmin[2] && p[2] <= L.bmax[2]) {
            id = L.block;
            break;
          }
        }
      }
    }
    own = id >= 0 && id == c0.w;  // a walking cell has no owner
  }
  if (id < 0) return make_float4(0.f, 0.f, 0.f, 0.f);
  const BlockRec r = own ? unpack_rec(__ldg(q + 2), __ldg(q + 3), __ldg(q + 4))
                         : load_rec(t.blocks + id);
  return sample_rec(t, r, pf, fl, lut);
}

// One fetch per thread per round, grid-strided (coalesced coordinates and
// RGBA).
__global__ void __launch_bounds__(256)
sparse_fetch_kernel(SparseTex t, const float *__restrict__ uvw, size_t n,
                    float4 *__restrict__ rgba, uint32_t *__restrict__ err) {
  __shared__ float lut[256];  // byte texel b -> (float)b / 255.0f
  for (int k = threadIdx.x; k < 256; k += blockDim.x) lut[k] = (float)k / 255.0f;
  __syncthreads();
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    float pf[3];
#pragma unroll
    for (int k = 0; k < 3; k++) pf[k] = __ldg(&uvw[3 * i + k]) * (float)t.gdim[k];
    float4 out;
    if (t.cells) {
      out = fetch_cells(t, pf, lut, err);
    } else {
      const double p[3] = {(double)pf[0], (double)pf[1], (double)pf[2]};
      int fl[3];
#pragma unroll
      for (int k = 0; k < 3; k++) fl[k] = __float2int_rd(pf[k]);
      const int id = locate(t.tree, p, t.max_iter, err);
      out = id >= 0 ? sample_rec(t, load_rec(t.blocks + id), pf, fl, lut)
                    : make_float4(0.f, 0.f, 0.f, 0.f);
    }
    rgba[i] = out;
  }
}

size_t format_bytes(int f) { return f == 0 ? 1 : f == 1 ? 4 : 8; }

srt_status upload(srt_ctx *ctx, DevBuf &dst, const void *src, size_t bytes) {
  cudaError_t e = dst.ensure(bytes ? bytes : 1);
  if (e == cudaSuccess && bytes)
    e = cudaMemcpyAsync(dst.p, src, bytes,
                        is_device_ptr(src) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                        ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);  // src may be freed next
  return cuda_status(e, "texture upload");
}

// The cell grid of a block tree (host).  Lattice: origin at the smallest
// block offset, per-axis cell size the power of two nearest the median block
// extent, at most 2^20 cells; built = false when the blocks would need more
// than 2^26 (leaf, cell) pairs, and every point then walks the tree.
struct CellGrid {
  bool built = false;
  std::vector<SparseCell> cells;
  std::vector<SparseLeaf> leaves;
  std::vector<uint32_t> list;
  double org[3], inv[3], ulo[3], uhi[3];
  int g[3], shift[3];
};

float round_up_f(double x) {
  float f = (float)x;
  if ((double)f < x) f = nextafterf(f, INFINITY);
  return f;
}
float round_down_f(double x) {
  float f = (float)x;
  if ((double)f > x) f = nextafterf(f, -INFINITY);
  return f;
}

void build_cell_grid(const std::vector<TopNode> &tree, const srt_volume_block *blocks,
                     const std::vector<BlockRec> &recs, size_t nblocks, CellGrid &G) {
  G = CellGrid();
  // leaves in depth-first order, left child first (Locate's visiting order)
  std::vector<int32_t> stk{0};
  while (!stk.empty()) {
    const TopNode &t = tree[stk.back()];
    stk.pop_back();
    if (t.leaf) {
      SparseLeaf L{};
      for (int k = 0; k < 3; k++) {
        L.bmin[k] = t.bmin[k];
        L.bmax[k] = t.bmax[k];
      }
      L.block = (int32_t)t.id;
      G.leaves.push_back(L);
      continue;
    }
    if (t.child[1] > 0) stk.push_back(t.child[1]);
    if (t.child[0] > 0) stk.push_back(t.child[0]);
  }
  if (G.leaves.empty()) return;
  double c[3];
  for (int k = 0; k < 3; k++) {
    int64_t lo = blocks[0].offset[k], hi = (int64_t)blocks[0].offset[k] + blocks[0].extent[k];
    std::vector<int32_t> ext(nblocks);
    for (size_t i = 0; i < nblocks; i++) {
      lo = std::min<int64_t>(lo, blocks[i].offset[k]);
      hi = std::max<int64_t>(hi, (int64_t)blocks[i].offset[k] + blocks[i].extent[k]);
      ext[i] = blocks[i].extent[k];
    }
    std::nth_element(ext.begin(), ext.begin() + nblocks / 2, ext.end());
    const int e2 = std::max(0, (int)lrint(log2((double)ext[nblocks / 2])));
    c[k] = ldexp(1.0, std::min(e2, 24));
    G.org[k] = (double)lo;
    const double span = (double)(hi - lo);
    while (ceil(span / c[k]) > 1024.0) c[k] *= 2.0;
    G.g[k] = std::max(1, (int)ceil(span / c[k]));
    G.ulo[k] = G.leaves[0].bmin[k];
    G.uhi[k] = G.leaves[0].bmax[k];
    for (const SparseLeaf &L : G.leaves) {
      G.ulo[k] = std::min(G.ulo[k], L.bmin[k]);
      G.uhi[k] = std::max(G.uhi[k], L.bmax[k]);
    }
  }
  while ((int64_t)G.g[0] * G.g[1] * G.g[2] > (1 << 20)) {
    const int k = (G.g[0] >= G.g[1] && G.g[0] >= G.g[2]) ? 0 : (G.g[1] >= G.g[2] ? 1 : 2);
    c[k] *= 2.0;
    G.g[k] = (G.g[k] + 1) / 2;
  }
  for (int k = 0; k < 3; k++) {
    G.inv[k] = 1.0 / c[k];
    G.shift[k] = ilogb(c[k]);
  }
  // the region of points mapped to cell i on axis k: the lattice interval
  // with a margin far above the rounding of the index, the outer cells out
  // to the union box
  auto cell_lo = [&](int k, int i) {
    double v = G.org[k] + i * c[k];
    v -= c[k] * 0x1p-30;
    return i == 0 ? std::min(v, G.ulo[k]) : v;
  };
  auto cell_hi = [&](int k, int i) {
    double v = G.org[k] + (i + 1) * c[k];
    v += c[k] * 0x1p-30;
    return i == G.g[k] - 1 ? std::max(v, G.uhi[k]) : v;
  };
  auto range = [&](int k, double a, double b, int &i0, int &i1) {
    i0 = (int)std::max(0.0, std::min((double)G.g[k] - 1, floor((a - G.org[k]) * G.inv[k]) - 1));
    i1 = (int)std::max(0.0, std::min((double)G.g[k] - 1, floor((b - G.org[k]) * G.inv[k]) + 1));
  };
  uint64_t pairs = 0;
  for (const SparseLeaf &L : G.leaves) {
    int r[3][2];
    for (int k = 0; k < 3; k++) range(k, L.bmin[k], L.bmax[k], r[k][0], r[k][1]);
    pairs += (uint64_t)(r[0][1] - r[0][0] + 1) * (r[1][1] - r[1][0] + 1) * (r[2][1] - r[2][0] + 1);
    if (pairs > (1ull << 26)) return;
  }
  const size_t ncell = (size_t)G.g[0] * G.g[1] * G.g[2];
  // the first kCellList + 1 leaves reaching into each cell, in order
  const uint32_t cap = kCellList + 1;
  std::vector<uint32_t> cnt(ncell, 0), cand(ncell * (size_t)cap);
  std::vector<uint8_t> more(ncell, 0);
  for (uint32_t li = 0; li < (uint32_t)G.leaves.size(); li++) {
    const SparseLeaf &L = G.leaves[li];
    int r[3][2];
    for (int k = 0; k < 3; k++) range(k, L.bmin[k], L.bmax[k], r[k][0], r[k][1]);
    for (int z = r[2][0]; z <= r[2][1]; z++)
      for (int y = r[1][0]; y <= r[1][1]; y++)
        for (int x = r[0][0]; x <= r[0][1]; x++) {
          const int ix[3] = {x, y, z};
          bool hit = true;
          for (int k = 0; k < 3 && hit; k++)
            hit = L.bmin[k] <= cell_hi(k, ix[k]) && L.bmax[k] >= cell_lo(k, ix[k]);
          if (!hit) continue;
          const size_t ci = ((size_t)z * G.g[1] + y) * G.g[0] + x;
          if (cnt[ci] < cap)
            cand[ci * cap + cnt[ci]++] = li;
          else
            more[ci] = 1;
        }
  }
  G.cells.resize(ncell);
  for (int z = 0; z < G.g[2]; z++)
    for (int y = 0; y < G.g[1]; y++)
      for (int x = 0; x < G.g[0]; x++) {
        const size_t ci = ((size_t)z * G.g[1] + y) * G.g[0] + x;
        const int ix[3] = {x, y, z};
        double lo[3], hi[3];
        for (int k = 0; k < 3; k++) {
          lo[k] = cell_lo(k, ix[k]);
          hi[k] = cell_hi(k, ix[k]);
        }
        SparseCell &C = G.cells[ci];
        C = SparseCell{};
        C.owner = -1;
        for (int k = 0; k < 3; k++) {  // an empty core until one is cut
          C.core_lo[k] = INFINITY;
          C.core_hi[k] = -INFINITY;
        }
        uint32_t own = cnt[ci];
        for (uint32_t j = 0; j < cnt[ci]; j++) {
          const SparseLeaf &L = G.leaves[cand[ci * cap + j]];
          if (L.bmin[0] <= lo[0] && L.bmax[0] >= hi[0] && L.bmin[1] <= lo[1] &&
              L.bmax[1] >= hi[1] && L.bmin[2] <= lo[2] && L.bmax[2] >= hi[2]) {
            own = j;
            break;
          }
        }
        const bool has_owner = own < cnt[ci];
        if ((has_owner ? own : cnt[ci]) > kCellList || (!has_owner && more[ci])) {
          C.list = kWalk;
          continue;
        }
        const uint32_t n = has_owner ? own : cnt[ci];
        C.list = (uint32_t)G.list.size() << 5 | n;
        for (uint32_t j = 0; j < n; j++) G.list.push_back(cand[ci * cap + j]);
        if (has_owner) {
          C.owner = G.leaves[cand[ci * cap + own]].block;
          C.rec = recs[C.owner];
        }
        // the open core: the cell cut clear of each listed leaf (those before
        // the owner; with no owner, all that reach in), on the side that keeps
        // the most of it.  A point in the core is in the owner (or in none).
        double a[3] = {lo[0], lo[1], lo[2]}, b[3] = {hi[0], hi[1], hi[2]};
        bool empty = false;
        for (uint32_t j = 0; j < n && !empty; j++) {
          const SparseLeaf &L = G.leaves[cand[ci * cap + j]];
          bool meets = true;
          for (int k = 0; k < 3; k++) meets = meets && L.bmin[k] < b[k] && L.bmax[k] > a[k];
          if (!meets) continue;
          int bk = -1, bside = 0;
          double best = -1.0;
          for (int k = 0; k < 3; k++) {
            const double w = b[k] - a[k];
            const double keep_hi = (b[k] - L.bmax[k]) / w;  // core above the leaf
            const double keep_lo = (L.bmin[k] - a[k]) / w;  // core below the leaf
            if (keep_hi > best) {
              best = keep_hi;
              bk = k;
              bside = 0;
            }
            if (keep_lo > best) {
              best = keep_lo;
              bk = k;
              bside = 1;
            }
          }
          if (best <= 0.0) {
            empty = true;
          } else if (bside == 0) {
            a[bk] = L.bmax[bk];
          } else {
            b[bk] = L.bmin[bk];
          }
        }
        if (empty) continue;
        for (int k = 0; k < 3; k++) {
          C.core_lo[k] = round_up_f(a[k]);
          C.core_hi[k] = round_down_f(b[k]);
        }
      }
  G.built = true;
}

}  // namespace
}  // namespace srt

extern "C" {

SRT_API srt_status srt_texture3d_create(srt_ctx *ctx, srt_texture3d **out) {
  if (!ctx || !out) return SRT_ERR_INVALID;
  srt_texture3d *t = new (std::nothrow) srt_texture3d();
  if (!t) return SRT_ERR_NO_MEMORY;
  t->ctx = ctx;
  *out = t;
  return SRT_OK;
}

SRT_API srt_status srt_texture3d_destroy(srt_texture3d *t) {
  if (!t) return SRT_OK;
  cudaSetDevice(t->ctx->device);
  cudaStreamSynchronize(t->ctx->stream);
  delete t;
  return SRT_OK;
}

SRT_API srt_status srt_texture3d_set_dense(srt_texture3d *t, int format, int width, int height,
                                           int depth, int components, const void *data) {
  if (!t || !data) return SRT_ERR_INVALID;
  if (format < 0 || format > 2 || components < 1 || components > 4 || width < 1 ||
      height < 1 || depth < 1) {
    set_error("srt_texture3d_set_dense: format 0..2, 1..4 components, positive size");
    return SRT_ERR_INVALID;
  }
  cudaSetDevice(t->ctx->device);
  const size_t bytes =
      (size_t)width * height * depth * components * format_bytes(format);
  srt_status s = upload(t->ctx, t->data, data, bytes);
  if (s != SRT_OK) return s;
  t->sparse = false;
  t->format = format;
  t->comps = components;
  t->dim[0] = width;
  t->dim[1] = height;
  t->dim[2] = depth;
  t->data_bytes = bytes;
  return SRT_OK;
}

SRT_API srt_status srt_texture3d_set_wrap(srt_texture3d *t, int clamp_s, int clamp_t,
                                          int clamp_r) {
  if (!t) return SRT_ERR_INVALID;
  t->clamp[0] = clamp_s != 0;
  t->clamp[1] = clamp_t != 0;
  t->clamp[2] = clamp_r != 0;
  return SRT_OK;
}

SRT_API srt_status srt_texture3d_set_remap(srt_texture3d *t, int axis, const float *table,
                                           size_t n) {
  if (!t || axis < 0 || axis > 2 || (n && !table) || n > 0x7fffffffu) {
    set_error("srt_texture3d_set_remap: axis 0..2 and a table of n < 2^31 entries");
    return SRT_ERR_INVALID;
  }
  cudaSetDevice(t->ctx->device);
  if (n) {
    srt_status s = upload(t->ctx, t->remap[axis], table, n * sizeof(float));
    if (s != SRT_OK) return s;
  }
  t->nremap[axis] = (uint32_t)n;
  return SRT_OK;
}

SRT_API srt_status srt_texture3d_set_sparse(srt_texture3d *t, int format, int components,
                                            const int global_dim[3],
                                            const srt_volume_block *blocks, size_t nblocks,
                                            const void *pool, size_t pool_bytes) {
  if (!t || !global_dim || !blocks || !nblocks || !pool) return SRT_ERR_INVALID;
  if (format < 0 || format > 2 || components < 1 || nblocks >= (1u << 30)) {
    set_error("srt_texture3d_set_sparse: format 0..2, at least one component and block");
    return SRT_ERR_INVALID;
  }
  const int nc = components >= 4 ? 4 : components;
  std::vector<double> lo(3 * nblocks), hi(3 * nblocks);
  for (size_t i = 0; i < nblocks; i++) {
    const srt_volume_block &b = blocks[i];
    uint64_t vox = (uint64_t)nc * format_bytes(format);
    for (int k = 0; k < 3; k++) {
      if (b.size[k] < 1 || b.extent[k] < 1) {
        set_error("srt_texture3d_set_sparse: block sizes and extents must be positive");
        return SRT_ERR_INVALID;
      }
      vox *= (uint64_t)b.size[k];
      lo[3 * i + k] = (double)b.offset[k];
      hi[3 * i + k] = (double)((int64_t)b.offset[k] + b.extent[k]);
    }
    if (b.data_offset > pool_bytes || vox > pool_bytes - b.data_offset ||
        (b.data_offset % format_bytes(format)) != 0) {
      set_error("srt_texture3d_set_sparse: a block's voxels lie outside the pool or misaligned");
      return SRT_ERR_INVALID;
    }
  }
  std::vector<TopNode> tree;
  build_top_tree(lo.data(), hi.data(), nblocks, tree);
  std::vector<BlockRec> recs(nblocks);
  for (size_t i = 0; i < nblocks; i++) {
    BlockRec &r = recs[i];
    r = BlockRec{};
    r.sx = (double)blocks[i].size[0] / (double)blocks[i].extent[0];
    r.data_off = blocks[i].data_offset;
    r.fast = blocks[i].size[0] == blocks[i].extent[0];
    for (int k = 0; k < 3; k++) {
      r.off[k] = blocks[i].offset[k];
      if (blocks[i].offset[k] < 0 ||
          (int64_t)blocks[i].offset[k] + blocks[i].extent[k] > (int64_t)1 << 22)
        r.fast = 0;
    }
    r.size0 = blocks[i].size[0];
    r.size1 = blocks[i].size[1];
    r.size2 = blocks[i].size[2];
  }
  CellGrid G;
  build_cell_grid(tree, blocks, recs, nblocks, G);
  cudaSetDevice(t->ctx->device);
  srt_status s = upload(t->ctx, t->data, pool, pool_bytes);
  if (s == SRT_OK) s = upload(t->ctx, t->tree, tree.data(), tree.size() * sizeof(TopNode));
  if (s == SRT_OK) s = upload(t->ctx, t->blocks, recs.data(), nblocks * sizeof(BlockRec));
  t->cells.release();
  if (s == SRT_OK && G.built) {
    s = upload(t->ctx, t->leaves, G.leaves.data(), G.leaves.size() * sizeof(SparseLeaf));
    if (s == SRT_OK)
      s = upload(t->ctx, t->list, G.list.data(), G.list.size() * sizeof(uint32_t));
    if (s == SRT_OK)
      s = upload(t->ctx, t->cells, G.cells.data(), G.cells.size() * sizeof(SparseCell));
    for (int k = 0; k < 3; k++) {
      t->org[k] = (int)G.org[k];
      t->shift[k] = G.shift[k];
      t->ulo[k] = round_up_f(G.ulo[k]);
      t->uhi[k] = round_down_f(G.uhi[k]);
      t->g[k] = G.g[k];
    }
  }
  if (s != SRT_OK) {
    t->cells.release();
    return s;
  }
  t->sparse = true;
  t->format = format;
  t->comps = components;
  for (int k = 0; k < 3; k++) t->dim[k] = global_dim[k];
  t->data_bytes = pool_bytes;
  t->nblocks = (uint32_t)nblocks;
  t->ntree = (uint32_t)tree.size();
  return SRT_OK;
}

SRT_API srt_status srt_texture3d_fetch(srt_texture3d *t, const float *uvw, size_t n,
                                       float *rgba) {
  if (!t || (n && (!uvw || !rgba))) return SRT_ERR_INVALID;
  if (!t->data.p) {
    set_error("srt_texture3d_fetch: no texture data set");
    return SRT_ERR_INVALID;
  }
  if (n == 0) return SRT_OK;
  srt_ctx *ctx = t->ctx;
  cudaSetDevice(ctx->device);
  // host arrays are staged through the context's scratch
  const bool uhost = !is_device_ptr(uvw), ohost = !is_device_ptr(rgba);
  cudaError_t se;
  if (uhost) {
    if ((se = ctx->s_stage_in.ensure(n * 12)) != cudaSuccess ||
        (se = cudaMemcpyAsync(ctx->s_stage_in.p, uvw, n * 12, cudaMemcpyHostToDevice,
                              ctx->stream)) != cudaSuccess)
      return cuda_status(se, "texture coordinates");
    uvw = ctx->s_stage_in.as<float>();
  }
  float *const user_rgba = rgba;
  if (ohost) {
    if ((se = ctx->s_stage_out.ensure(n * 16)) != cudaSuccess)
      return cuda_status(se, "texture output");
    rgba = ctx->s_stage_out.as<float>();
  }
  if (reinterpret_cast<uintptr_t>(rgba) & 15u) {
    set_error("srt_texture3d_fetch: device rgba must be 16-byte aligned");
    return SRT_ERR_INVALID;
  }
  const unsigned grid = (unsigned)std::min<size_t>((n + 255) / 256, (size_t)ctx->num_sms * 16);
  float4 *out = reinterpret_cast<float4 *>(rgba);
  if (t->sparse) {
    SparseTex st;
    st.tree = t->tree.as<TopNode>();
    st.blocks = t->blocks.as<BlockRec>();
    st.pool = t->data.as<unsigned char>();
    for (int k = 0; k < 3; k++) st.gdim[k] = t->dim[k];
    st.comps = t->comps;
    st.format = t->format;
    st.max_iter = 4 * t->ntree + 8;
    st.cells = t->cells.as<SparseCell>();
    st.leaves = t->leaves.as<SparseLeaf>();
    st.list = t->list.as<uint32_t>();
    for (int k = 0; k < 3; k++) {
      st.org[k] = t->org[k];
      st.shift[k] = t->shift[k];
      st.ulo[k] = t->ulo[k];
      st.uhi[k] = t->uhi[k];
      st.g[k] = t->g[k];
    }
    sparse_fetch_kernel<<<grid, 256, 0, ctx->stream>>>(st, uvw, n, out, ctx->d_err);
  } else {
    DenseTex dt;
    dt.data = t->data.p;
    for (int k = 0; k < 3; k++) {
      dt.remap[k] = t->remap[k].as<float>();
      dt.nremap[k] = t->nremap[k];
      dt.dim[k] = t->dim[k];
      dt.clamp[k] = t->clamp[k];
    }
    dt.comps = t->comps;
    dt.format = t->format;
    if (t->format == 0)
      dense_fetch_kernel<0><<<grid, 256, 0, ctx->stream>>>(dt, uvw, n, out);
    else if (t->format == 1)
      dense_fetch_kernel<1><<<grid, 256, 0, ctx->stream>>>(dt, uvw, n, out);
    else
      dense_fetch_kernel<2><<<grid, 256, 0, ctx->stream>>>(dt, uvw, n, out);
  }
  ctx->launches++;
  if ((se = cudaGetLastError()) != cudaSuccess) return cuda_status(se, "texture fetch");
  if (ohost &&
      (se = cudaMemcpyAsync(user_rgba, rgba, n * 16, cudaMemcpyDeviceToHost, ctx->stream)) !=
          cudaSuccess)
    return cuda_status(se, "texture output");
  // a host-staged call waits anyway: report the sparse walk's cap flag here
  if (uhost || ohost) return check_device_errors(ctx);
  return SRT_OK;
}

}  // extern "C"
