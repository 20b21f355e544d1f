// srt_line.cu -- LineAccel (render/render_accel_line.cc) on the GPU: capped
// cylinders between segment end points, closest hit.
//
// Build (LineAccel::BuildTree, :167-296) on the GPU, level by level: the
// reference's tree exactly -- a leaf below min_leaf lines or at max_depth,
// else a cut at the spatial median of the node box's longest axis (the
// position formed in double and stored as float), then the other axes in
// turn, with the order std::partition's two-ended scan leaves on the
// segment midpoints, and the object median when no axis separates them.
// Nodes are laid out in pre-order; the device copy packs each into 32
// bytes.  The lines are gathered in leaf order into 64-byte records holding
// the per-line terms of CylinderIsect (end points, max radius, |d|^2, the
// cap plane normal and offsets), computed with the reference's float
// operations.
//
// Trace (LineAccel::Traverse, :704-774): one thread per ray (in a Morton
// order of the rays for large batches), the stack of
// the reference (a popped branch tests its own box against the closest hit
// so far, then pushes far and near children by the sign of the ray's
// direction on the branch's axis), every line of a popped leaf tested in
// order by CylinderIsect (:488-577).  Compiled without FMA contraction; the
// reference's unqualified sqrt and fabs are the double C functions, so the
// quadratic's first root is formed in double, and every other sqrt and
// reciprocal rounds as the float operation does.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "srt_internal.cuh"
#include "srt_walks.cuh"

namespace {

using namespace srt_line_walk;

// The reference's LineNode (Dump record, 40 bytes).
struct LineNodeH {
  float bmin[3], bmax[3];
  int32_t flag, axis;  // flag 1: leaf (data = count, first), 0: branch (children)
  uint32_t data[2];
};
static_assert(sizeof(LineNodeH) == 40, "LineNode layout");

}  // namespace

struct srt_line_accel {
  srt_ctx *ctx = nullptr;
  bool built = false;
  size_t nlines = 0, nnodes = 0;
  int depth = 0, cap = 1;
  LineNodeH root{};              // the root record (BoundingBox)
  srt::DevBuf dref, didx;        // reference layout (Dump, export) and the line order
  bool host_ready = false;       // host copies below filled from dref / didx
  std::vector<LineNodeH> nodes;
  std::vector<uint32_t> idx;
  srt::DevBuf dnodes, drecs;
  // build scratch, kept between builds (grown by doubling)
  srt::DevBuf s_lbox, s_mid, s_node_of, s_pairs, s_bsum, s_level, s_nchild, s_cbase, s_bfs,
      s_sizes, s_pre, s_cnt;
};

namespace {

using srt::DevBuf;

// ------------------------------------------------------------------ build
// The tree is built breadth first, one level per round of launches, and
// is then laid out in the reference's pre-order.  Per level, with the
// level's nodes numbered v = 0..m-1 in order of their ranges and
// node_of[p] naming the node that holds order position p:
//   box    min / max of the lines' boxes over each node's range.  The
//          reference folds `(a < b) ? a : b` left to right, which keeps the
//          LAST of equal values (-0 and +0 compare equal); the fold is
//          associative when its operands keep their order, so each
//          coordinate is reduced as a 64-bit key (value order << 32 | the
//          position, reversed for the minimum) and the winning position's
//          own float is read back.  NaN coordinates are rejected.
//   cut    leaf below min_leaf lines or at max_depth; else the spatial
//          median of each axis, the count T_a of midpoints below it per
//          axis, and the first axis (longest first) with 0 < T_a < n;
//          none: the object median, no reordering (a failed partition
//          moves nothing).
//   swap   std::partition's two-ended scan on [lo, hi) with T trues swaps
//          the j-th false of [lo, lo+T) (from the left) with the j-th true
//          of [lo+T, hi) (from the right), and moves nothing else.  A
//          prefix sum over the flags (false left of the split, true right
//          of it) lists each node's flagged positions in order, lefts then
//          rights; the j-th from the front pairs with the j-th from the
//          back.
//   next   children ranges [lo, split) and [split, hi), numbered by a
//          prefix sum over the splitting nodes.
constexpr uint32_t kLDone = 0xffffffffu;
constexpr int kLChunk = 16;       // order positions per thread in the reductions
constexpr int kLThreads = 256;
constexpr int kLItems = 8;        // positions per thread in the prefix sums
constexpr int kLTile = kLThreads * kLItems;
constexpr uint32_t kLErrVertex = 1u, kLErrNaN = 2u;

struct LBNode {  // a node of the breadth-first build
  float bmin[3], bmax[3];
  uint32_t lo, hi;  // its range of the line order
  uint32_t child;   // breadth-first index of the left child (right: + 1) or kLDone
  uint32_t axis;
};

struct LLevel {  // per node of the level being split
  unsigned long long kmin[3], kmax[3];
  uint32_t cnt[3];
  float pos[3];
  uint32_t lo, hi, split, longest, axis;
  uint32_t state;     // 0 leaf, 1 spatial split (swaps), 2 object median
  uint32_t beg, end;  // the node's run of flagged positions
};

__device__ __forceinline__ uint32_t ford(float x) {
  uint32_t u = __float_as_uint(x);
  if (x == 0.0f) u = 0u;
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

// GetBoundingBoxOfLine (:83-116) and the segment midpoint of PartPred.
__global__ void line_prep_kernel(const float *__restrict__ pos, const float *__restrict__ rad,
                                 float constr, const uint32_t *__restrict__ seg, size_t nverts,
                                 size_t n, float *__restrict__ lbox, float *__restrict__ mid,
                                 uint32_t *__restrict__ idx, uint32_t *__restrict__ node_of,
                                 uint32_t *__restrict__ err) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    idx[i] = (uint32_t)i;
    node_of[i] = 0u;
    const uint32_t a = seg[2 * i], b = seg[2 * i + 1];
    if (a >= nverts || b >= nverts) {
      atomicOr(err, kLErrVertex);
      for (int k = 0; k < 6; k++) lbox[6 * i + k] = 0.0f;
      for (int k = 0; k < 3; k++) mid[3 * i + k] = 0.0f;
      continue;
    }
    const float r0 = rad ? rad[a] : constr, r1 = rad ? rad[b] : constr;
    bool bad = false;
    for (int k = 0; k < 3; k++) {
      const float pa = pos[3 * a + k], pb = pos[3 * b + k];
      const float q0 = pa - r0, q1 = pa + r0, q2 = pb - r1, q3 = pb + r1;
      float lo = q0, hi = q0;
      lo = (lo < q1) ? lo : q1;
      hi = (hi > q1) ? hi : q1;
      lo = (lo < q2) ? lo : q2;
      hi = (hi > q2) ? hi : q2;
      lo = (lo < q3) ? lo : q3;
      hi = (hi > q3) ? hi : q3;
      const float eps = FLT_EPSILON * 16.0f;
      lo -= lo * eps;
      hi += hi * eps;
      bad |= (lo != lo) || (hi != hi);
      lbox[6 * i + k] = lo;
      lbox[6 * i + 3 + k] = hi;
      mid[3 * i + k] = (pa + pb) * 0.5f;
    }
    if (bad) atomicOr(err, kLErrNaN);
  }
}

__global__ void lvl_init_kernel(LLevel *__restrict__ L, uint32_t m) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < m; v += gridDim.x * blockDim.x) {
    for (int k = 0; k < 3; k++) {
      L[v].kmin[k] = ~0ull;
      L[v].kmax[k] = 0ull;
      L[v].cnt[k] = 0u;
    }
  }
}

// ComputeBoundingBox (:142-163) of every node of the level: each thread
// folds kLChunk consecutive positions, flushing a node's keys when the node
// changes; a warp whose threads end in one node reduces before the flush.
__global__ void __launch_bounds__(kLThreads)
lvl_box_kernel(const uint32_t *__restrict__ node_of, const uint32_t *__restrict__ idx,
               const float *__restrict__ lbox, size_t n, LLevel *__restrict__ L) {
  const size_t p0 = (blockIdx.x * (size_t)blockDim.x + threadIdx.x) * kLChunk;
  uint32_t cur = kLDone;
  unsigned long long mn[3], mx[3];
  auto flush = [&](uint32_t v) {
    for (int k = 0; k < 3; k++) {
      atomicMin(&L[v].kmin[k], mn[k]);
      atomicMax(&L[v].kmax[k], mx[k]);
    }
  };
  for (int j = 0; j < kLChunk; j++) {
    const size_t p = p0 + j;
    if (p >= n) break;
    const uint32_t v = node_of[p];
    if (v != cur) {
      if (cur != kLDone) flush(cur);
      cur = v;
      for (int k = 0; k < 3; k++) {
        mn[k] = ~0ull;
        mx[k] = 0ull;
      }
    }
    if (v == kLDone) continue;
    const float *b = lbox + 6 * (size_t)idx[p];
    for (int k = 0; k < 3; k++) {
      const unsigned long long a = ((unsigned long long)ford(b[k]) << 32) | (0xffffffffu - (uint32_t)p);
      const unsigned long long z = ((unsigned long long)ford(b[3 + k]) << 32) | (uint32_t)p;
      mn[k] = a < mn[k] ? a : mn[k];
      mx[k] = z > mx[k] ? z : mx[k];
    }
  }
  const uint32_t c0 = __shfl_sync(0xffffffffu, cur, 0);
  if (__all_sync(0xffffffffu, cur == c0)) {
    if (c0 == kLDone) return;
    for (int o = 16; o > 0; o >>= 1)
      for (int k = 0; k < 3; k++) {
        const unsigned long long a = __shfl_xor_sync(0xffffffffu, mn[k], o);
        const unsigned long long z = __shfl_xor_sync(0xffffffffu, mx[k], o);
        mn[k] = a < mn[k] ? a : mn[k];
        mx[k] = z > mx[k] ? z : mx[k];
      }
    if ((threadIdx.x & 31u) == 0) flush(c0);
  } else if (cur != kLDone) {
    flush(cur);
  }
}

// The node's box (the winning positions' own floats; an empty range has
// the box of the line at its start, as the reference's fold reads it),
// the leaf rule and the spatial medians of LineAccel::BuildTree.
__global__ void lvl_node_kernel(LBNode *__restrict__ nodes, uint32_t off, uint32_t m,
                                LLevel *__restrict__ L, const float *__restrict__ lbox,
                                const uint32_t *__restrict__ idx, size_t n, int depth,
                                int min_leaf, int max_depth) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < m; v += gridDim.x * blockDim.x) {
    LBNode &nd = nodes[off + v];
    LLevel &q = L[v];
    const uint32_t lo = nd.lo, hi = nd.hi;
    float bmin[3], bmax[3];
    for (int k = 0; k < 3; k++) {
      if (lo == hi) {
        const float *b = lbox + 6 * (size_t)idx[lo < n ? lo : n - 1];
        bmin[k] = b[k];
        bmax[k] = b[3 + k];
      } else {
        const uint32_t pa = 0xffffffffu - (uint32_t)q.kmin[k], pz = (uint32_t)q.kmax[k];
        bmin[k] = lbox[6 * (size_t)idx[pa] + k];
        bmax[k] = lbox[6 * (size_t)idx[pz] + 3 + k];
      }
      nd.bmin[k] = bmin[k];
      nd.bmax[k] = bmax[k];
    }
    nd.child = kLDone;
    nd.axis = 0u;
    q.lo = lo;
    q.hi = hi;
    if (hi - lo < (uint32_t)min_leaf || depth >= max_depth) {
      q.state = 0u;
      continue;
    }
    q.state = 1u;
    float bsize[3];
    for (int k = 0; k < 3; k++) bsize[k] = bmax[k] - bmin[k];
    uint32_t longest = 0;
    float mm = bsize[0];
    if (mm < bsize[1]) {
      mm = bsize[1];
      longest = 1;
    }
    if (mm < bsize[2]) longest = 2;
    q.longest = longest;
    for (int k = 0; k < 3; k++) q.pos[k] = (float)((double)bmin[k] + 0.5 * (double)bsize[k]);
  }
}

// Per splitting node and axis, the lines whose midpoint lies below the median.
__global__ void __launch_bounds__(kLThreads)
lvl_count_kernel(const uint32_t *__restrict__ node_of, const uint32_t *__restrict__ idx,
                 const float *__restrict__ mid, size_t n, LLevel *__restrict__ L) {
  const size_t p0 = (blockIdx.x * (size_t)blockDim.x + threadIdx.x) * kLChunk;
  uint32_t cur = kLDone, c[3] = {0u, 0u, 0u};
  float ps[3] = {0.0f, 0.0f, 0.0f};
  bool live = false;
  for (int j = 0; j < kLChunk; j++) {
    const size_t p = p0 + j;
    if (p >= n) break;
    const uint32_t v = node_of[p];
    if (v != cur) {
      if (live)
        for (int k = 0; k < 3; k++) atomicAdd(&L[cur].cnt[k], c[k]);
      cur = v;
      live = v != kLDone && L[v].state != 0u;
      for (int k = 0; k < 3; k++) {
        c[k] = 0u;
        if (live) ps[k] = L[v].pos[k];
      }
    }
    if (!live) continue;
    const float *d = mid + 3 * (size_t)idx[p];
    for (int k = 0; k < 3; k++) c[k] += d[k] < ps[k] ? 1u : 0u;
  }
  const uint32_t c0 = __shfl_sync(0xffffffffu, cur, 0);
  const bool l0 = __shfl_sync(0xffffffffu, live, 0);
  if (__all_sync(0xffffffffu, cur == c0)) {
    if (!l0) return;
    for (int o = 16; o > 0; o >>= 1)
      for (int k = 0; k < 3; k++) c[k] += __shfl_xor_sync(0xffffffffu, c[k], o);
    if ((threadIdx.x & 31u) == 0)
      for (int k = 0; k < 3; k++) atomicAdd(&L[c0].cnt[k], c[k]);
  } else if (live) {
    for (int k = 0; k < 3; k++) atomicAdd(&L[cur].cnt[k], c[k]);
  }
}

// The cut: the first axis, longest first, whose partition separates the
// lines (split = lo + T_a), else the object median on the last axis tried.
__global__ void lvl_split_kernel(LBNode *__restrict__ nodes, uint32_t off, uint32_t m,
                                 LLevel *__restrict__ L, uint32_t *__restrict__ nchild) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < m; v += gridDim.x * blockDim.x) {
    LLevel &q = L[v];
    if (q.state == 0u) {
      nchild[v] = 0u;
      continue;
    }
    uint32_t axis = 0, split = q.lo;
    bool found = false;
    for (uint32_t t = 0; t < 3 && !found; t++) {
      axis = (q.longest + t) % 3u;
      split = q.lo + q.cnt[axis];
      found = split != q.lo && split != q.hi;
    }
    if (!found) {
      split = q.lo + ((q.hi - q.lo) >> 1);
      q.state = 2u;
    }
    q.axis = axis;
    q.split = split;
    nodes[off + v].axis = axis;
    nchild[v] = 2u;
  }
}

// Flag of position p: a line on the wrong side of its node's split.
struct PairFlag {
  const uint32_t *node_of, *idx;
  const float *mid;
  const LLevel *L;
  __device__ __forceinline__ uint32_t operator()(size_t p) const {
    const uint32_t v = node_of[p];
    if (v == kLDone) return 0u;
    const LLevel &q = L[v];
    if (q.state != 1u) return 0u;
    const bool below = mid[3 * (size_t)idx[p] + q.axis] < q.pos[q.axis];
    return ((uint32_t)p < q.split) ? (below ? 0u : 1u) : (below ? 1u : 0u);
  }
};
struct PairOut {
  const uint32_t *node_of;
  LLevel *L;
  uint32_t *P;
  __device__ __forceinline__ void operator()(size_t p, uint32_t excl, uint32_t f) const {
    if (f) P[excl] = (uint32_t)p;
    const uint32_t v = node_of[p];
    if (v == kLDone) return;
    LLevel &q = L[v];
    if (q.state != 1u) return;
    if ((uint32_t)p == q.lo) q.beg = excl;
    if ((uint32_t)p + 1u == q.hi) q.end = excl + f;
  }
};
struct ChildFlag {
  const uint32_t *nchild;
  __device__ __forceinline__ uint32_t operator()(size_t v) const { return nchild[v]; }
};
struct ChildOut {
  uint32_t *cbase;
  __device__ __forceinline__ void operator()(size_t v, uint32_t excl, uint32_t) const {
    cbase[v] = excl;
  }
};

__device__ __forceinline__ uint32_t block_excl_scan(uint32_t x, uint32_t *ws, uint32_t &total) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  uint32_t s = x;
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
    if (lane >= o) s += y;
  }
  if (lane == 31) ws[w] = s;
  __syncthreads();
  if (w == 0) {
    const int nw = blockDim.x >> 5;
    uint32_t t = lane < nw ? ws[lane] : 0u;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += y;
    }
    if (lane < nw) ws[lane] = t;
  }
  __syncthreads();
  total = ws[(blockDim.x >> 5) - 1];
  const uint32_t before = w ? ws[w - 1] : 0u;
  __syncthreads();
  return before + s - x;
}

// Prefix sums over n flags in tiles of kLTile: the tiles' sums, their
// exclusive scan (one block), then each tile's scan with its offset.
template <class F>
__global__ void __launch_bounds__(kLThreads) lscan_count_kernel(F f, size_t n, uint32_t *bsum) {
  __shared__ uint32_t ws[32];
  const size_t base = (size_t)blockIdx.x * kLTile;
  uint32_t s = 0;
  for (int j = threadIdx.x; j < kLTile; j += kLThreads)
    if (base + j < n) s += f(base + j);
  uint32_t tot;
  block_excl_scan(s, ws, tot);
  if (threadIdx.x == 0) bsum[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(1024) lscan_top_kernel(uint32_t *bsum, uint32_t nb,
                                                         uint32_t *total) {
  __shared__ uint32_t ws[32];
  uint32_t carry = 0;
  for (uint32_t b0 = 0; b0 < nb; b0 += 1024) {
    const uint32_t i = b0 + threadIdx.x;
    const uint32_t x = i < nb ? bsum[i] : 0u;
    uint32_t tot;
    const uint32_t e = block_excl_scan(x, ws, tot);
    if (i < nb) bsum[i] = carry + e;
    carry += tot;
  }
  if (threadIdx.x == 0) *total = carry;
}

template <class F, class O>
__global__ void __launch_bounds__(kLThreads)
lscan_apply_kernel(F f, O out, size_t n, const uint32_t *__restrict__ bsum) {
  __shared__ uint32_t ws[32];
  const size_t base = (size_t)blockIdx.x * kLTile + (size_t)threadIdx.x * kLItems;
  uint32_t fl[kLItems], s = 0;
  for (int j = 0; j < kLItems; j++) {
    fl[j] = base + j < n ? f(base + j) : 0u;
    s += fl[j];
  }
  uint32_t tot;
  uint32_t e = bsum[blockIdx.x] + block_excl_scan(s, ws, tot);
  for (int j = 0; j < kLItems; j++) {
    if (base + j < n) out(base + j, e, fl[j]);
    e += fl[j];
  }
}

// The two-ended swaps: flagged position c of a node's run [beg, end) in
// the run's front half trades lines with its mirror beg + end - 1 - c.
__global__ void lvl_swap_kernel(const uint32_t *__restrict__ P, const uint32_t *__restrict__ total,
                                const uint32_t *__restrict__ node_of,
                                const LLevel *__restrict__ L, uint32_t *__restrict__ idx) {
  const uint32_t cnt = *total;
  for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < cnt; c += gridDim.x * blockDim.x) {
    const uint32_t p = P[c];
    const LLevel &q = L[node_of[p]];
    if (c - q.beg >= (q.end - q.beg) >> 1) continue;
    const uint32_t r = P[q.beg + q.end - 1u - c];
    const uint32_t x = idx[p];
    idx[p] = idx[r];
    idx[r] = x;
  }
}

__global__ void lvl_children_kernel(LBNode *__restrict__ nodes, uint32_t off, uint32_t m,
                                    const LLevel *__restrict__ L,
                                    const uint32_t *__restrict__ cbase) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < m; v += gridDim.x * blockDim.x) {
    const LLevel &q = L[v];
    if (q.state == 0u) continue;
    const uint32_t c = off + m + cbase[v];
    nodes[off + v].child = c;
    nodes[c].lo = q.lo;
    nodes[c].hi = q.split;
    nodes[c + 1].lo = q.split;
    nodes[c + 1].hi = q.hi;
  }
}

__global__ void lvl_next_kernel(uint32_t *__restrict__ node_of, const LLevel *__restrict__ L,
                                const uint32_t *__restrict__ cbase, size_t n) {
  for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n;
       p += (size_t)gridDim.x * blockDim.x) {
    const uint32_t v = node_of[p];
    if (v == kLDone) continue;
    const LLevel &q = L[v];
    node_of[p] = q.state == 0u ? kLDone : cbase[v] + ((uint32_t)p >= q.split ? 1u : 0u);
  }
}

// Pre-order layout: subtree sizes bottom up, then positions top down, each
// node written (reference record and 32-byte device record) once its
// position and its children's are known.
__global__ void lvl_size_kernel(const LBNode *__restrict__ nodes, uint32_t off, uint32_t m,
                                uint32_t *__restrict__ size) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < m; v += gridDim.x * blockDim.x) {
    const uint32_t g = off + v, c = nodes[g].child;
    size[g] = 1u + (c == kLDone ? 0u : size[c] + size[c + 1]);
  }
}

__global__ void lvl_emit_kernel(const LBNode *__restrict__ nodes, uint32_t off, uint32_t m,
                                const uint32_t *__restrict__ size, uint32_t *__restrict__ pre,
                                LineNodeH *__restrict__ ref, LNode *__restrict__ dev) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < m; v += gridDim.x * blockDim.x) {
    const uint32_t g = off + v;
    const LBNode nd = nodes[g];
    const uint32_t pv = g == 0 ? 0u : pre[g];
    LineNodeH h;
    LNode d;
    for (int k = 0; k < 3; k++) {
      h.bmin[k] = d.bmin[k] = nd.bmin[k];
      h.bmax[k] = d.bmax[k] = nd.bmax[k];
    }
    if (nd.child == kLDone) {
      h.flag = 1;
      h.axis = 0;
      h.data[0] = nd.hi - nd.lo;
      h.data[1] = nd.lo;
      d.w0 = nd.lo;
      d.w1 = kLineLeaf | (nd.hi - nd.lo);
    } else {
      const uint32_t l = pv + 1u, r = pv + 1u + size[nd.child];
      pre[nd.child] = l;
      pre[nd.child + 1] = r;
      h.flag = 0;
      h.axis = (int32_t)nd.axis;
      h.data[0] = l;
      h.data[1] = r;
      d.w0 = l;
      d.w1 = r | (nd.axis << 29);
    }
    ref[pv] = h;
    dev[pv] = d;
  }
}

// ------------------------------------------------------------------ device
__global__ void line_rec_kernel(const float *__restrict__ pos, const float *__restrict__ rad,
                                float constr, const uint32_t *__restrict__ seg,
                                const uint32_t *__restrict__ order, size_t n,
                                LineRec *__restrict__ out) {
  for (size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x; j < n;
       j += (size_t)gridDim.x * blockDim.x) {
    const uint32_t i = order[j];
    const uint32_t a = seg[2 * i], b = seg[2 * i + 1];
    LineRec r;
    float e[3], d[3], dn1[3];
    for (int k = 0; k < 3; k++) {
      r.p0[k] = pos[3 * a + k];
      r.p1[k] = pos[3 * b + k];
      e[k] = r.p0[k] - r.p1[k];
      d[k] = r.p1[k] - r.p0[k];
    }
    const float r0 = rad ? rad[a] : constr, r1 = rad ? rad[b] : constr;
    r.rr = (r0 < r1) ? r1 : r0;  // std::max<real>(r0, r1)
    r.dd = dot3(d, d);
    normalize3(e, r.dn0);
    for (int k = 0; k < 3; k++) dn1[k] = -r.dn0[k];
    r.p0D = -dot3(r.p0, r.dn0);
    r.p1D = -dot3(r.p1, dn1);
    r.prim = i;
    r.pad[0] = r.pad[1] = 0.0f;
    out[j] = r;
  }
}

// One thread per ray (grid-strided).  order (may be null): thread k traces
// ray order[k].  STATS: count popped branches, popped leaves and line tests
// into stats[0..2].
template <int STACK, bool STATS>
__global__ void __launch_bounds__(128)
line_trace_kernel(const LNode *__restrict__ nodes, const LineRec *__restrict__ recs, bool cap,
                  const srt_ray *__restrict__ rays, const uint32_t *__restrict__ order,
                  size_t n, srt_hit *__restrict__ hits, float *__restrict__ normals,
                  unsigned long long *__restrict__ stats) {
  unsigned long long nb = 0, nl = 0, nt = 0;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
       k += (size_t)gridDim.x * blockDim.x) {
    const size_t i = order ? (size_t)__ldg(&order[k]) : k;
    const float4 *rq = reinterpret_cast<const float4 *>(rays + i);
    const float4 r0 = __ldg(rq), r1 = __ldg(rq + 1);
    const float ro[3] = {r0.x, r0.y, r0.z}, rdir[3] = {r1.x, r1.y, r1.z};
    const RayL R = make_ray(ro, rdir);
    const LineHit H = line_walk<STACK, STATS>(nodes, recs, cap, R, nb, nl, nt);
    const float it = H.t, iu = H.u, iv = H.v;
    const bool icap = H.cap;
    const int best = H.rec;
    srt_hit h;
    if (it < FLT_MAX) {
      const LineRec L = load_line(recs + best);
      h.t = it;
      h.u = iu;
      h.v = iv;
      h.prim = L.prim;
      if (normals) {
        // BuildIntersection (:654-701)
        float p[3], d[3], nrm[3], e[3];
        for (int k = 0; k < 3; k++) {
          p[k] = R.org[k] + it * R.dir[k];
          d[k] = L.p1[k] - L.p0[k];
        }
        if (icap) {
          normalize3(d, nrm);
          for (int k = 0; k < 3; k++) e[k] = p[k] - (d[k] * 0.5f + L.p0[k]);
          if (!(dot3(e, nrm) > 0.0f))
            for (int k = 0; k < 3; k++) nrm[k] = -nrm[k];
        } else {
          for (int k = 0; k < 3; k++) e[k] = p[k] - (L.p0[k] + iv * d[k]);
          normalize3(e, nrm);
        }
        for (int k = 0; k < 3; k++) normals[3 * i + k] = nrm[k];
      }
    } else {
      h.t = FLT_MAX;
      h.u = h.v = 0.0f;
      h.prim = SRT_MISS;
      if (normals)
        for (int k = 0; k < 3; k++) normals[3 * i + k] = 0.0f;
    }
    reinterpret_cast<float4 *>(hits)[i] = make_float4(h.t, h.u, h.v, __uint_as_float(h.prim));
  }
  if (STATS) {
    for (int o = 16; o > 0; o >>= 1) {
      nb += __shfl_xor_sync(0xffffffffu, nb, o);
      nl += __shfl_xor_sync(0xffffffffu, nl, o);
      nt += __shfl_xor_sync(0xffffffffu, nt, o);
    }
    if ((threadIdx.x & 31) == 0) {
      atomicAdd(&stats[0], nb);
      atomicAdd(&stats[1], nl);
      atomicAdd(&stats[2], nt);
    }
  }
}

srt_status line_view(srt_ctx *ctx, const void *p, size_t bytes, DevBuf &stage,
                     const void **out) {
  if (!p || srt::is_device_ptr(p)) {
    *out = p;
    return SRT_OK;
  }
  cudaError_t e = stage.ensure(bytes ? bytes : 1);
  if (e == cudaSuccess && bytes)
    e = cudaMemcpyAsync(stage.p, p, bytes, cudaMemcpyHostToDevice, ctx->stream);
  if (e != cudaSuccess) return srt::cuda_status(e, "line staging");
  *out = stage.p;
  return SRT_OK;
}

}  // namespace

namespace srt {
uint64_t line_accel_bytes(const srt_line_accel *a) {
  return a->dnodes.cap + a->drecs.cap + a->dref.cap + a->didx.cap;
}
bool line_scene_view(const srt_line_accel *a, srt_ctx **ctx, SceneElem &e, int &depth) {
  if (!a || !a->built) return false;
  *ctx = a->ctx;
  e.kind = kSceneLines;
  e.nprims = (uint32_t)a->nlines;
  e.aux = a->cap;
  e.nodes = a->dnodes.p;
  e.prims = a->drecs.as<float4>();
  e.sidx = nullptr;
  e.scene = nullptr;
  depth = a->depth;
  return true;
}
}  // namespace srt

using namespace srt;

namespace {
// Host copies of the reference-layout nodes and the line order, fetched
// once per build for Dump and export.
srt_status line_host(srt_line_accel *a) {
  if (a->host_ready) return SRT_OK;
  cudaSetDevice(a->ctx->device);
  a->nodes.resize(a->nnodes);
  a->idx.resize(a->nlines);
  cudaStream_t st = a->ctx->stream;
  cudaError_t e = cudaMemcpyAsync(a->nodes.data(), a->dref.p, a->nnodes * sizeof(LineNodeH),
                                  cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(a->idx.data(), a->didx.p, a->nlines * 4, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_status(e, "line accel export");
  a->host_ready = true;
  return SRT_OK;
}
}  // namespace

extern "C" {

SRT_API srt_status srt_line_create(srt_ctx *ctx, srt_line_accel **out) {
  if (!ctx || !out) return SRT_ERR_INVALID;
  srt_line_accel *a = new (std::nothrow) srt_line_accel();
  if (!a) return SRT_ERR_NO_MEMORY;
  a->ctx = ctx;
  *out = a;
  return SRT_OK;
}

SRT_API srt_status srt_line_destroy(srt_line_accel *a) {
  if (!a) return SRT_OK;
  cudaSetDevice(a->ctx->device);
  cudaStreamSynchronize(a->ctx->stream);
  delete a;
  return SRT_OK;
}

SRT_API srt_status srt_line_build(srt_line_accel *a, const float *positions, size_t nverts,
                                  const float *radius, float constant_radius,
                                  const uint32_t *segments, size_t nlines, int32_t min_leaf,
                                  int32_t max_depth, int32_t cap) {
  if (!a || !positions || !segments || nlines == 0 || nverts == 0) {
    set_error("srt_line_build: positions, segments and at least one line");
    return SRT_ERR_INVALID;
  }
  if (nlines >= (1u << 31)) {
    set_error("srt_line_build: fewer than 2^31 lines");
    return SRT_ERR_INVALID;
  }
  if (min_leaf <= 0) min_leaf = 4;    // LineBuildOptions defaults
  if (max_depth <= 0) max_depth = 512;
  if (max_depth > 512) {
    set_error("srt_line_build: max_depth above 512 (the traversal stack)");
    return SRT_ERR_INVALID;
  }
  srt_ctx *ctx = a->ctx;
  cudaSetDevice(ctx->device);
  cudaStream_t st = ctx->stream;
  a->built = false;
  a->host_ready = false;
  srt_status s;
  DevBuf sp, sr, ss;
  const void *dp, *dr, *ds;
  if ((s = line_view(ctx, positions, nverts * 12, sp, &dp)) != SRT_OK) return s;
  if ((s = line_view(ctx, radius, radius ? nverts * 4 : 0, sr, &dr)) != SRT_OK) return s;
  if ((s = line_view(ctx, segments, nlines * 8, ss, &ds)) != SRT_OK) return s;
  const size_t n = nlines;
  DevBuf &lbox = a->s_lbox, &mid = a->s_mid, &node_of = a->s_node_of, &pairs = a->s_pairs,
         &bsum = a->s_bsum, &level = a->s_level, &nchild = a->s_nchild, &cbase = a->s_cbase,
         &bfs = a->s_bfs, &sizes = a->s_sizes, &pre = a->s_pre, &cnt = a->s_cnt;
  // scratch grows by doubling, so a deepening build reallocates rarely
  auto grow = [](DevBuf &b, size_t bytes) {
    return b.cap >= bytes ? cudaSuccess : b.ensure(std::max(bytes, 2 * b.cap));
  };
  const unsigned tiles = (unsigned)((n + kLTile - 1) / kLTile);
  cudaError_t e;
  if ((e = grow(lbox, n * 24)) != cudaSuccess || (e = grow(mid, n * 12)) != cudaSuccess ||
      (e = grow(node_of, n * 4)) != cudaSuccess || (e = grow(pairs, n * 4)) != cudaSuccess ||
      (e = a->didx.ensure(n * 4)) != cudaSuccess ||
      (e = grow(bsum, ((size_t)tiles + 1) * 4)) != cudaSuccess ||
      (e = grow(cnt, 16)) != cudaSuccess)
    return cuda_status(e, "line build scratch");
  uint32_t *d_err = cnt.as<uint32_t>(), *d_pairs = d_err + 1, *d_next = d_err + 2;
  cudaMemsetAsync(d_err, 0, 16, st);
  const unsigned egrid = (unsigned)std::min<size_t>((n + 255) / 256, (size_t)ctx->num_sms * 16);
  line_prep_kernel<<<egrid, 256, 0, st>>>(
      static_cast<const float *>(dp), static_cast<const float *>(dr), constant_radius,
      static_cast<const uint32_t *>(ds), nverts, n, lbox.as<float>(), mid.as<float>(),
      a->didx.as<uint32_t>(), node_of.as<uint32_t>(), d_err);
  ctx->launches++;
  uint32_t *idx = a->didx.as<uint32_t>(), *nof = node_of.as<uint32_t>();
  // the breadth-first node array grows by doubling (a level adds at most
  // twice its node count)
  if ((e = grow(bfs, 1024 * sizeof(LBNode))) != cudaSuccess)
    return cuda_status(e, "line build nodes");
  size_t bfs_cap = bfs.cap / sizeof(LBNode);
  LBNode root{};
  root.lo = 0;
  root.hi = (uint32_t)n;
  root.child = kLDone;
  cudaMemcpyAsync(bfs.p, &root, sizeof(root), cudaMemcpyHostToDevice, st);
  const unsigned cgrid = (unsigned)((n + (size_t)kLThreads * kLChunk - 1) / ((size_t)kLThreads * kLChunk));
  std::vector<std::pair<uint32_t, uint32_t>> levels;  // (first node, count)
  uint32_t off = 0, m = 1;
  for (int depth = 0; m; depth++) {
    if ((size_t)off + 3 * (size_t)m >= (1u << 29)) {
      set_error("srt_line_build: more than 2^29 nodes");
      return SRT_ERR_INVALID;
    }
    if ((size_t)off + 3 * (size_t)m > bfs_cap) {
      size_t want = bfs_cap;
      while (want < (size_t)off + 3 * (size_t)m) want *= 2;
      DevBuf grown;
      if ((e = grown.ensure(want * sizeof(LBNode))) != cudaSuccess)
        return cuda_status(e, "line build nodes");
      cudaMemcpyAsync(grown.p, bfs.p, (size_t)off * sizeof(LBNode) + (size_t)m * sizeof(LBNode),
                      cudaMemcpyDeviceToDevice, st);
      cudaStreamSynchronize(st);
      std::swap(grown.p, bfs.p);
      std::swap(grown.cap, bfs.cap);
      bfs_cap = bfs.cap / sizeof(LBNode);
    }
    if ((e = grow(level, (size_t)m * sizeof(LLevel))) != cudaSuccess ||
        (e = grow(nchild, (size_t)m * 4)) != cudaSuccess ||
        (e = grow(cbase, (size_t)m * 4)) != cudaSuccess ||
        (e = grow(bsum, (((size_t)m + kLTile - 1) / kLTile + (size_t)tiles + 1) * 4)) !=
            cudaSuccess)
      return cuda_status(e, "line build level");
    LBNode *nodes = bfs.as<LBNode>();
    LLevel *L = level.as<LLevel>();
    const unsigned ngrid = (unsigned)std::min<size_t>(((size_t)m + 255) / 256, 65535);
    const unsigned mtiles = (unsigned)(((size_t)m + kLTile - 1) / kLTile);
    lvl_init_kernel<<<ngrid, 256, 0, st>>>(L, m);
    lvl_box_kernel<<<cgrid, kLThreads, 0, st>>>(nof, idx, lbox.as<float>(), n, L);
    lvl_node_kernel<<<ngrid, 256, 0, st>>>(nodes, off, m, L, lbox.as<float>(), idx, n, depth,
                                           min_leaf, max_depth);
    lvl_count_kernel<<<cgrid, kLThreads, 0, st>>>(nof, idx, mid.as<float>(), n, L);
    lvl_split_kernel<<<ngrid, 256, 0, st>>>(nodes, off, m, L, nchild.as<uint32_t>());
    const PairFlag pf{nof, idx, mid.as<float>(), L};
    lscan_count_kernel<<<tiles, kLThreads, 0, st>>>(pf, n, bsum.as<uint32_t>());
    lscan_top_kernel<<<1, 1024, 0, st>>>(bsum.as<uint32_t>(), tiles, d_pairs);
    lscan_apply_kernel<<<tiles, kLThreads, 0, st>>>(pf, PairOut{nof, L, pairs.as<uint32_t>()},
                                                    n, bsum.as<uint32_t>());
    lvl_swap_kernel<<<egrid, 256, 0, st>>>(pairs.as<uint32_t>(), d_pairs, nof, L, idx);
    const ChildFlag cf{nchild.as<uint32_t>()};
    lscan_count_kernel<<<mtiles, kLThreads, 0, st>>>(cf, m, bsum.as<uint32_t>());
    lscan_top_kernel<<<1, 1024, 0, st>>>(bsum.as<uint32_t>(), mtiles, d_next);
    lscan_apply_kernel<<<mtiles, kLThreads, 0, st>>>(cf, ChildOut{cbase.as<uint32_t>()}, m,
                                                     bsum.as<uint32_t>());
    lvl_children_kernel<<<ngrid, 256, 0, st>>>(nodes, off, m, L, cbase.as<uint32_t>());
    lvl_next_kernel<<<egrid, 256, 0, st>>>(nof, L, cbase.as<uint32_t>(), n);
    ctx->launches += 14;
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_status(e, "line build level");
    uint32_t next = 0;
    if ((e = cudaMemcpyAsync(&next, d_next, 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
      return cuda_status(e, "line build level");
    levels.emplace_back(off, m);
    off += m;
    m = next;
  }
  const size_t total = off;
  uint32_t herr = 0;
  cudaMemcpy(&herr, d_err, 4, cudaMemcpyDeviceToHost);
  if (herr & kLErrVertex) {
    set_error("srt_line_build: a segment names a vertex beyond nverts");
    return SRT_ERR_INVALID;
  }
  if (herr & kLErrNaN) {
    set_error("srt_line_build: NaN in a line's position or radius");
    return SRT_ERR_INVALID;
  }
  if ((e = grow(sizes, total * 4)) != cudaSuccess || (e = grow(pre, total * 4)) != cudaSuccess ||
      (e = a->dref.ensure(total * sizeof(LineNodeH))) != cudaSuccess ||
      (e = a->dnodes.ensure(total * sizeof(LNode))) != cudaSuccess ||
      (e = a->drecs.ensure(n * sizeof(LineRec))) != cudaSuccess)
    return cuda_status(e, "line accel");
  for (size_t k = levels.size(); k-- > 0;) {
    const auto [lo, cntl] = levels[k];
    lvl_size_kernel<<<(unsigned)std::min<size_t>(((size_t)cntl + 255) / 256, 65535), 256, 0, st>>>(
        bfs.as<LBNode>(), lo, cntl, sizes.as<uint32_t>());
  }
  for (const auto &[lo, cntl] : levels)
    lvl_emit_kernel<<<(unsigned)std::min<size_t>(((size_t)cntl + 255) / 256, 65535), 256, 0, st>>>(
        bfs.as<LBNode>(), lo, cntl, sizes.as<uint32_t>(), pre.as<uint32_t>(),
        a->dref.as<LineNodeH>(), a->dnodes.as<LNode>());
  ctx->launches += 2 * levels.size();
  const unsigned grid = (unsigned)std::min<size_t>((n + 255) / 256, 4096);
  line_rec_kernel<<<grid, 256, 0, st>>>(
      static_cast<const float *>(dp), static_cast<const float *>(dr), constant_radius,
      static_cast<const uint32_t *>(ds), idx, n, a->drecs.as<LineRec>());
  ctx->launches++;
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_status(e, "line records");
  cudaMemcpyAsync(&a->root, a->dref.p, sizeof(LineNodeH), cudaMemcpyDeviceToHost, st);
  // the staged inputs are freed on return: finish with them first
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_status(e, "line build");
  a->nlines = n;
  a->nnodes = total;
  a->depth = (int)levels.size() - 1;
  a->cap = cap != 0;
  a->built = true;
  return SRT_OK;
}

SRT_API srt_status srt_line_trace(srt_line_accel *a, const srt_ray *rays, size_t n,
                                  srt_hit *hits, float *normals, uint64_t *stats) {
  if (!a || (n && (!rays || !hits))) return SRT_ERR_INVALID;
  if (stats && !is_device_ptr(stats)) {
    set_error("stats must be device memory");
    return SRT_ERR_INVALID;
  }
  if (!a->built) {
    set_error("line accel not built");
    return SRT_ERR_INVALID;
  }
  if (n == 0) return SRT_OK;
  srt_ctx *ctx = a->ctx;
  cudaSetDevice(ctx->device);
  const void *dr;
  srt_status s = line_view(ctx, rays, n * sizeof(srt_ray), ctx->s_stage_in, &dr);
  if (s != SRT_OK) return s;
  const bool hdev = is_device_ptr(hits), ndev = !normals || is_device_ptr(normals);
  srt_hit *dh = hits;
  float *dn = normals;
  cudaError_t e;
  if (!hdev) {
    if ((e = ctx->s_stage_out.ensure(n * sizeof(srt_hit))) != cudaSuccess)
      return cuda_status(e, "hit staging");
    dh = ctx->s_stage_out.as<srt_hit>();
  }
  if (!ndev) {
    if ((e = ctx->s_stage_norm.ensure(n * 12)) != cudaSuccess)
      return cuda_status(e, "normal staging");
    dn = ctx->s_stage_norm.as<float>();
  }
  if ((reinterpret_cast<uintptr_t>(dr) | reinterpret_cast<uintptr_t>(dh)) & 15u) {
    set_error("ray and hit arrays must be 16-byte aligned");
    return SRT_ERR_INVALID;
  }
  const unsigned grid = (unsigned)std::min<size_t>((n + 127) / 128, (size_t)ctx->num_sms * 32);
  const LNode *nd = a->dnodes.as<LNode>();
  const LineRec *rc = a->drecs.as<LineRec>();
  const srt_ray *rr = static_cast<const srt_ray *>(dr);
  unsigned long long *st = reinterpret_cast<unsigned long long *>(stats);
  // a coherent ray order (a Morton curve over origin and direction) keeps
  // the lanes of a warp on nearby paths; the hits do not depend on it
  const uint32_t *ord = nullptr;
  if (n >= 32768 && (s = ray_order(ctx, rr, n, &ord)) != SRT_OK) return s;
  const bool shallow = a->depth + 2 <= 64;
  if (shallow && !st)
    line_trace_kernel<64, false><<<grid, 128, 0, ctx->stream>>>(nd, rc, a->cap, rr, ord, n, dh,
                                                                 dn, st);
  else if (shallow)
    line_trace_kernel<64, true><<<grid, 128, 0, ctx->stream>>>(nd, rc, a->cap, rr, ord, n, dh,
                                                                dn, st);
  else if (!st)
    line_trace_kernel<520, false><<<grid, 128, 0, ctx->stream>>>(nd, rc, a->cap, rr, ord, n, dh,
                                                                  dn, st);
  else
    line_trace_kernel<520, true><<<grid, 128, 0, ctx->stream>>>(nd, rc, a->cap, rr, ord, n, dh,
                                                                 dn, st);
  ctx->launches++;
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_status(e, "line trace");
  if (!hdev) cudaMemcpyAsync(hits, dh, n * sizeof(srt_hit), cudaMemcpyDeviceToHost, ctx->stream);
  if (!ndev) cudaMemcpyAsync(normals, dn, n * 12, cudaMemcpyDeviceToHost, ctx->stream);
  if (!hdev || !ndev || !is_device_ptr(rays))
    return cuda_status(cudaStreamSynchronize(ctx->stream), "line trace");
  return SRT_OK;
}

SRT_API srt_status srt_line_bbox(srt_line_accel *a, double bmin[3], double bmax[3]) {
  if (!a || !bmin || !bmax) return SRT_ERR_INVALID;
  if (!a->built) {  // LineAccel::BoundingBox of an empty tree
    for (int k = 0; k < 3; k++) {
      bmin[k] = DBL_MAX;
      bmax[k] = -DBL_MAX;
    }
    return SRT_OK;
  }
  for (int k = 0; k < 3; k++) {
    bmin[k] = a->root.bmin[k];
    bmax[k] = a->root.bmax[k];
  }
  return SRT_OK;
}

SRT_API srt_status srt_line_info(srt_line_accel *a, uint64_t *nlines, uint64_t *nnodes,
                                 int32_t *depth) {
  if (!a) return SRT_ERR_INVALID;
  if (nlines) *nlines = a->built ? a->nlines : 0;
  if (nnodes) *nnodes = a->built ? a->nnodes : 0;
  if (depth) *depth = a->built ? a->depth : 0;
  return SRT_OK;
}

SRT_API srt_status srt_line_export(srt_line_accel *a, void *nodes, uint32_t *indices) {
  if (!a || !a->built) return SRT_ERR_INVALID;
  if (srt_status s = line_host(a); s != SRT_OK) return s;
  if (nodes) std::memcpy(nodes, a->nodes.data(), a->nodes.size() * sizeof(LineNodeH));
  if (indices) std::memcpy(indices, a->idx.data(), a->idx.size() * sizeof(uint32_t));
  return SRT_OK;
}

SRT_API srt_status srt_line_dump(srt_line_accel *a, const char *path) {
  if (!a || !path || !a->built) return SRT_ERR_INVALID;
  if (srt_status s = line_host(a); s != SRT_OK) return s;
  FILE *fp = fopen(path, "wb");
  if (!fp) {
    set_error(std::string("cannot write ") + path);
    return SRT_ERR_INVALID;
  }
  const unsigned long long nn = a->nodes.size(), ni = a->idx.size();
  bool ok = fwrite(&nn, 8, 1, fp) == 1 &&
            fwrite(a->nodes.data(), sizeof(LineNodeH), nn, fp) == nn &&
            fwrite(&ni, 8, 1, fp) == 1 && fwrite(a->idx.data(), 4, ni, fp) == ni;
  ok = (fclose(fp) == 0) && ok;
  if (!ok) {
    set_error(std::string("write failed: ") + path);
    return SRT_ERR_INVALID;
  }
  return SRT_OK;
}

}  // extern "C"
