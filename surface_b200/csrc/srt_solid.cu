// srt_solid.cu -- SolidAccel (render/render_accel_solid.cc) on the GPU:
// pyramids (5 vertices), prisms (6) and hexahedra (8), closest hit.
//
// Build (SolidAccel::Build32, :1795-2124) on the GPU: the scene box (every
// vertex -+ FLT_EPSILON * 16, an order-free min / max), the Morton codes of
// the solids' centroids (the running sum of the vertices times 1.0f / nv,
// render/render_prefix_tree_util.cc:347-382), the stable 30-bit radix sort
// and the Karras split of every internal node (ConstructBinaryRadixTree30)
// -- the stages the tetrahedra use, with the same emitted-branch flags
// (BuildTreeRecursive32, :1361-1453: a leaf for a Karras leaf, for up to 5
// solids or below depth 22).  A gather kernel copies each solid's vertices
// into a record in leaf order; one kernel then writes every emitted node
// (branches by their slot, leaves by their first solid) and its box: leaf
// boxes over the solids' vertices -+ FLT_EPSILON * 16, branch boxes merged
// left then right as both children arrive.  The build stays on the GPU
// after one host read of the scene box; the reference's node order
// (pre-order, for Dump and export) is laid out on the host from the device
// tree only when asked for.
//
// Trace (SolidAccel::Traverse, :2345-2435): one lane per ray (in a Morton
// order of the rays for large batches) walking near child first; every
// popped node tests its own box; a leaf whose box is hit tests its solids
// (skipping Ray::prev_prim_id) with the Pluecker tests of Intersect*D
// (:455-717) in double, keeping the entry or exit point nearer than the
// current hit.  The reference's TestLeafNode returns a shadowed flag
// (always false), so its walk never lowers the distance bound of the box
// test: no box is culled by distance here either.  Compiled without FMA
// contraction, so every double and float operation rounds as the
// reference's x86-64 build does.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "srt_internal.cuh"
#include "srt_walks.cuh"

namespace {

using namespace srt_solid_walk;

// The reference's SolidNode (Dump record, 40 bytes).
struct SolidNodeH {
  float bmin[3], bmax[3];
  int32_t flag, axis;  // flag 1: leaf (data = count, first), 0: branch (children)
  uint32_t data[2];
};
static_assert(sizeof(SolidNodeH) == 40, "SolidNode layout");

}  // namespace

struct srt_solid_accel {
  srt_ctx *ctx = nullptr;
  bool built = false;
  int nv = 0;
  size_t n = 0;
  // device tree: branch b at node b, the leaf over sorted solids from r at
  // node n - 1 + r; records in sorted order; the sorted order itself; the
  // branch count (SceneInfo.nbranches)
  srt::DevBuf dnodes, drecs, dorder, dcodes, dinfo, dbox;
  // ordering across streams: the latest build's end (waited for by traces
  // and host reads) and the latest trace's launch (waited for by the next
  // build before it overwrites the tree)
  cudaEvent_t ev_built = nullptr, ev_used = nullptr;
  bool used = false;
  bool deep = false;  // tree deeper than the short walk stack (SAH builds)
  bool dbl = false;   // double-precision positions (records of doubles)
  // the reference layout (Dump, export), made from the device tree on first use
  bool host_ready = false;
  std::vector<SolidNodeH> nodes;
  std::vector<uint32_t> idx;
};

namespace {

using srt::DevBuf;

// ------------------------------------------------------------------ build
// A vertex coordinate padded by FLT_EPSILON * 16 (ComputeBoundingBox*'s
// `real v = vertices[i] -+ kEPS`): float positions in float, double
// positions in double, then rounded to float.
__host__ __device__ __forceinline__ float pad_lo(float x) { return x - FLT_EPSILON * 16; }
__host__ __device__ __forceinline__ float pad_hi(float x) { return x + FLT_EPSILON * 16; }
__host__ __device__ __forceinline__ float pad_lo(double x) {
  return (float)(x - (double)(FLT_EPSILON * 16));
}
__host__ __device__ __forceinline__ float pad_hi(double x) {
  return (float)(x + (double)(FLT_EPSILON * 16));
}

// CalculateMortonCodesSolid{Float,Double}30: the centroid of the vertices
// rounded to float.
template <typename T>
__global__ void solid_morton_kernel(const T *__restrict__ v, const uint32_t *__restrict__ ix,
                                    int nv, size_t n, float lx, float ly, float lz, float ix_,
                                    float iy, float iz, uint32_t *__restrict__ codes) {
  const float invdiv = 1.0f / (float)nv;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    float c[3] = {0.0f, 0.0f, 0.0f};
    for (int j = 0; j < nv; j++) {
      const uint32_t f = ix[(size_t)nv * i + j];
      for (int k = 0; k < 3; k++) c[k] = c[k] + (float)v[3 * (size_t)f + k];
    }
    for (int k = 0; k < 3; k++) c[k] *= invdiv;
    const uint32_t qx = srt::f2u32_x86((c[0] - lx) * ix_);
    const uint32_t qy = srt::f2u32_x86((c[1] - ly) * iy);
    const uint32_t qz = srt::f2u32_x86((c[2] - lz) * iz);
    codes[i] = (srt::spread10(qx) << 2) | (srt::spread10(qy) << 1) | srt::spread10(qz);
  }
}

// The solid's index in a record's word after the vertices.
__host__ __device__ __forceinline__ void rec_id(float *r, uint32_t p) {
  std::memcpy(r, &p, 4);
}
__host__ __device__ __forceinline__ void rec_id(double *r, uint32_t p) {
  const unsigned long long w = p;
  std::memcpy(r, &w, 8);
}

// Records in leaf order: the solid's vertices as given (T), its index.
template <typename T>
__global__ void solid_gather_kernel(const T *__restrict__ v, const uint32_t *__restrict__ ix,
                                    const uint32_t *__restrict__ order, int nv, size_t n,
                                    T *__restrict__ recs) {
  const int rw = rec_bytes<T>(nv) / (int)sizeof(T);
  for (size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x; j < n;
       j += (size_t)gridDim.x * blockDim.x) {
    const uint32_t p = order[j];
    T *r = recs + (size_t)rw * j;
    for (int q = 0; q < nv; q++) {
      const uint32_t f = ix[(size_t)nv * p + q];
      for (int k = 0; k < 3; k++) r[3 * q + k] = v[3 * (size_t)f + k];
    }
    rec_id(r + 3 * nv, p);
    for (int k = 3 * nv + 1; k < rw; k++) r[k] = (T)0;
  }
}

// order-preserving float -> int (for atomic min / max of non-NaN floats)
__device__ __forceinline__ int f2o(float f) {
  const int i = __float_as_int(f);
  return i >= 0 ? i : i ^ 0x7fffffff;
}

// Scene box: min / max of every referenced vertex -+ FLT_EPSILON * 16
// (ComputeBoundingBoxOMP; min and max do not depend on the order), and a
// flag for an index at or beyond nverts.  box: 3 mins then 3 maxes as
// ordered ints, initialised to INT_MAX / INT_MIN.
template <typename T>
__global__ void solid_box_kernel(const T *__restrict__ v, const uint32_t *__restrict__ ix,
                                 size_t refs, size_t nverts, int *__restrict__ box,
                                 uint32_t *__restrict__ bad) {
  int lo[3] = {INT_MAX, INT_MAX, INT_MAX}, hi[3] = {INT_MIN, INT_MIN, INT_MIN};
  bool oob = false;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < refs;
       i += (size_t)gridDim.x * blockDim.x) {
    const uint32_t f = ix[i];
    if (f >= nverts) {
      oob = true;
      continue;
    }
    for (int k = 0; k < 3; k++) {
      const T x = v[3 * (size_t)f + k];
      lo[k] = min(lo[k], f2o(pad_lo(x)));
      hi[k] = max(hi[k], f2o(pad_hi(x)));
    }
  }
  for (int o = 16; o > 0; o >>= 1)
    for (int k = 0; k < 3; k++) {
      lo[k] = min(lo[k], __shfl_xor_sync(0xffffffffu, lo[k], o));
      hi[k] = max(hi[k], __shfl_xor_sync(0xffffffffu, hi[k], o));
    }
  if (__any_sync(0xffffffffu, oob) && (threadIdx.x & 31) == 0) atomicOr(bad, 1u);
  if ((threadIdx.x & 31) == 0)
    for (int k = 0; k < 3; k++) {
      atomicMin(&box[k], lo[k]);
      atomicMax(&box[3 + k], hi[k]);
    }
}

// Leaf box (ComputeBoundingBox30, :1121-1169) over the records of sorted
// solids first..last: every vertex -+ FLT_EPSILON * 16, the first vertex
// first, then strict comparisons.
template <int NV, typename T>
__device__ __forceinline__ void leaf_box(const T *__restrict__ recs, uint32_t first,
                                         uint32_t last, float lo[3], float hi[3]) {
  constexpr int RW = rec_bytes<T>(NV) / (int)sizeof(T);
  const T *r0 = recs + (size_t)RW * first;
  for (int k = 0; k < 3; k++) {
    lo[k] = pad_lo(r0[k]);
    hi[k] = pad_hi(r0[k]);
  }
  for (uint32_t i = first; i <= last; i++) {
    const T *r = recs + (size_t)RW * i;
#pragma unroll
    for (int q = 0; q < NV; q++)
#pragma unroll
      for (int k = 0; k < 3; k++) {
        const T x = r[3 * q + k];
        const float a = pad_lo(x), b = pad_hi(x);
        if (lo[k] > a) lo[k] = a;
        if (hi[k] < b) hi[k] = b;
      }
  }
}

__device__ __forceinline__ void node_box_store(SNode *nd, const float lo[3], const float hi[3]) {
  for (int k = 0; k < 3; k++) {
    __stcg(&nd->bmin[k], lo[k]);
    __stcg(&nd->bmax[k], hi[k]);
  }
}
__device__ __forceinline__ void node_box_load(const SNode *nd, float lo[3], float hi[3]) {
  for (int k = 0; k < 3; k++) {
    lo[k] = __ldcg(&nd->bmin[k]);
    hi[k] = __ldcg(&nd->bmax[k]);
  }
}
// MergeBoundingBox: the right box's bound only where strictly beyond the left's.
__device__ __forceinline__ void merge_lr(const float llo[3], const float lhi[3],
                                         const float rlo[3], const float rhi[3], float lo[3],
                                         float hi[3]) {
  for (int k = 0; k < 3; k++) {
    lo[k] = (rlo[k] < llo[k]) ? rlo[k] : llo[k];
    hi[k] = (lhi[k] < rhi[k]) ? rhi[k] : lhi[k];
  }
}
// Arrival at a node's two-child counter: release this thread's box stores,
// acquire the other child's; returns the count before this arrival.
__device__ __forceinline__ uint32_t arrive_at(uint32_t *counter) {
  uint32_t old;
  asm volatile("atom.add.acq_rel.gpu.global.u32 %0, [%1], 1;" : "=r"(old) : "l"(counter)
               : "memory");
  return old;
}

// The emitted tree (BuildTreeRecursive32, :1361-1453: a leaf for a Karras
// leaf, for up to 5 solids or below depth 22) as device nodes, and its
// boxes, in one pass.  Thread per branch: branch b is node b (its slot; the
// root is slot 0), the leaf over sorted solids r.x..r.y is node m + r.x (m
// internal nodes; emitted leaves cover disjoint ranges).  A branch's thread
// writes its children links, axis ((clz(code) - 2) % 3 of its split code)
// and leaf children; boxes then climb to the root, the second child to
// arrive at a branch merging both (left then right).
template <int NV, typename V>
__global__ void __launch_bounds__(256)
solid_tree_kernel(const uint32_t *__restrict__ codes, srt::Topology T,
                  const srt::SceneInfo *__restrict__ info, uint32_t m,
                  const V *__restrict__ recs, SNode *__restrict__ nodes,
                  uint32_t *__restrict__ err) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= info->nbranches) return;
  const uint32_t i = __ldg(&T.kidx[t]);
  const uint32_t g = __ldg(&T.kchild[i]);
  const uint8_t fl = __ldg(&T.kflags[i]);
  uint32_t id[2];
  bool leaf[2];
  float clo[2][3], chi[2][3];
#pragma unroll
  for (int side = 0; side < 2; side++) {
    const uint32_t c = g + side;
    const bool kleaf = fl & (1 << side);
    leaf[side] = kleaf || !__ldg(&T.flag[c]);
    if (leaf[side]) {
      const uint2 r = kleaf ? make_uint2(c, c) : __ldg(&T.krange[c]);
      id[side] = m + r.x;
      leaf_box<NV, V>(recs, r.x, r.y, clo[side], chi[side]);
      SNode *ln = nodes + id[side];
      node_box_store(ln, clo[side], chi[side]);
      __stcg(&ln->w0, r.x);
      __stcg(&ln->w1, kSolidLeaf | (r.y - r.x + 1));
    } else {
      id[side] = __ldg(&T.slot[c]);
    }
  }
  const uint32_t code = __ldg(&codes[i]);
  const uint32_t axis = (uint32_t)(((code ? __clz(code) : 32) - 2) % 3);
  __stcg(&nodes[t].w0, id[0]);
  __stcg(&nodes[t].w1, id[1] | (axis << 29));
  if (!leaf[0] && !leaf[1]) return;  // both children climb here
  float lo[3], hi[3];
  if (leaf[0] && leaf[1]) {
    merge_lr(clo[0], chi[0], clo[1], chi[1], lo, hi);
  } else {
    // one leaf child: meet the branch child's climb
    if (arrive_at(&T.counter[i]) == 0) return;
    const int bs = leaf[0] ? 1 : 0;  // the branch side
    float blo[3], bhi[3];
    node_box_load(nodes + id[bs], blo, bhi);
    if (bs == 1)
      merge_lr(clo[0], chi[0], blo, bhi, lo, hi);
    else
      merge_lr(blo, bhi, clo[1], chi[1], lo, hi);
  }
  uint32_t node = i;
  for (int guard = 0; guard < 64; guard++) {
    const uint32_t ns = node == i ? t : __ldg(&T.slot[node]);
    node_box_store(nodes + ns, lo, hi);
    if (node == 0) return;
    const uint32_t q = __ldg(&T.kparent[node]);
    if (arrive_at(&T.counter[q]) == 0) return;
    const uint32_t gq = __ldg(&T.kchild[q]);
    const uint8_t fq = __ldg(&T.kflags[q]);
    const bool left = (gq == node) && !(fq & 1);
    const uint32_t sib = left ? gq + 1 : gq;
    const bool sib_kleaf = left ? (fq & 2) : (fq & 1);
    uint32_t sid;
    if (sib_kleaf)
      sid = m + sib;
    else if (__ldg(&T.flag[sib]))
      sid = __ldg(&T.slot[sib]);
    else
      sid = m + __ldg(&T.krange[sib]).x;
    float slo[3], shi[3];
    node_box_load(nodes + sid, slo, shi);
    float nlo[3], nhi[3];
    if (left)
      merge_lr(lo, hi, slo, shi, nlo, nhi);
    else
      merge_lr(slo, shi, lo, hi, nlo, nhi);
    for (int k = 0; k < 3; k++) {
      lo[k] = nlo[k];
      hi[k] = nhi[k];
    }
    node = q;
  }
  atomicOr(err, srt::kErrTree);
}

// ------------------------------------------------------------------ SAH build
// SolidAccel::Build (:1612-1793), which Build32 runs for fewer than 1024
// solids: a top-down binned-SAH build on the host (the inputs are small),
// float arithmetic in the reference's operation order, the tree in the
// reference's node order.  Options are the defaults of SolidBuildOptions
// (render_accel_solid.h:46-56): costTaabb 0.2, minLeafPrimitives 4,
// maxTreeDepth 256, binSize 64.  T: float or double positions (the
// reference's vertices / dvertices: boxes of double positions padded in
// double, bins over their float roundings, SAHPredD's double sum).
template <typename T>
struct SahBuilder {
  const T *v;
  const uint32_t *ix;
  int nv;
  std::vector<uint32_t> &idx;
  std::vector<SolidNodeH> &nodes;
  int max_depth = 0;
  static constexpr int kBins = 64, kMinLeaf = 4, kMaxDepth = 256;
  static constexpr float kTaabb = 0.2f;

  const T *vert(uint32_t solid, int j) const { return v + 3 * (size_t)ix[(size_t)nv * solid + j]; }

  // ComputeBoundingBox (:1076-1118): every vertex -+ FLT_EPSILON * 16
  void range_box(uint32_t l, uint32_t r, float lo[3], float hi[3]) const {
    const T *p0 = vert(idx[l], 0);
    for (int k = 0; k < 3; k++) {
      lo[k] = pad_lo(p0[k]);
      hi[k] = pad_hi(p0[k]);
    }
    for (uint32_t i = l; i < r; i++)
      for (int j = 0; j < nv; j++) {
        const T *p = vert(idx[i], j);
        for (int k = 0; k < 3; k++) {
          const float a = pad_lo(p[k]), b = pad_hi(p[k]);
          if (lo[k] > a) lo[k] = a;
          if (hi[k] < b) hi[k] = b;
        }
      }
  }
  // CalculateSurfaceArea (:791-799): float products and sums, doubled
  static float area(const float lo[3], const float hi[3]) {
    const float b0 = hi[0] - lo[0], b1 = hi[1] - lo[1], b2 = hi[2] - lo[2];
    return (float)(2.0 * (double)((b0 * b1 + b1 * b2) + b2 * b0));
  }
  // SAHPred / SAHPredD (:1034-1074): the summed vertex coordinate (a
  // float sum; double addends are added in double and rounded) against
  // pos * nv (float, or double for double positions)
  bool left_of(uint32_t solid, int axis, float pos) const {
    float c = 0.0f;
    for (int j = 0; j < nv; j++) c = (float)(c + vert(solid, j)[axis]);
    if (sizeof(T) == 8) return (double)c < (double)pos * (double)(float)nv;
    return c < pos * (float)nv;
  }
  // std::partition as libstdc++ runs it on bidirectional iterators: from
  // both ends, swapping a misplaced pair at a time
  uint32_t split(uint32_t l, uint32_t r, int axis, float pos) {
    uint32_t first = l, last = r;
    while (true) {
      while (true) {
        if (first == last) return first;
        if (left_of(idx[first], axis, pos)) first++;
        else break;
      }
      last--;
      while (true) {
        if (first == last) return first;
        if (!left_of(idx[last], axis, pos)) last--;
        else break;
      }
      std::swap(idx[first], idx[last]);
      first++;
    }
  }
  // ContributeBinBuffer + FindCutFromBinBuffer (:833-988): per axis the
  // cheapest bin boundary; returns the cheapest axis, cut[] per axis
  int find_cut(uint32_t l, uint32_t r, const float bmin[3], const float bmax[3], float cut[3]) const {
    const float eps = FLT_EPSILON * 16;
    std::vector<size_t> bins(2 * 3 * kBins, 0);
    float inv[3];
    for (int k = 0; k < 3; k++) {
      const float size = bmax[k] - bmin[k];
      inv[k] = size > eps ? (float)kBins / size : 0.0f;
    }
    for (uint32_t i = l; i < r; i++) {
      float slo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, shi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
      for (int j = 0; j < nv; j++) {  // GetBoundingBoxOfSolid: std::min / std::max
        const T *pv = vert(idx[i], j);
        const float p[3] = {(float)pv[0], (float)pv[1], (float)pv[2]};
        for (int k = 0; k < 3; k++) {
          slo[k] = (p[k] < slo[k]) ? p[k] : slo[k];
          shi[k] = (shi[k] < p[k]) ? p[k] : shi[k];
        }
      }
      for (int k = 0; k < 3; k++) {
        size_t a = (size_t)(unsigned int)std::floor((slo[k] - bmin[k]) * inv[k]);
        size_t b = (size_t)(unsigned int)std::floor((shi[k] - bmin[k]) * inv[k]);
        if (a >= (size_t)kBins) a = kBins - 1;
        if (b >= (size_t)kBins) b = kBins - 1;
        bins[0 * 3 * kBins + k * kBins + a]++;
        bins[1 * 3 * kBins + k * kBins + b]++;
      }
    }
    const size_t n = r - l;
    const float ttri = (float)(1.0 - (double)kTaabb);
    float bstep[3];
    for (int k = 0; k < 3; k++) bstep[k] = (bmax[k] - bmin[k]) * (float)(1.0 / kBins);
    const float sa = area(bmin, bmax);
    const float inv_sa = sa > eps ? (float)(1.0 / (double)sa) : 0.0f;
    float best[3];
    for (int k = 0; k < 3; k++) {
      float best_pos = bmin[k] + 0.5f * bstep[k];
      best[k] = FLT_MAX;
      size_t left = 0, right = n;
      float llo[3], lhi[3], rlo[3], rhi[3];
      for (int q = 0; q < 3; q++) {
        llo[q] = rlo[q] = bmin[q];
        lhi[q] = rhi[q] = bmax[q];
      }
      for (int i = 0; i < kBins - 1; i++) {
        left += bins[0 * 3 * kBins + k * kBins + i];
        right -= bins[1 * 3 * kBins + k * kBins + i];
        const float pos = bmin[k] + ((float)i + 0.5f) * bstep[k];
        lhi[k] = pos;
        rlo[k] = pos;
        const float sl = area(llo, lhi), sr = area(rlo, rhi);
        // SAH (:890-899), left to right
        const float cost = (2.0f * kTaabb + ((sl * inv_sa) * (float)left) * ttri) +
                           ((sr * inv_sa) * (float)right) * ttri;
        if (cost < best[k]) {
          best[k] = cost;
          best_pos = pos;
        }
      }
      cut[k] = best_pos;
    }
    int axis = 0;
    float c = best[0];
    if (c > best[1]) {
      axis = 1;
      c = best[1];
    }
    if (c > best[2]) axis = 2;
    return axis;
  }
  // BuildTree (:1612-1752); returns the node's index
  uint32_t build(uint32_t l, uint32_t r, int depth) {
    const uint32_t me = (uint32_t)nodes.size();
    max_depth = std::max(max_depth, depth);
    float bmin[3], bmax[3];
    range_box(l, r, bmin, bmax);
    nodes.push_back(SolidNodeH{});
    const uint32_t n = r - l;
    SolidNodeH h{};
    for (int k = 0; k < 3; k++) {
      h.bmin[k] = bmin[k];
      h.bmax[k] = bmax[k];
    }
    if ((int)n < kMinLeaf || depth >= kMaxDepth) {
      h.flag = 1;
      h.data[0] = n;
      h.data[1] = l;
      nodes[me] = h;
      return me;
    }
    float cut[3];
    const int best = find_cut(l, r, bmin, bmax, cut);
    uint32_t mid = l;
    int axis = best;
    for (int t = 0; t < 3; t++) {  // the cheapest axis first, then the others
      axis = (best + t) % 3;
      mid = split(l, r, axis, cut[axis]);
      if (mid == l || mid == r) mid = l + (n >> 1);  // object median unless another axis cuts
      else break;
    }
    h.flag = 0;
    h.axis = axis;
    h.data[0] = build(l, mid, depth + 1);
    h.data[1] = build(mid, r, depth + 1);
    nodes[me] = h;
    return me;
  }
};

// ------------------------------------------------------------------ trace
constexpr int kSolidQ = 32;  // solids a lane queues before the warp tests them
// walk stack entries: Build32 trees have at most 24 levels, SAH trees (Build,
// below 1024 solids) up to 257
constexpr int kSolidStackShort = 64, kSolidStackDeep = 264;

template <int NV, int STACK, typename T>
__global__ void __launch_bounds__(128, 3)  // 3 blocks per SM: 168 registers
solid_trace_kernel(const SNode *__restrict__ nodes, const void *__restrict__ recs,
                   const srt_ray *__restrict__ rays, const uint32_t *__restrict__ order,
                   size_t n, srt_hit *__restrict__ hits, float *__restrict__ normals,
                   float *__restrict__ positions, uint32_t *__restrict__ err) {
  // Each lane walks its ray and queues the solids of the leaves it enters
  // (in the walk's order) until kSolidQ are queued or the walk ends; then
  // the lanes test their queues side by side, so the costly solid tests run
  // on full warps instead of on the few lanes that reached a leaf.  A lane
  // whose walk and queue are done writes its hit and takes the next ray.
  __shared__ uint32_t queue[kSolidQ][128];
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  size_t i = 0;
  float org[3], dir[3], inv[3];
  int sign[3];
  uint32_t prev = 0;
  float t = FLT_MAX, bn[3], bp[3];
  uint32_t prim = SRT_MISS;
  int stack[STACK];
  int sp = -1;
  uint32_t leaf_next = 0, leaf_left = 0;
  auto start = [&]() {
    i = order ? (size_t)__ldg(&order[k]) : k;
    const float4 *rq = reinterpret_cast<const float4 *>(rays + i);
    const float4 r0 = __ldg(rq), r1 = __ldg(rq + 1);
    org[0] = r0.x; org[1] = r0.y; org[2] = r0.z;
    dir[0] = r1.x; dir[1] = r1.y; dir[2] = r1.z;
    prev = __float_as_uint(r0.w);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      sign[c] = dir[c] < 0.0f ? 1 : 0;
      inv[c] = __frcp_rn(dir[c]);  // (float)(1.0 / dir), correctly rounded
      bn[c] = bp[c] = 0.0f;
    }
    t = FLT_MAX;
    prim = SRT_MISS;
    stack[0] = 0;
    sp = 0;
    leaf_left = 0;
  };
  bool live = k < n;
  bool overflow = false;  // reported once, after the loop (an atomic inside it
                          // made the kernel several times slower)
  if (live) start();
  while (__any_sync(0xffffffffu, live)) {
    int len = 0;
    if (live) {
      while (len < kSolidQ) {
        if (leaf_left) {
          queue[len++][threadIdx.x] = leaf_next++;
          leaf_left--;
          continue;
        }
        if (sp < 0) break;
        const float4 *q = reinterpret_cast<const float4 *>(nodes + stack[sp]);
        const float4 a = __ldg(q), b = __ldg(q + 1);
        sp--;
        const SNode nd = {{a.x, a.y, a.z}, __float_as_uint(a.w), {b.x, b.y, b.z},
                          __float_as_uint(b.w)};
        if (!sbox_hit(nd, org, inv, sign)) continue;
        if (!(nd.w1 & kSolidLeaf)) {
          const int axis = (int)(nd.w1 >> 29);
          const int right = (int)(nd.w1 & 0x1fffffffu), left = (int)nd.w0;
          const int nearc = sign[axis];
          if (sp + 2 >= STACK) {  // deeper than the build's trees: stop the ray
            overflow = true;
            sp = -1;
            continue;
          }
          stack[++sp] = nearc ? left : right;  // far
          stack[++sp] = nearc ? right : left;  // near
          continue;
        }
        leaf_next = nd.w0;
        leaf_left = nd.w1 & ~kSolidLeaf;
      }
    }
    const D3 dorg = {org[0], org[1], org[2]}, ddir = {dir[0], dir[1], dir[2]};
    int jax = -1;  // the last axis with |dir| > 0.1
#pragma unroll
    for (int c = 0; c < 3; c++)
      if (dir[c] > 0.1 || dir[c] < -0.1) jax = c;
    for (int qi = 0; qi < len; qi++)
      solid_test<NV, T>(recs, queue[qi][threadIdx.x], prev, dorg, ddir, jax, t, prim, bp, bn);
    if (live && sp < 0 && leaf_left == 0) {
      const bool got = t < FLT_MAX;
      reinterpret_cast<float4 *>(hits)[i] =
          make_float4(t, 0.0f, 0.0f, __uint_as_float(got ? prim : SRT_MISS));
      for (int c = 0; c < 3; c++) {
        if (normals) normals[3 * i + c] = got ? bn[c] : 0.0f;
        if (positions) positions[3 * i + c] = got ? bp[c] : 0.0f;
      }
      k += stride;
      live = k < n;
      if (live) start();
    }
  }
  if (overflow) atomicOr(err, srt::kErrStack);
}

// The trace kernel for nv vertices per solid, a deep tree (SAH builds), and
// double-precision positions.
template <typename T>
const void *solid_kernel_t(int nv, bool deep) {
  if (deep)
    return nv == 5   ? (const void *)solid_trace_kernel<5, kSolidStackDeep, T>
           : nv == 6 ? (const void *)solid_trace_kernel<6, kSolidStackDeep, T>
                     : (const void *)solid_trace_kernel<8, kSolidStackDeep, T>;
  return nv == 5   ? (const void *)solid_trace_kernel<5, kSolidStackShort, T>
         : nv == 6 ? (const void *)solid_trace_kernel<6, kSolidStackShort, T>
                   : (const void *)solid_trace_kernel<8, kSolidStackShort, T>;
}
const void *solid_kernel(int nv, bool deep, bool dbl) {
  return dbl ? solid_kernel_t<double>(nv, deep) : solid_kernel_t<float>(nv, deep);
}

srt_status solid_view(srt_ctx *ctx, const void *p, size_t bytes, DevBuf &stage,
                      const void **out) {
  if (!p || srt::is_device_ptr(p)) {
    *out = p;
    return SRT_OK;
  }
  cudaError_t e = stage.ensure(bytes ? bytes : 1);
  if (e == cudaSuccess && bytes)
    e = cudaMemcpyAsync(stage.p, p, bytes, cudaMemcpyHostToDevice, ctx->stream);
  if (e != cudaSuccess) return srt::cuda_status(e, "solid staging");
  *out = stage.p;
  return SRT_OK;
}

}  // namespace

namespace srt {
uint64_t solid_accel_bytes(const srt_solid_accel *a) { return a->dnodes.cap + a->drecs.cap; }
bool solid_scene_view(const srt_solid_accel *a, srt_ctx **ctx, SceneElem &e, bool &deep) {
  if (!a || !a->built) return false;
  cudaEventSynchronize(a->ev_built);  // the build may have run on another stream
  *ctx = a->ctx;
  e.kind = kSceneSolids;
  e.nprims = (uint32_t)a->n;
  e.aux = a->nv | (a->dbl ? kSolidAuxDouble : 0);
  e.nodes = a->dnodes.p;
  e.prims = a->drecs.as<float4>();
  e.sidx = nullptr;
  e.scene = nullptr;
  deep = a->deep;
  return true;
}
}  // namespace srt

using namespace srt;

namespace {

// The device tree's root node (its box is the accel's BoundingBox).
srt_status solid_root(srt_solid_accel *a, SNode &root) {
  cudaSetDevice(a->ctx->device);
  cudaError_t e = cudaStreamWaitEvent(a->ctx->stream, a->ev_built, 0);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&root, a->dnodes.p, sizeof(SNode), cudaMemcpyDeviceToHost,
                        a->ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(a->ctx->stream);
  return cuda_status(e, "solid root");
}

// Pre-order (root, left, right) copy of the device subtree at node id in
// the reference's node layout; returns its index.
uint32_t solid_preorder(const std::vector<SNode> &dn, uint32_t id, std::vector<SolidNodeH> &out) {
  const SNode &d = dn[id];
  const uint32_t me = (uint32_t)out.size();
  out.push_back(SolidNodeH{});
  SolidNodeH h{};
  for (int k = 0; k < 3; k++) {
    h.bmin[k] = d.bmin[k];
    h.bmax[k] = d.bmax[k];
  }
  if (d.w1 & kSolidLeaf) {
    h.flag = 1;
    h.data[0] = d.w1 & ~kSolidLeaf;
    h.data[1] = d.w0;
  } else {
    h.axis = (int)(d.w1 >> 29);
    h.data[0] = solid_preorder(dn, d.w0, out);
    h.data[1] = solid_preorder(dn, d.w1 & 0x1fffffffu, out);
  }
  out[me] = h;
  return me;
}

// The reference layout of the tree (BuildTreeRecursive32's node order:
// pre-order) and the solid order, from the device tree, once per build.
srt_status solid_host_layout(srt_solid_accel *a) {
  if (a->host_ready) return SRT_OK;
  srt_ctx *ctx = a->ctx;
  cudaSetDevice(ctx->device);
  const size_t n = a->n, m = n - 1;
  std::vector<SNode> dn(m + n);
  a->idx.resize(n);
  cudaError_t e = cudaStreamWaitEvent(ctx->stream, a->ev_built, 0);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(dn.data(), a->dnodes.p, dn.size() * sizeof(SNode),
                        cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(a->idx.data(), a->dorder.p, n * 4, cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return cuda_status(e, "solid layout");
  a->nodes.clear();
  a->nodes.reserve(2 * n);
  solid_preorder(dn, 0, a->nodes);
  a->host_ready = true;
  return SRT_OK;
}

// Build32 below kSahMax solids: SolidAccel::Build on the host (SahBuilder),
// then the tree and the records in leaf order are uploaded.  v / ix may be
// host or device memory (device copies are read after the context's
// stream).
constexpr size_t kSahMax = 1024;

template <typename T>
srt_status solid_build_sah(srt_solid_accel *a, int nv, const T *v, size_t nverts,
                           const uint32_t *ix, size_t n) {
  srt_ctx *ctx = a->ctx;
  const size_t refs = n * (size_t)nv;
  std::vector<T> hv(3 * nverts);
  std::vector<uint32_t> hix(refs);
  cudaError_t e =
      cudaMemcpyAsync(hv.data(), v, hv.size() * sizeof(T), cudaMemcpyDefault, ctx->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(hix.data(), ix, refs * 4, cudaMemcpyDefault, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return cuda_status(e, "solid inputs");
  for (size_t i = 0; i < refs; i++)
    if (hix[i] >= nverts) {
      set_error("srt_solid_build: an index names a vertex beyond nverts");
      return SRT_ERR_INVALID;
    }
  a->nodes.clear();
  a->idx.resize(n);
  for (size_t i = 0; i < n; i++) a->idx[i] = (uint32_t)i;
  SahBuilder<T> B{hv.data(), hix.data(), nv, a->idx, a->nodes};
  B.build(0, (uint32_t)n, 0);
  // device layout: node k is reference node k; records in leaf order
  std::vector<SNode> dn(a->nodes.size());
  for (size_t k = 0; k < dn.size(); k++) {
    const SolidNodeH &h = a->nodes[k];
    for (int c = 0; c < 3; c++) {
      dn[k].bmin[c] = h.bmin[c];
      dn[k].bmax[c] = h.bmax[c];
    }
    if (h.flag) {
      dn[k].w0 = h.data[1];
      dn[k].w1 = kSolidLeaf | h.data[0];
    } else {
      dn[k].w0 = h.data[0];
      dn[k].w1 = h.data[1] | ((uint32_t)h.axis << 29);
    }
  }
  const int rw = rec_bytes<T>(nv) / (int)sizeof(T);
  std::vector<T> recs((size_t)rw * n, (T)0);
  for (size_t j = 0; j < n; j++) {
    const uint32_t p = a->idx[j];
    T *r = recs.data() + (size_t)rw * j;
    for (int q = 0; q < nv; q++)
      for (int k = 0; k < 3; k++) r[3 * q + k] = hv[3 * (size_t)hix[(size_t)nv * p + q] + k];
    rec_id(r + 3 * nv, p);
  }
  if ((e = a->dnodes.ensure(dn.size() * sizeof(SNode))) != cudaSuccess ||
      (e = a->drecs.ensure(recs.size() * sizeof(T))) != cudaSuccess ||
      (e = a->dorder.ensure(n * 4)) != cudaSuccess)
    return cuda_status(e, "solid accel");
  e = cudaMemcpyAsync(a->dnodes.p, dn.data(), dn.size() * sizeof(SNode), cudaMemcpyHostToDevice,
                      ctx->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(a->drecs.p, recs.data(), recs.size() * sizeof(T), cudaMemcpyHostToDevice,
                        ctx->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(a->dorder.p, a->idx.data(), n * 4, cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess) e = cudaEventRecord(a->ev_built, ctx->stream);
  // the host vectors go out of scope: the copies must be done
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return cuda_status(e, "solid upload");
  a->deep = B.max_depth + 2 > kSolidStackShort;
  a->dbl = sizeof(T) == 8;
  a->host_ready = true;
  a->nv = nv;
  a->n = n;
  a->built = true;
  return SRT_OK;
}

// sah: SolidAccel::Build (the binned-SAH build) for every size, as the
// GLES accel builder calls it; else Build32 (SAH below kSahMax, LBVH above).
template <typename T>
srt_status solid_build_t(srt_solid_accel *a, int32_t verts_per_solid, const T *vertices,
                         size_t nverts, const uint32_t *indices, size_t nsolids,
                         bool sah = false) {
  if (!a || !vertices || !indices) return SRT_ERR_INVALID;
  const int nv = verts_per_solid;
  if ((nv != 5 && nv != 6 && nv != 8) || nsolids < 2 || nsolids >= (1u << 28)) {
    set_error("srt_solid_build: 5, 6 or 8 vertices per solid and 2 .. 2^28 - 1 solids");
    return SRT_ERR_INVALID;
  }
  srt_ctx *ctx = a->ctx;
  cudaSetDevice(ctx->device);
  const size_t n = nsolids, refs = nsolids * (size_t)nv, m = n - 1;
  DevBuf sv, si;  // staging of host inputs
  const void *dv, *di;
  srt_status s;
  if ((s = solid_view(ctx, vertices, nverts * 3 * sizeof(T), sv, &dv)) != SRT_OK) return s;
  if ((s = solid_view(ctx, indices, refs * 4, si, &di)) != SRT_OK) return s;
  const T *d_v = static_cast<const T *>(dv);
  const uint32_t *d_ix = static_cast<const uint32_t *>(di);
  cudaError_t e;
  a->built = false;
  a->host_ready = false;
  // the latest trace (on any stream) reads the tree this build overwrites
  if (a->used && (e = cudaStreamWaitEvent(ctx->stream, a->ev_used, 0)) != cudaSuccess)
    return cuda_status(e, "solid build");
  if (sah || n < kSahMax) return solid_build_sah<T>(a, nv, d_v, nverts, d_ix, n);
  a->deep = false;
  a->dbl = sizeof(T) == 8;
  if ((e = a->dbox.ensure(64)) != cudaSuccess || (e = a->dcodes.ensure(n * 4)) != cudaSuccess ||
      (e = a->dorder.ensure(n * 4)) != cudaSuccess ||
      (e = a->dinfo.ensure(sizeof(srt::SceneInfo))) != cudaSuccess ||
      (e = a->dnodes.ensure((m + n) * sizeof(SNode))) != cudaSuccess ||
      (e = a->drecs.ensure(n * (size_t)rec_bytes<T>(nv))) != cudaSuccess)
    return cuda_status(e, "solid accel");
  // scene box and index check on the GPU: the one host round trip (an index
  // beyond nverts must fail before any kernel reads through it)
  int hbox[8] = {INT_MAX, INT_MAX, INT_MAX, INT_MIN, INT_MIN, INT_MIN, 0, 0};
  if ((e = cudaMemcpyAsync(a->dbox.p, hbox, sizeof(hbox), cudaMemcpyHostToDevice,
                           ctx->stream)) != cudaSuccess)
    return cuda_status(e, "solid box");
  const unsigned gbox = (unsigned)std::min<size_t>((refs + 255) / 256, (size_t)ctx->num_sms * 8);
  solid_box_kernel<<<gbox, 256, 0, ctx->stream>>>(d_v, d_ix, refs, nverts, a->dbox.as<int>(),
                                                   reinterpret_cast<uint32_t *>(a->dbox.as<int>() + 6));
  ctx->launches++;
  if ((e = cudaMemcpyAsync(hbox, a->dbox.p, sizeof(hbox), cudaMemcpyDeviceToHost,
                           ctx->stream)) != cudaSuccess ||
      (e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess)
    return cuda_status(e, "solid box");
  if (hbox[6]) {
    set_error("srt_solid_build: an index names a vertex beyond nverts");
    return SRT_ERR_INVALID;
  }
  float lo[3], hi3[3], inv[3];
  auto o2f_h = [](int i) {
    const int b = i >= 0 ? i : i ^ 0x7fffffff;
    float f;
    std::memcpy(&f, &b, 4);
    return f;
  };
  const int kdiv = 1 << 10;
  for (int k = 0; k < 3; k++) {
    lo[k] = o2f_h(hbox[k]);
    hi3[k] = o2f_h(hbox[3 + k]);
    inv[k] = kdiv / (hi3[k] - lo[k]);
  }
  uint32_t *codes = a->dcodes.as<uint32_t>(), *order = a->dorder.as<uint32_t>();
  const unsigned grid = (unsigned)std::min<size_t>((n + 255) / 256, (size_t)ctx->num_sms * 16);
  solid_morton_kernel<<<grid, 256, 0, ctx->stream>>>(d_v, d_ix, nv, n, lo[0], lo[1], lo[2],
                                                      inv[0], inv[1], inv[2], codes);
  ctx->launches++;
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_status(e, "solid morton");
  if ((s = sort_pairs(ctx, codes, order, n, true, 30)) != SRT_OK) return s;
  srt::Topology topo;
  srt::SceneInfo *info = a->dinfo.as<srt::SceneInfo>();
  if ((s = srt::stage_topology(ctx, codes, n, 4, info, topo)) != SRT_OK) return s;
  solid_gather_kernel<T><<<grid, 256, 0, ctx->stream>>>(d_v, d_ix, order, nv, n,
                                                         a->drecs.as<T>());
  const unsigned gt = (unsigned)((m + 255) / 256);
  SNode *d_nodes = a->dnodes.as<SNode>();
  const T *recs = a->drecs.as<T>();
  if (nv == 5)
    solid_tree_kernel<5, T><<<gt, 256, 0, ctx->stream>>>(codes, topo, info, (uint32_t)m, recs, d_nodes,
                                                      ctx->d_err);
  else if (nv == 6)
    solid_tree_kernel<6, T><<<gt, 256, 0, ctx->stream>>>(codes, topo, info, (uint32_t)m, recs, d_nodes,
                                                      ctx->d_err);
  else
    solid_tree_kernel<8, T><<<gt, 256, 0, ctx->stream>>>(codes, topo, info, (uint32_t)m, recs, d_nodes,
                                                      ctx->d_err);
  ctx->launches += 2;
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_status(e, "solid tree");
  if ((e = cudaEventRecord(a->ev_built, ctx->stream)) != cudaSuccess)
    return cuda_status(e, "solid build");
  // staged host inputs are freed on return: finish with them first
  if ((sv.p || si.p) && (e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess)
    return cuda_status(e, "solid build");
  a->nv = nv;
  a->n = n;
  a->built = true;
  return SRT_OK;
}

}  // namespace

extern "C" {

SRT_API srt_status srt_solid_create(srt_ctx *ctx, srt_solid_accel **out) {
  if (!ctx || !out) return SRT_ERR_INVALID;
  srt_solid_accel *a = new (std::nothrow) srt_solid_accel();
  if (!a) return SRT_ERR_NO_MEMORY;
  a->ctx = ctx;
  cudaSetDevice(ctx->device);
  cudaError_t e = cudaEventCreateWithFlags(&a->ev_built, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&a->ev_used, cudaEventDisableTiming);
  if (e != cudaSuccess) {
    if (a->ev_built) cudaEventDestroy(a->ev_built);
    delete a;
    return cuda_status(e, "solid accel events");
  }
  *out = a;
  return SRT_OK;
}

SRT_API srt_status srt_solid_destroy(srt_solid_accel *a) {
  if (!a) return SRT_OK;
  cudaSetDevice(a->ctx->device);
  cudaStreamSynchronize(a->ctx->stream);
  cudaEventSynchronize(a->ev_built);
  cudaEventSynchronize(a->ev_used);
  cudaEventDestroy(a->ev_built);
  cudaEventDestroy(a->ev_used);
  delete a;
  return SRT_OK;
}

SRT_API srt_status srt_solid_build(srt_solid_accel *a, int32_t verts_per_solid,
                                   const float *vertices, size_t nverts,
                                   const uint32_t *indices, size_t nsolids) {
  return solid_build_t<float>(a, verts_per_solid, vertices, nverts, indices, nsolids);
}

SRT_API srt_status srt_solid_build_double(srt_solid_accel *a, int32_t verts_per_solid,
                                          const double *vertices, size_t nverts,
                                          const uint32_t *indices, size_t nsolids) {
  return solid_build_t<double>(a, verts_per_solid, vertices, nverts, indices, nsolids);
}

SRT_API srt_status srt_solid_build_sah(srt_solid_accel *a, int32_t verts_per_solid,
                                       const float *vertices, size_t nverts,
                                       const uint32_t *indices, size_t nsolids) {
  return solid_build_t<float>(a, verts_per_solid, vertices, nverts, indices, nsolids, true);
}

SRT_API srt_status srt_solid_build_sah_double(srt_solid_accel *a, int32_t verts_per_solid,
                                              const double *vertices, size_t nverts,
                                              const uint32_t *indices, size_t nsolids) {
  return solid_build_t<double>(a, verts_per_solid, vertices, nverts, indices, nsolids, true);
}

SRT_API srt_status srt_solid_trace(srt_solid_accel *a, const srt_ray *rays, size_t n,
                                   srt_hit *hits, float *normals, float *positions) {
  if (!a || (n && (!rays || !hits))) return SRT_ERR_INVALID;
  if (!a->built) {
    set_error("solid accel not built");
    return SRT_ERR_INVALID;
  }
  if (n == 0) return SRT_OK;
  srt_ctx *ctx = a->ctx;
  cudaSetDevice(ctx->device);
  const void *dr;
  srt_status s = solid_view(ctx, rays, n * sizeof(srt_ray), ctx->s_stage_in, &dr);
  if (s != SRT_OK) return s;
  cudaError_t e;
  srt_hit *dh = hits;
  float *dn = normals, *dp = positions;
  const bool hdev = is_device_ptr(hits), ndev = !normals || is_device_ptr(normals),
             pdev = !positions || is_device_ptr(positions);
  if (!hdev) {
    if ((e = ctx->s_stage_out.ensure(n * sizeof(srt_hit))) != cudaSuccess)
      return cuda_status(e, "hit staging");
    dh = ctx->s_stage_out.as<srt_hit>();
  }
  if (!ndev) {
    if ((e = ctx->s_stage_norm.ensure(n * 12)) != cudaSuccess) return cuda_status(e, "staging");
    dn = ctx->s_stage_norm.as<float>();
  }
  if (!pdev) {
    if ((e = ctx->s_stage_scal.ensure(n * 12)) != cudaSuccess) return cuda_status(e, "staging");
    dp = ctx->s_stage_scal.as<float>();
  }
  if ((reinterpret_cast<uintptr_t>(dr) | reinterpret_cast<uintptr_t>(dh)) & 15u) {
    set_error("ray and hit arrays must be 16-byte aligned");
    return SRT_ERR_INVALID;
  }
  // as many blocks as the SMs hold at once: lanes take their next ray as
  // soon as they finish one
  const void *kfn = solid_kernel(a->nv, a->deep, a->dbl);
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, 128, 0) != cudaSuccess ||
      per_sm < 1) {
    cudaGetLastError();
    per_sm = 1;
  }
  const unsigned grid =
      (unsigned)std::min<size_t>((n + 127) / 128, (size_t)ctx->num_sms * per_sm);
  const SNode *nd = a->dnodes.as<SNode>();
  const void *rc = a->drecs.p;
  const srt_ray *rr = static_cast<const srt_ray *>(dr);
  // a coherent ray order (a Morton curve over origin and direction) for
  // large batches; the hits do not depend on it
  const uint32_t *ord = nullptr;
  if (n >= 32768 && (s = ray_order(ctx, rr, n, &ord)) != SRT_OK) return s;
  // the build may have run on another stream
  if ((e = cudaStreamWaitEvent(ctx->stream, a->ev_built, 0)) != cudaSuccess)
    return cuda_status(e, "solid trace");
  void *args[] = {(void *)&nd, (void *)&rc, (void *)&rr, (void *)&ord, (void *)&n,
                  (void *)&dh, (void *)&dn, (void *)&dp, (void *)&ctx->d_err};
  if ((e = cudaLaunchKernel(kfn, dim3(grid), dim3(128), args, 0, ctx->stream)) != cudaSuccess)
    return cuda_status(e, "solid trace");
  ctx->launches++;
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_status(e, "solid trace");
  if ((e = cudaEventRecord(a->ev_used, ctx->stream)) != cudaSuccess)
    return cuda_status(e, "solid trace");
  a->used = true;
  if (!hdev) cudaMemcpyAsync(hits, dh, n * sizeof(srt_hit), cudaMemcpyDeviceToHost, ctx->stream);
  if (!ndev) cudaMemcpyAsync(normals, dn, n * 12, cudaMemcpyDeviceToHost, ctx->stream);
  if (!pdev) cudaMemcpyAsync(positions, dp, n * 12, cudaMemcpyDeviceToHost, ctx->stream);
  if (!hdev || !ndev || !pdev || !is_device_ptr(rays))
    return cuda_status(cudaStreamSynchronize(ctx->stream), "solid trace");
  return SRT_OK;
}

SRT_API srt_status srt_solid_bbox(srt_solid_accel *a, double bmin[3], double bmax[3]) {
  if (!a || !bmin || !bmax) return SRT_ERR_INVALID;
  if (!a->built) {
    for (int k = 0; k < 3; k++) {
      bmin[k] = DBL_MAX;
      bmax[k] = -DBL_MAX;
    }
    return SRT_OK;
  }
  SNode root;
  srt_status s = solid_root(a, root);
  if (s != SRT_OK) return s;
  for (int k = 0; k < 3; k++) {
    bmin[k] = root.bmin[k];
    bmax[k] = root.bmax[k];
  }
  return SRT_OK;
}

SRT_API srt_status srt_solid_info(srt_solid_accel *a, uint64_t *nsolids, uint64_t *nnodes) {
  if (!a) return SRT_ERR_INVALID;
  if (nsolids) *nsolids = a->built ? a->n : 0;
  if (nnodes) {
    *nnodes = 0;
    if (a->built) {
      srt_status s = solid_host_layout(a);
      if (s != SRT_OK) return s;
      *nnodes = a->nodes.size();
    }
  }
  return SRT_OK;
}

SRT_API srt_status srt_solid_export(srt_solid_accel *a, void *nodes, uint32_t *indices) {
  if (!a || !a->built) return SRT_ERR_INVALID;
  srt_status s = solid_host_layout(a);
  if (s != SRT_OK) return s;
  if (nodes) std::memcpy(nodes, a->nodes.data(), a->nodes.size() * sizeof(SolidNodeH));
  if (indices) std::memcpy(indices, a->idx.data(), a->idx.size() * 4);
  return SRT_OK;
}

SRT_API srt_status srt_solid_dump(srt_solid_accel *a, const char *path) {
  if (!a || !path || !a->built) return SRT_ERR_INVALID;
  srt_status s = solid_host_layout(a);
  if (s != SRT_OK) return s;
  FILE *fp = fopen(path, "wb");
  if (!fp) {
    set_error(std::string("cannot write ") + path);
    return SRT_ERR_INVALID;
  }
  const unsigned long long nn = a->nodes.size(), ni = a->idx.size();
  bool ok = fwrite(&nn, 8, 1, fp) == 1 &&
            fwrite(a->nodes.data(), sizeof(SolidNodeH), nn, fp) == nn &&
            fwrite(&ni, 8, 1, fp) == 1 && fwrite(a->idx.data(), 4, ni, fp) == ni;
  ok = (fclose(fp) == 0) && ok;
  if (!ok) {
    set_error(std::string("write failed: ") + path);
    return SRT_ERR_INVALID;
  }
  return SRT_OK;
}

}  // extern "C"
