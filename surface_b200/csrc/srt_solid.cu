// srt_solid.cu -- SolidAccel (render/render_accel_solid.cc) on the GPU:
// pyramids (5 vertices), prisms (6) and hexahedra (8), closest hit.
//
// Build (SolidAccel::Build32, :1795-2124) on the GPU: the scene box (every
// vertex -+ FLT_EPSILON * 16, an order-free min / max), the Morton codes of
// the solids' centroids (the running sum of the vertices times 1.0f / nv,
// render/render_prefix_tree_util.cc:347-382), the stable 30-bit radix sort
// and the Karras split of every internal node (ConstructBinaryRadixTree30)
// -- the stages the tetrahedra use; the reference's top-down emission
// order (BuildTreeRecursive32, :1361-1453: a leaf for a Karras leaf, for up
// to 5 solids or below depth 22) is laid out on the host from the split
// table alone, then the GPU fills the boxes: leaf boxes over the solids'
// vertices -+ FLT_EPSILON * 16, branch boxes merged left then right, one
// depth level at a time from the deepest.  A gather kernel copies each
// solid's vertices into a record in leaf order.
//
// Trace (SolidAccel::Traverse, :2345-2435): one thread per ray (in a Morton
// order of the rays for large batches), every
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

namespace {

// The reference's SolidNode (Dump record, 40 bytes).
struct SolidNodeH {
  float bmin[3], bmax[3];
  int32_t flag, axis;  // flag 1: leaf (data = count, first), 0: branch (children)
  uint32_t data[2];
};
static_assert(sizeof(SolidNodeH) == 40, "SolidNode layout");

// Device node: w1 bit 31 set for a leaf (w0 = first record, low bits = count),
// else w0 = left child, w1 = right child | axis << 29.
struct alignas(16) SNode {
  float bmin[3];
  uint32_t w0;
  float bmax[3];
  uint32_t w1;
};
static_assert(sizeof(SNode) == 32, "two 16-byte loads");

constexpr uint32_t kSolidLeaf = 0x80000000u;

// floats per record: nv vertices (xyz) and the solid's index, padded to 16 bytes
__host__ __device__ constexpr int rec_floats(int nv) { return ((3 * nv + 1) + 3) / 4 * 4; }

}  // namespace

struct srt_solid_accel {
  srt_ctx *ctx = nullptr;
  bool built = false;
  int nv = 0;
  size_t n = 0;
  std::vector<SolidNodeH> nodes;  // reference layout (Dump, export)
  std::vector<uint32_t> idx;
  srt::DevBuf dnodes, drecs;
};

namespace {

using srt::DevBuf;

// ------------------------------------------------------------------ build
__global__ void solid_morton_kernel(const float *__restrict__ v, const uint32_t *__restrict__ ix,
                                    int nv, size_t n, float lx, float ly, float lz, float ix_,
                                    float iy, float iz, uint32_t *__restrict__ codes) {
  const float invdiv = 1.0f / (float)nv;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    float c[3] = {0.0f, 0.0f, 0.0f};
    for (int j = 0; j < nv; j++) {
      const uint32_t f = ix[(size_t)nv * i + j];
      for (int k = 0; k < 3; k++) c[k] = c[k] + v[3 * (size_t)f + k];
    }
    for (int k = 0; k < 3; k++) c[k] *= invdiv;
    const uint32_t qx = srt::f2u32_x86((c[0] - lx) * ix_);
    const uint32_t qy = srt::f2u32_x86((c[1] - ly) * iy);
    const uint32_t qz = srt::f2u32_x86((c[2] - lz) * iz);
    codes[i] = (srt::spread10(qx) << 2) | (srt::spread10(qy) << 1) | srt::spread10(qz);
  }
}

__global__ void solid_gather_kernel(const float *__restrict__ v, const uint32_t *__restrict__ ix,
                                    const uint32_t *__restrict__ order, int nv, size_t n,
                                    float *__restrict__ recs) {
  const int rf = rec_floats(nv);
  for (size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x; j < n;
       j += (size_t)gridDim.x * blockDim.x) {
    const uint32_t p = order[j];
    float *r = recs + (size_t)rf * j;
    for (int q = 0; q < nv; q++) {
      const uint32_t f = ix[(size_t)nv * p + q];
      for (int k = 0; k < 3; k++) r[3 * q + k] = v[3 * (size_t)f + k];
    }
    r[3 * nv] = __uint_as_float(p);
    for (int k = 3 * nv + 1; k < rf; k++) r[k] = 0.0f;
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
__global__ void solid_box_kernel(const float *__restrict__ v, const uint32_t *__restrict__ ix,
                                 size_t refs, size_t nverts, int *__restrict__ box,
                                 uint32_t *__restrict__ bad) {
  const float eps = FLT_EPSILON * 16;
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
      const float x = v[3 * (size_t)f + k];
      lo[k] = min(lo[k], f2o(x - eps));
      hi[k] = max(hi[k], f2o(x + eps));
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

// Leaf boxes (ComputeBoundingBox30, :1121-1169): node ids of the leaves in
// leaves[], each over its sorted solids.
__global__ void solid_leafbox_kernel(const float *__restrict__ v, const uint32_t *__restrict__ ix,
                                     const uint32_t *__restrict__ order, int nv,
                                     const uint32_t *__restrict__ leaves, size_t nleaves,
                                     SNode *__restrict__ nodes) {
  const float eps = FLT_EPSILON * 16;
  for (size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x; j < nleaves;
       j += (size_t)gridDim.x * blockDim.x) {
    SNode &nd = nodes[leaves[j]];
    const uint32_t first = nd.w0, cnt = nd.w1 & ~kSolidLeaf;
    const uint32_t f0 = ix[(size_t)nv * order[first]];
    float lo[3], hi[3];
    for (int k = 0; k < 3; k++) {
      lo[k] = v[3 * (size_t)f0 + k] - eps;
      hi[k] = v[3 * (size_t)f0 + k] + eps;
    }
    for (uint32_t i = first; i < first + cnt; i++)
      for (int q = 0; q < nv; q++) {
        const uint32_t f = ix[(size_t)nv * order[i] + q];
        for (int k = 0; k < 3; k++) {
          const float a = v[3 * (size_t)f + k] - eps, b = v[3 * (size_t)f + k] + eps;
          if (lo[k] > a) lo[k] = a;
          if (hi[k] < b) hi[k] = b;
        }
      }
    for (int k = 0; k < 3; k++) {
      nd.bmin[k] = lo[k];
      nd.bmax[k] = hi[k];
    }
  }
}

// Branch boxes of one depth level (MergeBoundingBox: std::min / std::max of
// the left then the right child), deepest level first.
__global__ void solid_merge_kernel(const uint32_t *__restrict__ ids, size_t n,
                                   SNode *__restrict__ nodes) {
  for (size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x; j < n;
       j += (size_t)gridDim.x * blockDim.x) {
    SNode &nd = nodes[ids[j]];
    const SNode &l = nodes[nd.w0], &r = nodes[nd.w1 & 0x1fffffffu];
    for (int k = 0; k < 3; k++) {
      nd.bmin[k] = (r.bmin[k] < l.bmin[k]) ? r.bmin[k] : l.bmin[k];
      nd.bmax[k] = (l.bmax[k] < r.bmax[k]) ? r.bmax[k] : l.bmax[k];
    }
  }
}

// The reference's emission order (BuildTreeRecursive32, :1361-1453) on the
// host, topology only: device nodes in pre-order, each node's depth.
struct Topology {
  const uint32_t *code, *child;
  const uint8_t *flags;  // bit 0: left child is a single key, bit 1: right
  std::vector<SNode> &nodes;
  std::vector<int> &depth;

  static int axis_of(uint32_t c) { return ((c ? __builtin_clz(c) : 32) - 2) % 3; }

  size_t emit(uint32_t root, uint32_t l, uint32_t r, bool leaf, int d) {
    const size_t off = nodes.size();
    nodes.push_back(SNode{});
    depth.push_back(d);
    if (leaf || (r - l) <= 4 || d > 22) {
      nodes[off].w0 = l;
      nodes[off].w1 = kSolidLeaf | (r + 1 - l);
      return off;
    }
    const uint32_t mid = child[root];
    const size_t left = emit(mid, l, mid, flags[root] & 1, d + 1);
    const size_t right = emit(mid + 1, mid + 1, r, flags[root] & 2, d + 1);
    nodes[off].w0 = (uint32_t)left;
    nodes[off].w1 = (uint32_t)right | ((uint32_t)axis_of(code[root]) << 29);
    return off;
  }
};

// ------------------------------------------------------------------ trace
struct D3 {
  double x, y, z;
};
__device__ __forceinline__ D3 dsub(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ D3 dadd(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ D3 dscale(D3 a, double f) { return {a.x * f, a.y * f, a.z * f}; }
__device__ __forceinline__ D3 dcross(D3 a, D3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ double ddot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

// normalize (:85), then to float
__device__ __forceinline__ void s_unit(D3 a, float out[3]) {
  const double len = sqrt(a.x * a.x + a.y * a.y + a.z * a.z);
  out[0] = (float)(a.x / len);
  out[1] = (float)(a.y / len);
  out[2] = (float)(a.z / len);
}

__device__ __forceinline__ double comp(D3 a, int j) { return j == 0 ? a.x : (j == 1 ? a.y : a.z); }

// The crossing point of a face, every coordinate (FULL) or coordinate j
// only (out[j]; the one a hit's t is measured along).
// SetCrossPoint_Sq (double, :438-444): a quad face.
template <bool FULL>
__device__ __forceinline__ void s_quad(float out[3], int j, D3 v0, D3 v1, D3 v2, double ws0,
                                       double ws1, double ws2, double ws3, D3 e2, D3 e3,
                                       D3 dir) {
  const double w = ws2 + ws3 + ddot(dcross(e2, e3), dir);
  const double den = ws0 + ws1 + w;
  if (FULL) {
    const D3 p = dadd(dadd(dscale(v2, ws0), dscale(v0, ws1)), dscale(v1, w));
    out[0] = (float)(p.x / den);
    out[1] = (float)(p.y / den);
    out[2] = (float)(p.z / den);
  } else {
    const double pj = (comp(v2, j) * ws0 + comp(v0, j) * ws1) + comp(v1, j) * w;
    out[j] = (float)(pj / den);
  }
}

// A triangle face: the weighted sum in double, then the float vector
// divided by the float sum of the weights.
template <bool FULL>
__device__ __forceinline__ void s_tri(float out[3], int j, D3 a, double wa, D3 b, double wb,
                                      D3 c, double wc, double den) {
  const float f = (float)den;
  if (FULL) {
    const D3 p = dadd(dadd(dscale(a, wa), dscale(b, wb)), dscale(c, wc));
    out[0] = (float)p.x / f;
    out[1] = (float)p.y / f;
    out[2] = (float)p.z / f;
  } else {
    out[j] = (float)((comp(a, j) * wa + comp(b, j) * wb) + comp(c, j) * wc) / f;
  }
}

// Edges of each solid (GetEdges, :119-154): edge i = vertex hi[i] - vertex
// lo[i]; the Pluecker moment of edge i uses vertex i % MOD (:470).
template <int NV>
struct SolidTab;
template <>
struct SolidTab<5> {
  static constexpr int NE = 8, MOD = 4;
  __device__ static int hi(int i) {
    constexpr int t[8] = {1, 2, 3, 0, 4, 4, 4, 4};
    return t[i];
  }
  __device__ static int lo(int i) {
    constexpr int t[8] = {0, 1, 2, 3, 0, 1, 2, 3};
    return t[i];
  }
};
template <>
struct SolidTab<6> {
  static constexpr int NE = 9, MOD = 6;
  __device__ static int hi(int i) {
    constexpr int t[9] = {1, 2, 0, 4, 5, 3, 3, 4, 5};
    return t[i];
  }
  __device__ static int lo(int i) {
    constexpr int t[9] = {0, 1, 2, 3, 4, 5, 0, 1, 2};
    return t[i];
  }
};
template <>
struct SolidTab<8> {
  static constexpr int NE = 12, MOD = 8;
  __device__ static int hi(int i) {
    constexpr int t[12] = {1, 2, 3, 0, 5, 6, 7, 4, 4, 5, 6, 7};
    return t[i];
  }
  __device__ static int lo(int i) {
    constexpr int t[12] = {0, 1, 2, 3, 4, 5, 6, 7, 0, 1, 2, 3};
    return t[i];
  }
};

// One solid's vertices (floats, exactly as stored) read as doubles on use;
// edges are recomputed from them (the same double subtraction each time).
template <int NV>
struct SolidV {
  float x[NV][3];
  __device__ __forceinline__ D3 v(int k) const {
    return {(double)x[k][0], (double)x[k][1], (double)x[k][2]};
  }
  __device__ __forceinline__ D3 e(int i) const {
    return dsub(v(SolidTab<NV>::hi(i)), v(SolidTab<NV>::lo(i)));
  }
};

// ws[i] = dir . (e_i x v_{i % MOD}) + e_i . (dir x org) (:467-476)
template <int NV>
__device__ __forceinline__ void s_weights(const SolidV<NV> &S, D3 dir, D3 org,
                                          double (&ws)[SolidTab<NV>::NE]) {
  const D3 rpc = dcross(dir, org);
#pragma unroll
  for (int i = 0; i < SolidTab<NV>::NE; i++) {
    const D3 ei = S.e(i);
    ws[i] = ddot(dir, dcross(ei, S.v(i % SolidTab<NV>::MOD))) + ddot(ei, rpc);
  }
}

// The reference's Intersect{Pyramid,Prism,Hexa}D (:455-505, :559-611,
// :664-716) split in two.  face(ws, slot): the face its sign tests pick for
// crossing point `slot` (0 the first point, 1 the second; -1: the solid is
// missed).  point<FULL>(S, ws, face, ...): that face's crossing point (all
// of it and the face normal when FULL, else only coordinate j) by the same
// expressions.  A ray tests every solid's two points for t and forms the
// full point and normal only for a point that becomes its closest hit.
__device__ __forceinline__ bool s_cw(const double *ws, int side, int k) {
  return side == 0 ? ws[k] >= 0 : ws[k] <= 0;
}

template <int NV>
struct SolidFaces;

template <>
struct SolidFaces<5> {  // IntersectPyramidD: point n uses i = 1 - n
  __device__ static int face(const double (&ws)[8], int slot) {
    const int n = slot, i = 1 - slot;
    if (s_cw(ws, i, 0) && s_cw(ws, i, 1) && s_cw(ws, i, 2) && s_cw(ws, i, 3)) return 0;
    if (s_cw(ws, n, 0) && s_cw(ws, i, 4) && s_cw(ws, n, 5)) return 1;
    if (s_cw(ws, n, 1) && s_cw(ws, i, 5) && s_cw(ws, n, 6)) return 2;
    if (s_cw(ws, n, 2) && s_cw(ws, i, 6) && s_cw(ws, n, 7)) return 3;
    if (s_cw(ws, n, 3) && s_cw(ws, i, 7) && s_cw(ws, n, 4)) return 4;
    return -1;
  }
  template <bool FULL>
  __device__ static void point(const SolidV<5> &S, const double (&ws)[8], int f, D3 dir, int j,
                               float pos[3], float nrm[3]) {
    switch (f) {
      case 0:
        s_quad<FULL>(pos, j, S.v(0), S.v(1), S.v(2), ws[0], ws[1], ws[2], ws[3], S.e(2), S.e(3),
                     dir);
        if (FULL) s_unit(dcross(S.e(1), S.e(0)), nrm);
        break;
      case 1:
        s_tri<FULL>(pos, j, S.v(4), -ws[0], S.v(1), ws[4], S.v(0), -ws[5], -ws[0] + ws[4] - ws[5]);
        if (FULL) s_unit(dcross(S.e(4), S.e(0)), nrm);
        break;
      case 2:
        s_tri<FULL>(pos, j, S.v(4), -ws[1], S.v(2), ws[5], S.v(1), -ws[6], -ws[1] + ws[5] - ws[6]);
        if (FULL) s_unit(dcross(S.e(5), S.e(1)), nrm);
        break;
      case 3:
        s_tri<FULL>(pos, j, S.v(4), -ws[2], S.v(3), ws[6], S.v(2), -ws[7], -ws[2] + ws[6] - ws[7]);
        if (FULL) s_unit(dcross(S.e(6), S.e(2)), nrm);
        break;
      default:
        s_tri<FULL>(pos, j, S.v(4), -ws[3], S.v(0), ws[7], S.v(3), -ws[4], -ws[3] + ws[7] - ws[4]);
        if (FULL) s_unit(dcross(S.e(7), S.e(3)), nrm);
        break;
    }
  }
};

template <>
struct SolidFaces<6> {  // IntersectPrismD: point i uses n = 1 - i
  __device__ static int face(const double (&ws)[9], int slot) {
    const int i = slot, n = 1 - slot;
    if (s_cw(ws, n, 0) && s_cw(ws, n, 1) && s_cw(ws, n, 2)) return 0;
    if (s_cw(ws, i, 3) && s_cw(ws, i, 4) && s_cw(ws, i, 5)) return 1;
    if (s_cw(ws, i, 2) && s_cw(ws, i, 6) && s_cw(ws, n, 5) && s_cw(ws, n, 8)) return 2;
    if (s_cw(ws, i, 0) && s_cw(ws, i, 7) && s_cw(ws, n, 3) && s_cw(ws, n, 6)) return 3;
    if (s_cw(ws, i, 1) && s_cw(ws, i, 8) && s_cw(ws, n, 4) && s_cw(ws, n, 7)) return 4;
    return -1;
  }
  template <bool FULL>
  __device__ static void point(const SolidV<6> &S, const double (&ws)[9], int f, D3 dir, int j,
                               float pos[3], float nrm[3]) {
    switch (f) {
      case 0:
        s_tri<FULL>(pos, j, S.v(2), ws[0], S.v(0), ws[1], S.v(1), ws[2], ws[0] + ws[1] + ws[2]);
        if (FULL) s_unit(dcross(S.e(0), S.e(1)), nrm);
        break;
      case 1:
        s_tri<FULL>(pos, j, S.v(5), ws[3], S.v(3), ws[4], S.v(4), ws[5], ws[3] + ws[4] + ws[5]);
        if (FULL) s_unit(dcross(S.e(3), S.e(4)), nrm);
        break;
      case 2:
        s_quad<FULL>(pos, j, S.v(2), S.v(0), S.v(3), ws[2], ws[6], -ws[5], -ws[8], S.e(5),
                     S.e(8), dir);
        if (FULL) s_unit(dcross(S.e(2), S.e(6)), nrm);
        break;
      case 3:
        s_quad<FULL>(pos, j, S.v(0), S.v(1), S.v(4), ws[0], ws[7], -ws[3], -ws[6], S.e(3),
                     S.e(6), dir);
        if (FULL) s_unit(dcross(S.e(0), S.e(7)), nrm);
        break;
      default:
        s_quad<FULL>(pos, j, S.v(1), S.v(2), S.v(5), ws[1], ws[8], -ws[4], -ws[7], S.e(4),
                     S.e(7), dir);
        if (FULL) s_unit(dcross(S.e(1), S.e(8)), nrm);
        break;
    }
  }
};

template <>
struct SolidFaces<8> {  // IntersectHexaD: point i uses n = 1 - i
  __device__ static int face(const double (&ws)[12], int slot) {
    const int i = slot, n = 1 - slot;
    if (s_cw(ws, n, 0) && s_cw(ws, n, 1) && s_cw(ws, n, 2) && s_cw(ws, n, 3)) return 0;
    if (s_cw(ws, i, 4) && s_cw(ws, i, 5) && s_cw(ws, i, 6) && s_cw(ws, i, 7)) return 1;
    if (s_cw(ws, i, 0) && s_cw(ws, i, 9) && s_cw(ws, n, 4) && s_cw(ws, n, 8)) return 2;
    if (s_cw(ws, i, 1) && s_cw(ws, i, 10) && s_cw(ws, n, 5) && s_cw(ws, n, 9)) return 3;
    if (s_cw(ws, i, 2) && s_cw(ws, i, 11) && s_cw(ws, n, 6) && s_cw(ws, n, 10)) return 4;
    if (s_cw(ws, i, 3) && s_cw(ws, i, 8) && s_cw(ws, n, 7) && s_cw(ws, n, 11)) return 5;
    return -1;
  }
  template <bool FULL>
  __device__ static void point(const SolidV<8> &S, const double (&ws)[12], int f, D3 dir, int j,
                               float pos[3], float nrm[3]) {
    switch (f) {
      case 0:
        s_quad<FULL>(pos, j, S.v(0), S.v(1), S.v(2), ws[0], ws[1], ws[2], ws[3], S.e(2), S.e(3),
                     dir);
        if (FULL) s_unit(dcross(S.e(0), S.e(1)), nrm);
        break;
      case 1:
        s_quad<FULL>(pos, j, S.v(4), S.v(5), S.v(6), ws[4], ws[5], ws[6], ws[7], S.e(6), S.e(7),
                     dir);
        if (FULL) s_unit(dcross(S.e(4), S.e(5)), nrm);
        break;
      case 2:
        s_quad<FULL>(pos, j, S.v(0), S.v(1), S.v(5), ws[0], ws[9], -ws[4], -ws[8], S.e(4),
                     S.e(8), dir);
        if (FULL) s_unit(dcross(S.e(0), S.e(9)), nrm);
        break;
      case 3:
        s_quad<FULL>(pos, j, S.v(1), S.v(2), S.v(6), ws[1], ws[10], -ws[5], -ws[9], S.e(5),
                     S.e(9), dir);
        if (FULL) s_unit(dcross(S.e(1), S.e(10)), nrm);
        break;
      case 4:
        s_quad<FULL>(pos, j, S.v(2), S.v(3), S.v(7), ws[2], ws[11], -ws[6], -ws[10], S.e(6),
                     S.e(10), dir);
        if (FULL) s_unit(dcross(S.e(2), S.e(11)), nrm);
        break;
      default:
        s_quad<FULL>(pos, j, S.v(3), S.v(0), S.v(4), ws[3], ws[8], -ws[7], -ws[11], S.e(7),
                     S.e(11), dir);
        if (FULL) s_unit(dcross(S.e(3), S.e(8)), nrm);
        break;
    }
  }
};

// The full crossing point and normal of a hit that becomes a ray's closest
// (seldom: kept out of line so the test loop keeps its registers).
template <int NV>
__device__ __noinline__ void s_full_point(const SolidV<NV> &S,
                                          const double (&ws)[SolidTab<NV>::NE], int f, D3 dir,
                                          float pos[3], float nrm[3]) {
  SolidFaces<NV>::template point<true>(S, ws, f, dir, 0, pos, nrm);
}

// t of a crossing point along axis j (the last with |dir| > 0.1; none: 0),
// as the reference's parameter step computes it (:2280-2290).
__device__ __forceinline__ float s_t(float pj, int j, D3 org, D3 dir) {
  if (j < 0) return 0.0f;
  return (float)(((double)pj - comp(org, j)) / comp(dir, j));
}

// IntersectRayAABB (:2160-2204) with the reference's selection order.
__device__ __forceinline__ bool sbox_hit(const SNode &nd, const float org[3], const float inv[3],
                                         const int sign[3]) {
  float lo[3], hi[3];
  for (int k = 0; k < 3; k++) {
    lo[k] = sign[k] ? nd.bmax[k] : nd.bmin[k];
    hi[k] = sign[k] ? nd.bmin[k] : nd.bmax[k];
  }
  const float tx0 = (lo[0] - org[0]) * inv[0], tx1 = (hi[0] - org[0]) * inv[0];
  const float ty0 = (lo[1] - org[1]) * inv[1], ty1 = (hi[1] - org[1]) * inv[1];
  float tmin = (tx0 > ty0) ? tx0 : ty0;
  float tmax = (tx1 < ty1) ? tx1 : ty1;
  const float tz0 = (lo[2] - org[2]) * inv[2], tz1 = (hi[2] - org[2]) * inv[2];
  tmin = (tmin > tz0) ? tmin : tz0;
  tmax = (tmax < tz1) ? tmax : tz1;
  return (tmax > 0.0f) && (tmin <= tmax) && (tmin <= FLT_MAX);
}

// The reference's walk (render/render_accel_solid.cc:2345): near child first,
// every solid whose leaf box the ray enters tested (no culling by distance:
// a quad face's crossing point is an affine combination of its corners that
// can fall outside the solid's box, so a box entered beyond the running
// distance may still hold a nearer hit), the first of the smallest t kept.
constexpr int kSolidQ = 32;  // solids a lane queues before the warp tests them

template <int NV>
__global__ void __launch_bounds__(128, 3)  // 3 blocks per SM: 168 registers
solid_trace_kernel(const SNode *__restrict__ nodes, const float *__restrict__ recs,
                   const srt_ray *__restrict__ rays, const uint32_t *__restrict__ order,
                   size_t n, srt_hit *__restrict__ hits, float *__restrict__ normals,
                   float *__restrict__ positions) {
  // Each lane walks its ray and queues the solids of the leaves it enters
  // (in the walk's order) until kSolidQ are queued or the walk ends; then
  // the lanes test their queues side by side, so the costly solid tests run
  // on full warps instead of on the few lanes that reached a leaf.  A lane
  // whose walk and queue are done writes its hit and takes the next ray.
  constexpr int RF = rec_floats(NV);
  __shared__ uint32_t queue[kSolidQ][128];
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  size_t i = 0;
  float org[3], dir[3], inv[3];
  int sign[3];
  uint32_t prev = 0;
  float t = FLT_MAX, bn[3], bp[3];
  uint32_t prim = SRT_MISS;
  int stack[64];
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
    for (int qi = 0; qi < len; qi++) {
      const uint32_t j = queue[qi][threadIdx.x];
      const float4 *r4 = reinterpret_cast<const float4 *>(recs + (size_t)RF * j);
      float rv[RF];
#pragma unroll
      for (int q4 = 0; q4 < RF / 4; q4++) {
        const float4 v4 = __ldg(r4 + q4);
        rv[4 * q4] = v4.x;
        rv[4 * q4 + 1] = v4.y;
        rv[4 * q4 + 2] = v4.z;
        rv[4 * q4 + 3] = v4.w;
      }
      const uint32_t p = __float_as_uint(rv[3 * NV]);
      if (p == prev) continue;  // Ray::prev_prim_id
      SolidV<NV> S;
#pragma unroll
      for (int c = 0; c < NV; c++)
#pragma unroll
        for (int e = 0; e < 3; e++) S.x[c][e] = rv[3 * c + e];
      double ws[SolidTab<NV>::NE];
      s_weights<NV>(S, ddir, dorg, ws);
      const int f0 = SolidFaces<NV>::face(ws, 0);
      const int f1 = f0 < 0 ? -1 : SolidFaces<NV>::face(ws, 1);
      if (f1 < 0) continue;
      float pt[3] = {0.0f, 0.0f, 0.0f}, nd3[3];
      float th[2];
#pragma unroll
      for (int h = 0; h < 2; h++) {
        if (jax >= 0) SolidFaces<NV>::template point<false>(S, ws, h ? f1 : f0, ddir, jax, pt, nd3);
        th[h] = s_t(jax >= 0 ? pt[jax] : 0.0f, jax, dorg, ddir);
      }
#pragma unroll
      for (int h = 0; h < 2; h++)
        if (th[h] >= 0.0f && th[h] < t) {
          t = th[h];
          prim = p;
          s_full_point<NV>(S, ws, h ? f1 : f0, ddir, bp, bn);
          if (h) {  // the second point's normal is flipped
#pragma unroll
            for (int c = 0; c < 3; c++) bn[c] = -1.0f * bn[c];
          }
        }
    }
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
}  // namespace srt

using namespace srt;

extern "C" {

SRT_API srt_status srt_solid_create(srt_ctx *ctx, srt_solid_accel **out) {
  if (!ctx || !out) return SRT_ERR_INVALID;
  srt_solid_accel *a = new (std::nothrow) srt_solid_accel();
  if (!a) return SRT_ERR_NO_MEMORY;
  a->ctx = ctx;
  *out = a;
  return SRT_OK;
}

SRT_API srt_status srt_solid_destroy(srt_solid_accel *a) {
  if (!a) return SRT_OK;
  cudaSetDevice(a->ctx->device);
  cudaStreamSynchronize(a->ctx->stream);
  delete a;
  return SRT_OK;
}

SRT_API srt_status srt_solid_build(srt_solid_accel *a, int32_t verts_per_solid,
                                   const float *vertices, size_t nverts,
                                   const uint32_t *indices, size_t nsolids) {
  if (!a || !vertices || !indices) return SRT_ERR_INVALID;
  const int nv = verts_per_solid;
  if ((nv != 5 && nv != 6 && nv != 8) || nsolids < 2 || nsolids >= (1u << 29)) {
    set_error("srt_solid_build: 5, 6 or 8 vertices per solid and 2 .. 2^29 solids");
    return SRT_ERR_INVALID;
  }
  srt_ctx *ctx = a->ctx;
  cudaSetDevice(ctx->device);
  const size_t n = nsolids, refs = nsolids * (size_t)nv;
  DevBuf sv, si, codes, order, child, flags, boxbuf, dleaves, dlevel;
  const void *dv, *di;
  srt_status s;
  if ((s = solid_view(ctx, vertices, nverts * 12, sv, &dv)) != SRT_OK) return s;
  if ((s = solid_view(ctx, indices, refs * 4, si, &di)) != SRT_OK) return s;
  const float *d_v = static_cast<const float *>(dv);
  const uint32_t *d_ix = static_cast<const uint32_t *>(di);
  cudaError_t e;
  // scene box and index check on the GPU
  int hbox[8] = {INT_MAX, INT_MAX, INT_MAX, INT_MIN, INT_MIN, INT_MIN, 0, 0};
  if ((e = boxbuf.ensure(sizeof(hbox))) != cudaSuccess ||
      (e = cudaMemcpyAsync(boxbuf.p, hbox, sizeof(hbox), cudaMemcpyHostToDevice, ctx->stream)) !=
          cudaSuccess)
    return cuda_status(e, "solid box");
  const unsigned gbox = (unsigned)std::min<size_t>((refs + 255) / 256, (size_t)ctx->num_sms * 8);
  solid_box_kernel<<<gbox, 256, 0, ctx->stream>>>(d_v, d_ix, refs, nverts, boxbuf.as<int>(),
                                                   reinterpret_cast<uint32_t *>(boxbuf.as<int>() + 6));
  ctx->launches++;
  if ((e = cudaMemcpyAsync(hbox, boxbuf.p, sizeof(hbox), cudaMemcpyDeviceToHost, ctx->stream)) !=
          cudaSuccess ||
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
  if ((e = codes.ensure(n * 4)) != cudaSuccess || (e = order.ensure(n * 4)) != cudaSuccess ||
      (e = child.ensure(n * 4)) != cudaSuccess || (e = flags.ensure(n)) != cudaSuccess)
    return cuda_status(e, "solid build");
  const unsigned grid = (unsigned)std::min<size_t>((n + 255) / 256, (size_t)ctx->num_sms * 16);
  solid_morton_kernel<<<grid, 256, 0, ctx->stream>>>(d_v, d_ix, nv, n, lo[0], lo[1], lo[2],
                                                      inv[0], inv[1], inv[2], codes.as<uint32_t>());
  ctx->launches++;
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_status(e, "solid morton");
  if ((s = sort_pairs(ctx, codes.as<uint32_t>(), order.as<uint32_t>(), n, true, 30)) != SRT_OK)
    return s;
  if ((s = stage_karras(ctx, codes.as<uint32_t>(), n, child.as<uint32_t>(),
                        flags.as<uint8_t>())) != SRT_OK)
    return s;
  std::vector<uint32_t> hcode(n), hchild(n), hidx(n);
  std::vector<uint8_t> hflags(n);
  if ((e = cudaMemcpyAsync(hcode.data(), codes.p, n * 4, cudaMemcpyDeviceToHost, ctx->stream)) !=
          cudaSuccess ||
      (e = cudaMemcpyAsync(hidx.data(), order.p, n * 4, cudaMemcpyDeviceToHost, ctx->stream)) !=
          cudaSuccess ||
      (e = cudaMemcpyAsync(hchild.data(), child.p, (n - 1) * 4, cudaMemcpyDeviceToHost,
                           ctx->stream)) != cudaSuccess ||
      (e = cudaMemcpyAsync(hflags.data(), flags.p, n - 1, cudaMemcpyDeviceToHost, ctx->stream)) !=
          cudaSuccess ||
      (e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess)
    return cuda_status(e, "solid tree");
  // topology on the host, in the reference's pre-order (root, left, right)
  a->built = false;
  std::vector<SNode> dn;
  std::vector<int> depth;
  dn.reserve(n);
  depth.reserve(n);
  Topology T{hcode.data(), hchild.data(), hflags.data(), dn, depth};
  dn.push_back(SNode{});
  depth.push_back(-1);
  const uint32_t mid = hchild[0];
  const size_t left = T.emit(mid, 0, mid, hflags[0] & 1, 0);
  const size_t right = T.emit(mid + 1, mid + 1, (uint32_t)n - 1, hflags[0] & 2, 0);
  dn[0].w0 = (uint32_t)left;
  dn[0].w1 = (uint32_t)right | ((uint32_t)Topology::axis_of(hcode[0]) << 29);
  // leaves, then branches grouped by depth (deepest first) for the refit
  int maxd = 0;
  for (int d : depth) maxd = std::max(maxd, d);
  std::vector<uint32_t> leaves, byd;
  std::vector<size_t> start(maxd + 3, 0);
  for (size_t i = 0; i < dn.size(); i++)
    if (dn[i].w1 & kSolidLeaf)
      leaves.push_back((uint32_t)i);
    else
      start[depth[i] + 2]++;
  for (int d = 1; d < maxd + 3; d++) start[d] += start[d - 1];
  byd.resize(start[maxd + 2]);
  {
    std::vector<size_t> fill(start.begin(), start.end());
    for (size_t i = 0; i < dn.size(); i++)
      if (!(dn[i].w1 & kSolidLeaf)) byd[fill[depth[i] + 1]++] = (uint32_t)i;
  }
  if ((e = a->dnodes.ensure(dn.size() * sizeof(SNode))) != cudaSuccess ||
      (e = a->drecs.ensure(n * rec_floats(nv) * 4)) != cudaSuccess ||
      (e = dleaves.ensure(leaves.size() * 4)) != cudaSuccess ||
      (e = dlevel.ensure(std::max<size_t>(byd.size(), 1) * 4)) != cudaSuccess)
    return cuda_status(e, "solid accel");
  if ((e = cudaMemcpyAsync(a->dnodes.p, dn.data(), dn.size() * sizeof(SNode),
                           cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess ||
      (e = cudaMemcpyAsync(dleaves.p, leaves.data(), leaves.size() * 4, cudaMemcpyHostToDevice,
                           ctx->stream)) != cudaSuccess ||
      (byd.size() && (e = cudaMemcpyAsync(dlevel.p, byd.data(), byd.size() * 4,
                                          cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess))
    return cuda_status(e, "solid nodes");
  SNode *d_nodes = a->dnodes.as<SNode>();
  solid_leafbox_kernel<<<grid, 256, 0, ctx->stream>>>(d_v, d_ix, order.as<uint32_t>(), nv,
                                                       dleaves.as<uint32_t>(), leaves.size(),
                                                       d_nodes);
  ctx->launches++;
  for (int d = maxd; d >= -1; d--) {  // depth -1 is the root
    const size_t b0 = start[d + 1], b1 = start[d + 2];
    if (b1 == b0) continue;
    const unsigned gm = (unsigned)std::min<size_t>((b1 - b0 + 255) / 256, 1024);
    solid_merge_kernel<<<gm, 256, 0, ctx->stream>>>(dlevel.as<uint32_t>() + b0, b1 - b0, d_nodes);
    ctx->launches++;
  }
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_status(e, "solid refit");
  solid_gather_kernel<<<grid, 256, 0, ctx->stream>>>(d_v, d_ix, order.as<uint32_t>(), nv, n,
                                                      a->drecs.as<float>());
  ctx->launches++;
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_status(e, "solid records");
  // the reference-layout copy (Dump, export, BoundingBox)
  if ((e = cudaMemcpyAsync(dn.data(), d_nodes, dn.size() * sizeof(SNode), cudaMemcpyDeviceToHost,
                           ctx->stream)) != cudaSuccess)
    return cuda_status(e, "solid nodes");
  // staged inputs and scratch are freed on return: finish with them first
  if ((e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess) return cuda_status(e, "solid build");
  a->nodes.resize(dn.size());
  for (size_t i = 0; i < dn.size(); i++) {
    SolidNodeH &h = a->nodes[i];
    h = SolidNodeH{};
    for (int k = 0; k < 3; k++) {
      h.bmin[k] = dn[i].bmin[k];
      h.bmax[k] = dn[i].bmax[k];
    }
    if (dn[i].w1 & kSolidLeaf) {
      h.flag = 1;
      h.data[0] = dn[i].w1 & ~kSolidLeaf;
      h.data[1] = dn[i].w0;
    } else {
      h.axis = (int)(dn[i].w1 >> 29);
      h.data[0] = dn[i].w0;
      h.data[1] = dn[i].w1 & 0x1fffffffu;
    }
  }
  a->idx = std::move(hidx);
  a->nv = nv;
  a->n = n;
  a->built = true;
  return SRT_OK;
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
  const void *kfn = a->nv == 5   ? (const void *)solid_trace_kernel<5>
                    : a->nv == 6 ? (const void *)solid_trace_kernel<6>
                                 : (const void *)solid_trace_kernel<8>;
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, 128, 0) != cudaSuccess ||
      per_sm < 1) {
    cudaGetLastError();
    per_sm = 1;
  }
  const unsigned grid =
      (unsigned)std::min<size_t>((n + 127) / 128, (size_t)ctx->num_sms * per_sm);
  const SNode *nd = a->dnodes.as<SNode>();
  const float *rc = a->drecs.as<float>();
  const srt_ray *rr = static_cast<const srt_ray *>(dr);
  // a coherent ray order (a Morton curve over origin and direction) for
  // large batches; the hits do not depend on it
  const uint32_t *ord = nullptr;
  if (n >= 32768 && (s = ray_order(ctx, rr, n, &ord)) != SRT_OK) return s;
  if (a->nv == 5)
    solid_trace_kernel<5><<<grid, 128, 0, ctx->stream>>>(nd, rc, rr, ord, n, dh, dn, dp);
  else if (a->nv == 6)
    solid_trace_kernel<6><<<grid, 128, 0, ctx->stream>>>(nd, rc, rr, ord, n, dh, dn, dp);
  else
    solid_trace_kernel<8><<<grid, 128, 0, ctx->stream>>>(nd, rc, rr, ord, n, dh, dn, dp);
  ctx->launches++;
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_status(e, "solid trace");
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
  for (int k = 0; k < 3; k++) {
    bmin[k] = a->nodes[0].bmin[k];
    bmax[k] = a->nodes[0].bmax[k];
  }
  return SRT_OK;
}

SRT_API srt_status srt_solid_info(srt_solid_accel *a, uint64_t *nsolids, uint64_t *nnodes) {
  if (!a) return SRT_ERR_INVALID;
  if (nsolids) *nsolids = a->built ? a->n : 0;
  if (nnodes) *nnodes = a->built ? a->nodes.size() : 0;
  return SRT_OK;
}

SRT_API srt_status srt_solid_export(srt_solid_accel *a, void *nodes, uint32_t *indices) {
  if (!a || !a->built) return SRT_ERR_INVALID;
  if (nodes) std::memcpy(nodes, a->nodes.data(), a->nodes.size() * sizeof(SolidNodeH));
  if (indices) std::memcpy(indices, a->idx.data(), a->idx.size() * 4);
  return SRT_OK;
}

SRT_API srt_status srt_solid_dump(srt_solid_accel *a, const char *path) {
  if (!a || !path || !a->built) return SRT_ERR_INVALID;
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
