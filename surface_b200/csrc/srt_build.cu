// srt_build.cu -- LBVH build on the GPU, bit-exact with the reference's Build32.
//
// Pipeline (one CUDA stream, no host round trip):
//   1. scene box          bbox_partial + bbox_final
//        render/render_accel_triangle.cc:713-796 (eps 0),
//        render/render_accel_tetra.cc:973-1030, render/render_accel_particle.cc:304-369
//   2. Morton codes       morton_kernel
//        render/render_prefix_tree_util.cc:151-304, render/render_prefix_tree_util.h:113-157
//   3. stable sort        3 x 10-bit LSD passes over the 30-bit codes:
//        sort_codes30 (srt_sort.cu; one look-back kernel per pass) up to 2^18
//        keys, rs_hist / scan / rs_scatter below for more keys, full 32-bit
//        keys and segmented sorts
//        render/render_prefix_tree_util.h:296-457 (stable; ties keep input order)
//   4. Karras tree        karras_kernel
//        render/render_prefix_tree_util.cc:501-649
//   5. leaf collapse      level_scan_kernel: a Karras node is emitted as a
//        branch iff its range holds more than max_leaf+1 keys and its level
//        is <= 23; both tests are monotone along root paths, so the emitted
//        branches are exactly the top-down recursion's (BuildTreeRecursive32,
//        render/render_accel_triangle.cc:896-992; tetra :1113-1243;
//        particle :521-661).  The same kernel compacts: the exclusive prefix
//        sum of the branch flags (node slots) by tile look-back.
//   6. primitive cache    cache_kernel: leaf-ordered primitives for traversal
//   7. boxes              refit_kernel over the emitted tree only: leaves by
//        ComputeBoundingBox30 order (render/render_accel_triangle.cc:661-709),
//        branches bottom up by MergeBoundingBox, left first (:804)
//   8. emission           emit_node2_kernel / emit_tet_kernel
#include <algorithm>
#include <climits>
#include <cstdio>

#include "srt_internal.cuh"

namespace srt {
namespace {

constexpr int kBlock = 256;

inline int grid_for(size_t n, int block, int max_blocks) {
  size_t g = (n + block - 1) / block;
  if (g < 1) g = 1;
  if ((size_t)max_blocks < g) g = max_blocks;
  return (int)g;
}

// ------------------------------------------------------------------ primitives
// Leaf-ordered primitive cache (written by cache_kernel, read by traversal):
//   triangles: 3 float4 per prim: (p0, id bits), (p1, 0), (p2, 0)
//   tetrahedra: 3 float4 per prim: 12 vertex coordinates v0..v3
//   spheres:   1 float4 per prim: (centre, radius)
template <int KIND>
struct PrimTraits;

template <>
struct PrimTraits<SRT_TRIANGLES> {
  static constexpr int kCacheF4 = 3;
  static constexpr int kMaxLeaf = 16;
};
template <>
struct PrimTraits<SRT_TETRAHEDRA> {
  static constexpr int kCacheF4 = 3;
  static constexpr int kMaxLeaf = 4;
};
template <>
struct PrimTraits<SRT_SPHERES> {
  static constexpr int kCacheF4 = 1;
  static constexpr int kMaxLeaf = 16;
};

__device__ __forceinline__ void box_init(Box &b) {
  b.lo[0] = b.lo[1] = b.lo[2] = FLT_MAX;
  b.hi[0] = b.hi[1] = b.hi[2] = -FLT_MAX;
}

// Fold point p padded by e into b, first-value-kept on ties (the
// `if (bmin[k] > minval) bmin[k] = minval` loop of ComputeBoundingBox30).
__device__ __forceinline__ void box_add(Box &b, float x, float y, float z, float e) {
  float m;
  m = x - e; if (b.lo[0] > m) b.lo[0] = m;
  m = y - e; if (b.lo[1] > m) b.lo[1] = m;
  m = z - e; if (b.lo[2] > m) b.lo[2] = m;
  m = x + e; if (b.hi[0] < m) b.hi[0] = m;
  m = y + e; if (b.hi[1] < m) b.hi[1] = m;
  m = z + e; if (b.hi[2] < m) b.hi[2] = m;
}

// MergeBoundingBox (render/render_accel_triangle.cc:804): left first.
__device__ __forceinline__ Box box_merge(const Box &l, const Box &r) {
  Box o;
#pragma unroll
  for (int k = 0; k < 3; k++) {
    o.lo[k] = fmin_ref(l.lo[k], r.lo[k]);
    o.hi[k] = fmax_ref(l.hi[k], r.hi[k]);
  }
  return o;
}

// Box of sorted primitive j from the primitive cache.
template <int KIND>
__device__ __forceinline__ Box cache_box(const float4 *__restrict__ prims, uint32_t j,
                                         float keps) {
  Box b;
  box_init(b);
  if (KIND == SRT_TRIANGLES) {
    float4 p0 = __ldcg(&prims[3 * (size_t)j + 0]);
    float4 p1 = __ldcg(&prims[3 * (size_t)j + 1]);
    float4 p2 = __ldcg(&prims[3 * (size_t)j + 2]);
    box_add(b, p0.x, p0.y, p0.z, keps);
    box_add(b, p1.x, p1.y, p1.z, keps);
    box_add(b, p2.x, p2.y, p2.z, keps);
  } else if (KIND == SRT_TETRAHEDRA) {
    float4 a = __ldcg(&prims[3 * (size_t)j + 0]);
    float4 c = __ldcg(&prims[3 * (size_t)j + 1]);
    float4 d = __ldcg(&prims[3 * (size_t)j + 2]);
    box_add(b, a.x, a.y, a.z, keps);
    box_add(b, a.w, c.x, c.y, keps);
    box_add(b, c.z, c.w, d.x, keps);
    box_add(b, d.y, d.z, d.w, keps);
  } else {
    float4 s = __ldcg(&prims[j]);
    // (centre - radius) - eps, (centre + radius) + eps
    float lx = s.x - s.w, ly = s.y - s.w, lz = s.z - s.w;
    float hx = s.x + s.w, hy = s.y + s.w, hz = s.z + s.w;
    b.lo[0] = lx - keps; b.lo[1] = ly - keps; b.lo[2] = lz - keps;
    b.hi[0] = hx + keps; b.hi[1] = hy + keps; b.hi[2] = hz + keps;
  }
  return b;
}

// A tetrahedron of double-precision positions in the primitive cache: 12
// doubles (six double2) per tetrahedron, its four corners.  Its box pads
// each coordinate in double and rounds to float (ComputeBoundingBox30 over
// dvertices: `real v = dvertices[i] -+ kEPS`).
__device__ __forceinline__ void box_add_d(Box &b, double x, double y, double z, float e) {
  const double de = (double)e;
  float m;
  m = (float)(x - de); if (b.lo[0] > m) b.lo[0] = m;
  m = (float)(y - de); if (b.lo[1] > m) b.lo[1] = m;
  m = (float)(z - de); if (b.lo[2] > m) b.lo[2] = m;
  m = (float)(x + de); if (b.hi[0] < m) b.hi[0] = m;
  m = (float)(y + de); if (b.hi[1] < m) b.hi[1] = m;
  m = (float)(z + de); if (b.hi[2] < m) b.hi[2] = m;
}
template <int KIND>
__device__ __forceinline__ Box cache_box(const double2 *__restrict__ prims, uint32_t j,
                                         float keps) {
  static_assert(KIND == SRT_TETRAHEDRA, "double-precision cache: tetrahedra only");
  Box b;
  box_init(b);
  double x[12];
#pragma unroll
  for (int q = 0; q < 6; q++) {
    const double2 d = __ldcg(&prims[6 * (size_t)j + q]);
    x[2 * q] = d.x;
    x[2 * q + 1] = d.y;
  }
#pragma unroll
  for (int c = 0; c < 4; c++) box_add_d(b, x[3 * c], x[3 * c + 1], x[3 * c + 2], keps);
  return b;
}

// Double-precision tetrahedra: the positions rounded to float (the Morton
// codes' and the shading records' vertices, as real3 takes them), the
// scene box's partial boxes padded in double, and the double cache.
__global__ void round_vertices_kernel(const double *__restrict__ dv, size_t n3,
                                      float *__restrict__ vf) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n3;
       i += (size_t)gridDim.x * blockDim.x)
    vf[i] = (float)dv[i];
}

__global__ void bbox_partial_tet_d_kernel(const double *__restrict__ dv,
                                          const uint32_t *__restrict__ f, size_t n,
                                          Box *__restrict__ partial) {
  Box b;
  box_init(b);
  const float e = FLT_EPSILON * 16;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
#pragma unroll
    for (int c = 0; c < 4; c++) {
      const size_t vi = f[4 * i + c];
      box_add_d(b, dv[3 * vi], dv[3 * vi + 1], dv[3 * vi + 2], e);
    }
  }
  __shared__ Box sh[kBlock / 32];
#pragma unroll
  for (int k = 0; k < 3; k++) {
    for (int o = 16; o > 0; o >>= 1) {
      b.lo[k] = fmin_ref(b.lo[k], __shfl_down_sync(0xffffffffu, b.lo[k], o));
      b.hi[k] = fmax_ref(b.hi[k], __shfl_down_sync(0xffffffffu, b.hi[k], o));
    }
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) sh[w] = b;
  __syncthreads();
  if (threadIdx.x == 0) {
    Box r = sh[0];
    for (int i = 1; i < (int)(blockDim.x >> 5); i++) r = box_merge(r, sh[i]);
    partial[blockIdx.x] = r;
  }
}

__global__ void cache_tet_d_kernel(const double *__restrict__ dv, const uint32_t *__restrict__ f,
                                   const uint32_t *__restrict__ sidx, int n,
                                   double2 *__restrict__ prims) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    const uint32_t p = sidx[j];
    double x[12];
#pragma unroll
    for (int c = 0; c < 4; c++) {
      const size_t q = f[4 * (size_t)p + c];
      x[3 * c] = dv[3 * q];
      x[3 * c + 1] = dv[3 * q + 1];
      x[3 * c + 2] = dv[3 * q + 2];
    }
#pragma unroll
    for (int q = 0; q < 6; q++) prims[6 * (size_t)j + q] = make_double2(x[2 * q], x[2 * q + 1]);
  }
}

// ------------------------------------------------------------------ 1. scene box
template <int KIND>
__global__ void bbox_partial_kernel(const float *__restrict__ v,
                                    const uint32_t *__restrict__ f,
                                    const float *__restrict__ radius, float constr,
                                    size_t n, Box *__restrict__ partial,
                                    uint32_t *__restrict__ hist_zero,
                                    unsigned long long *__restrict__ tickets_zero) {
  // block 0 clears the digit histograms the Morton kernel fills and the sort
  // passes' tile counters
  if (hist_zero && blockIdx.x == 0) {
    for (int i = threadIdx.x; i < 3 * 1024; i += blockDim.x) hist_zero[i] = 0;
    if (threadIdx.x < 3) tickets_zero[threadIdx.x] = 0ull;
  }
  Box b;
  box_init(b);
  const float e = (KIND == SRT_TRIANGLES) ? 0.0f : FLT_EPSILON * 16;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    if (KIND == SRT_SPHERES) {
      float r = radius ? radius[i] : constr;
      float x = v[3 * i], y = v[3 * i + 1], z = v[3 * i + 2];
      float m;
      m = x - r - e; if (b.lo[0] > m) b.lo[0] = m;
      m = y - r - e; if (b.lo[1] > m) b.lo[1] = m;
      m = z - r - e; if (b.lo[2] > m) b.lo[2] = m;
      m = x + r + e; if (b.hi[0] < m) b.hi[0] = m;
      m = y + r + e; if (b.hi[1] < m) b.hi[1] = m;
      m = z + r + e; if (b.hi[2] < m) b.hi[2] = m;
    } else {
      const int nv = (KIND == SRT_TRIANGLES) ? 3 : 4;
#pragma unroll
      for (int c = 0; c < nv; c++) {
        size_t vi = f[(size_t)nv * i + c];
        box_add(b, v[3 * vi], v[3 * vi + 1], v[3 * vi + 2], e);
      }
    }
  }
  // block reduction (min/max are exact; order only matters for the sign of
  // zero, which the reference's own OpenMP merge leaves unspecified)
  __shared__ Box sh[kBlock / 32];
#pragma unroll
  for (int k = 0; k < 3; k++) {
    for (int o = 16; o > 0; o >>= 1) {
      b.lo[k] = fmin_ref(b.lo[k], __shfl_down_sync(0xffffffffu, b.lo[k], o));
      b.hi[k] = fmax_ref(b.hi[k], __shfl_down_sync(0xffffffffu, b.hi[k], o));
    }
  }
  int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) sh[w] = b;
  __syncthreads();
  if (threadIdx.x == 0) {
    Box r = sh[0];
    for (int i = 1; i < (int)(blockDim.x >> 5); i++) r = box_merge(r, sh[i]);
    partial[blockIdx.x] = r;
  }
}

// Build constants of a scene box: Morton scale, leaf padding, epsScale.
template <int KIND>
__device__ __forceinline__ SceneInfo scene_of_box(const Box &r) {
  SceneInfo s;
  for (int k = 0; k < 3; k++) {
    s.lo[k] = r.lo[k];
    s.hi[k] = r.hi[k];
    s.inv[k] = 1024.0f / (r.hi[k] - r.lo[k]);
  }
  if (KIND == SRT_TRIANGLES) {
    // epsScale = max extent (render/render_accel_triangle.cc:1452-1463)
    double es = (double)(r.hi[0] - r.lo[0]);
    if (es < (double)(r.hi[1] - r.lo[1])) es = (double)(r.hi[1] - r.lo[1]);
    if (es < (double)(r.hi[2] - r.lo[2])) es = (double)(r.hi[2] - r.lo[2]);
    s.eps_scale = es;
    s.keps = FLT_EPSILON * (float)es;
  } else {
    s.eps_scale = 16.0;
    s.keps = FLT_EPSILON * 16;
  }
  s.nbranches = 0;
  s.pad = 0;
  return s;
}

template <int KIND>
__global__ void bbox_final_kernel(const Box *__restrict__ partial, int np,
                                  SceneInfo *__restrict__ scene) {
  // one warp: lane l merges the l-th contiguous chunk in order, then lanes
  // merge pairwise with the earlier chunk on the left (first value seen
  // wins, as in a sequential merge)
  const int lane = threadIdx.x;
  const int chunk = (np + 31) / 32;
  const int b0 = min(np, lane * chunk), b1 = min(np, b0 + chunk);
  Box r;
  box_init(r);
  bool any = b0 < b1;
  if (any) {
    r = partial[b0];
    for (int i = b0 + 1; i < b1; i++) r = box_merge(r, partial[i]);
  }
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    Box q;
#pragma unroll
    for (int k = 0; k < 3; k++) {
      q.lo[k] = __shfl_down_sync(0xffffffffu, r.lo[k], o);
      q.hi[k] = __shfl_down_sync(0xffffffffu, r.hi[k], o);
    }
    const bool qany = __shfl_down_sync(0xffffffffu, any ? 1 : 0, o) != 0;
    if ((lane & (2 * o - 1)) == 0 && lane + o < 32 && qany) {
      r = any ? box_merge(r, q) : q;
      any = true;
    }
  }
  if (lane != 0) return;
  *scene = scene_of_box<KIND>(r);
}

// ------------------------------------------------------------------ 2. Morton
template <int KIND>
__global__ void morton_kernel(const float *__restrict__ v,
                              const uint32_t *__restrict__ f, size_t n,
                              const SceneInfo *__restrict__ scene,
                              uint32_t *__restrict__ codes,
                              uint32_t *__restrict__ index) {
  const float lx = scene->lo[0], ly = scene->lo[1], lz = scene->lo[2];
  const float ix = scene->inv[0], iy = scene->inv[1], iz = scene->inv[2];
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    float cx, cy, cz;
    if (KIND == SRT_SPHERES) {
      cx = v[3 * i];
      cy = v[3 * i + 1];
      cz = v[3 * i + 2];
    } else if (KIND == SRT_TRIANGLES) {
      const float third = 1.0f / 3.0f;
      size_t a = f[3 * i], b = f[3 * i + 1], c = f[3 * i + 2];
      cx = third * ((v[3 * a] + v[3 * b]) + v[3 * c]);
      cy = third * ((v[3 * a + 1] + v[3 * b + 1]) + v[3 * c + 1]);
      cz = third * ((v[3 * a + 2] + v[3 * b + 2]) + v[3 * c + 2]);
    } else {
      const float fourth = 1.0f / 4.0f;
      size_t a = f[4 * i], b = f[4 * i + 1], c = f[4 * i + 2], d = f[4 * i + 3];
      cx = fourth * (((v[3 * a] + v[3 * b]) + v[3 * c]) + v[3 * d]);
      cy = fourth * (((v[3 * a + 1] + v[3 * b + 1]) + v[3 * c + 1]) + v[3 * d + 1]);
      cz = fourth * (((v[3 * a + 2] + v[3 * b + 2]) + v[3 * c + 2]) + v[3 * d + 2]);
    }
    uint32_t qx = f2u32_x86((cx - lx) * ix);
    uint32_t qy = f2u32_x86((cy - ly) * iy);
    uint32_t qz = f2u32_x86((cz - lz) * iz);
    codes[i] = (spread10(qx) << 2) | (spread10(qy) << 1) | spread10(qz);
    if (index) index[i] = (uint32_t)i;
  }
}

// The same codes with the scene box reduced from the partial boxes in every
// block (block 0 stores the SceneInfo) and, into `hist`, the digit counts of
// the sort's three 10-bit passes (shared histograms, warp-aggregated) -- so
// neither a final-box kernel nor a histogram pass over the codes is needed.
template <int KIND>
__global__ void __launch_bounds__(kBlock)
morton_hist_kernel(const float *__restrict__ v, const uint32_t *__restrict__ f, size_t n,
                   const Box *__restrict__ partial, int np, SceneInfo *__restrict__ scene,
                   uint32_t *__restrict__ codes, uint32_t *__restrict__ hist) {
  __shared__ uint32_t h[3][1024];
  __shared__ Box sh[kBlock / 32];
  __shared__ SceneInfo ss;
  for (int i = threadIdx.x; i < 3 * 1024; i += kBlock) (&h[0][0])[i] = 0;
  // scene box: any merge order gives the same values (min / max are exact;
  // the reference's OpenMP merge leaves only the sign of zero unspecified)
  Box b;
  box_init(b);
  for (int i = threadIdx.x; i < np; i += kBlock) b = box_merge(b, partial[i]);
#pragma unroll
  for (int k = 0; k < 3; k++) {
    for (int o = 16; o > 0; o >>= 1) {
      b.lo[k] = fmin_ref(b.lo[k], __shfl_down_sync(0xffffffffu, b.lo[k], o));
      b.hi[k] = fmax_ref(b.hi[k], __shfl_down_sync(0xffffffffu, b.hi[k], o));
    }
  }
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) sh[w] = b;
  __syncthreads();
  if (threadIdx.x == 0) {
    Box r = sh[0];
    for (int i = 1; i < kBlock / 32; i++) r = box_merge(r, sh[i]);
    ss = scene_of_box<KIND>(r);
    if (blockIdx.x == 0) *scene = ss;
  }
  __syncthreads();
  const float lx = ss.lo[0], ly = ss.lo[1], lz = ss.lo[2];
  const float ix = ss.inv[0], iy = ss.inv[1], iz = ss.inv[2];
  const size_t stride = (size_t)gridDim.x * kBlock;
  for (size_t base = (size_t)blockIdx.x * kBlock; base < n; base += stride) {
    const size_t i = base + threadIdx.x;
    const bool ok = i < n;
    uint32_t code = 0;
    if (ok) {
      float cx, cy, cz;
      if (KIND == SRT_SPHERES) {
        cx = v[3 * i];
        cy = v[3 * i + 1];
        cz = v[3 * i + 2];
      } else if (KIND == SRT_TRIANGLES) {
        const float third = 1.0f / 3.0f;
        size_t a = f[3 * i], b2 = f[3 * i + 1], c = f[3 * i + 2];
        cx = third * ((v[3 * a] + v[3 * b2]) + v[3 * c]);
        cy = third * ((v[3 * a + 1] + v[3 * b2 + 1]) + v[3 * c + 1]);
        cz = third * ((v[3 * a + 2] + v[3 * b2 + 2]) + v[3 * c + 2]);
      } else {
        const float fourth = 1.0f / 4.0f;
        size_t a = f[4 * i], b2 = f[4 * i + 1], c = f[4 * i + 2], d = f[4 * i + 3];
        cx = fourth * (((v[3 * a] + v[3 * b2]) + v[3 * c]) + v[3 * d]);
        cy = fourth * (((v[3 * a + 1] + v[3 * b2 + 1]) + v[3 * c + 1]) + v[3 * d + 1]);
        cz = fourth * (((v[3 * a + 2] + v[3 * b2 + 2]) + v[3 * c + 2]) + v[3 * d + 2]);
      }
      const uint32_t qx = f2u32_x86((cx - lx) * ix);
      const uint32_t qy = f2u32_x86((cy - ly) * iy);
      const uint32_t qz = f2u32_x86((cz - lz) * iz);
      code = (spread10(qx) << 2) | (spread10(qy) << 1) | spread10(qz);
      codes[i] = code;
    }
    const unsigned act = __ballot_sync(0xffffffffu, ok);
#pragma unroll
    for (int p = 0; p < 3; p++) {
      const uint32_t d = (code >> (10 * p)) & 1023u;
      const unsigned peers = __match_any_sync(0xffffffffu, d) & act;
      if (ok && lane == __ffs(peers) - 1) atomicAdd(&h[p][d], (uint32_t)__popc(peers));
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 3 * 1024; i += kBlock) {
    const uint32_t c = (&h[0][0])[i];
    if (c) atomicAdd(&hist[i], c);
  }
}

// ------------------------------------------------------------------ scan
constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;

// Block-wide exclusive scan of a tile; returns the tile total.
__device__ uint32_t block_exclusive_scan(uint32_t (&x)[kScanItems]) {
  __shared__ uint32_t warp_tot[32];
  __shared__ uint32_t total;
  const int nwarps = (int)(blockDim.x >> 5);
  uint32_t s = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; i++) {
    uint32_t t = x[i];
    x[i] = s;
    s += t;
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  uint32_t inc = s;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += y;
  }
  if (lane == 31) warp_tot[w] = inc;
  __syncthreads();
  if (w == 0) {
    uint32_t t = (lane < nwarps) ? warp_tot[lane] : 0u;
    uint32_t ti = t;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, ti, o);
      if (lane >= o) ti += y;
    }
    if (lane < nwarps) warp_tot[lane] = ti - t;
    if (lane == nwarps - 1) total = ti;
  }
  __syncthreads();
  const uint32_t base = warp_tot[w] + (inc - s);
#pragma unroll
  for (int i = 0; i < kScanItems; i++) x[i] += base;
  const uint32_t r = total;
  __syncthreads();
  return r;
}

__global__ void scan_tiles_kernel(const uint32_t *__restrict__ in,
                                  uint32_t *__restrict__ out, size_t n,
                                  uint32_t *__restrict__ tile_sums) {
  size_t base = (size_t)blockIdx.x * kScanTile + (size_t)threadIdx.x * kScanItems;
  uint32_t x[kScanItems];
#pragma unroll
  for (int i = 0; i < kScanItems; i++) x[i] = (base + i < n) ? in[base + i] : 0u;
  uint32_t tot = block_exclusive_scan(x);
#pragma unroll
  for (int i = 0; i < kScanItems; i++)
    if (base + i < n) out[base + i] = x[i];
  if (threadIdx.x == 0 && tile_sums) tile_sums[blockIdx.x] = tot;
}

__global__ void scan_add_kernel(uint32_t *__restrict__ out, size_t n,
                                const uint32_t *__restrict__ tile_off) {
  uint32_t add = tile_off[blockIdx.x];
  size_t base = (size_t)blockIdx.x * kScanTile;
  for (int i = threadIdx.x; i < kScanTile; i += blockDim.x)
    if (base + i < n) out[base + i] += add;
}

}  // namespace

// Exclusive scan of n uint32 (out may alias in); tile sums of each level go
// to `scratch` (needs about n / 4095 + 4 words).
static srt_status scan_levels(cudaStream_t st, const uint32_t *in, uint32_t *out,
                              size_t n, uint32_t *scratch, uint64_t &launches) {
  size_t tiles = (n + kScanTile - 1) / kScanTile;
  if (tiles <= 1) {
    scan_tiles_kernel<<<1, kScanThreads, 0, st>>>(in, out, n, nullptr);
    launches++;
    return cuda_status(cudaGetLastError(), "scan");
  }
  uint32_t *sums = scratch;
  scan_tiles_kernel<<<(unsigned)tiles, kScanThreads, 0, st>>>(in, out, n, sums);
  launches++;
  srt_status s = cuda_status(cudaGetLastError(), "scan tiles");
  if (s != SRT_OK) return s;
  s = scan_levels(st, sums, sums, tiles, scratch + tiles, launches);
  if (s != SRT_OK) return s;
  scan_add_kernel<<<(unsigned)tiles, 256, 0, st>>>(out, n, sums);
  launches++;
  return cuda_status(cudaGetLastError(), "scan add");
}

static srt_status exclusive_scan(srt_ctx *ctx, const uint32_t *in, uint32_t *out,
                                 size_t n) {
  size_t need = 64;
  for (size_t t = (n + kScanTile - 1) / kScanTile; t > 1;
       t = (t + kScanTile - 1) / kScanTile)
    need += t + 1;
  cudaError_t e = ctx->s_scan.ensure(need * sizeof(uint32_t));
  if (e != cudaSuccess) return cuda_status(e, "scan scratch");
  return scan_levels(ctx->stream, in, out, n, ctx->s_scan.as<uint32_t>(), ctx->launches);
}

srt_status scan_exclusive(srt_ctx *ctx, const uint32_t *in, uint32_t *out, size_t n) {
  return exclusive_scan(ctx, in, out, n);
}

namespace {
// ------------------------------------------------------------------ 3. radix sort
// Digits of BITS bits: 10-bit digits sort 30-bit Morton codes in three
// passes, 8-bit digits cover full 32-bit keys in four (and the scene-id
// pass of a batched build).
constexpr int kRsMaxBins = 1 << 10;
constexpr int kRsWarps = 8;
constexpr int kRsThreads = kRsWarps * 32;
constexpr int kRsRounds = 16;
constexpr int kRsWChunk = 32 * kRsRounds;
constexpr int kRsTile = kRsWarps * kRsWChunk;

// Sort digit: BITS bits of the key from `shift`, or (SEGDIG) the segment of
// the value -- the extra pass that groups a multi-scene sort by scene.
template <bool SEGDIG, int BITS>
__device__ __forceinline__ uint32_t rs_digit(uint32_t k, uint32_t v, int shift,
                                             const uint32_t *__restrict__ seg, int nseg) {
  if (SEGDIG) return (uint32_t)seg_of(seg, nseg, v);
  return (k >> shift) & ((1u << BITS) - 1u);
}

// Per-tile digit histogram, digit-major: hist[d * ntiles + tile].
template <bool SEGDIG, int BITS>
__global__ void __launch_bounds__(kRsThreads)
rs_hist_kernel(const uint32_t *__restrict__ keys, const uint32_t *__restrict__ vals,
               size_t n, int shift, uint32_t *__restrict__ hist, uint32_t ntiles,
               const uint32_t *__restrict__ seg, int nseg) {
  constexpr int kBins = 1 << BITS;
  __shared__ uint32_t wh[kRsWarps][kBins];
  for (int i = threadIdx.x; i < kRsWarps * kBins; i += kRsThreads)
    (&wh[0][0])[i] = 0;
  __syncthreads();
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  size_t base = (size_t)blockIdx.x * kRsTile + (size_t)w * kRsWChunk;
#pragma unroll 4
  for (int r = 0; r < kRsRounds; r++) {
    size_t idx = base + (size_t)r * 32 + lane;
    bool ok = idx < n;
    unsigned valid = __ballot_sync(0xffffffffu, ok);
    (void)valid;
    if (ok) {
      const uint32_t d =
          rs_digit<SEGDIG, BITS>(keys[idx], SEGDIG ? vals[idx] : 0u, shift, seg, nseg);
      atomicAdd(&wh[w][d], 1u);
    }
  }
  __syncthreads();
  for (int d = threadIdx.x; d < kBins; d += kRsThreads) {
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < kRsWarps; k++) s += wh[k][d];
    hist[(size_t)d * ntiles + blockIdx.x] = s;
  }
}

// Stable scatter of one tile: warps own consecutive chunks, rounds go in key
// order, lanes within a round are ranked by lane order among equal digits.
template <bool SEGDIG, int BITS>
__global__ void __launch_bounds__(kRsThreads)
rs_scatter_kernel(const uint32_t *__restrict__ kin, const uint32_t *__restrict__ vin,
                  uint32_t *__restrict__ kout, uint32_t *__restrict__ vout, size_t n,
                  int shift, const uint32_t *__restrict__ offs, uint32_t ntiles,
                  const uint32_t *__restrict__ seg, int nseg) {
  constexpr int kBins = 1 << BITS;
  __shared__ uint32_t wc[kRsWarps][kBins];
  for (int i = threadIdx.x; i < kRsWarps * kBins; i += kRsThreads)
    (&wc[0][0])[i] = 0;
  __syncthreads();
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  size_t base = (size_t)blockIdx.x * kRsTile + (size_t)w * kRsWChunk;
  uint32_t k[kRsRounds], v[kRsRounds];
#pragma unroll
  for (int r = 0; r < kRsRounds; r++) {
    size_t idx = base + (size_t)r * 32 + lane;
    if (idx < n) {
      k[r] = kin[idx];
      v[r] = vin ? vin[idx] : (uint32_t)idx;
    } else {
      k[r] = 0;
      v[r] = 0;
    }
  }
  // warp histograms; peers[r] = lanes of round r with this lane's digit
  // (one ballot per digit bit)
  uint32_t dg[kRsRounds];
  unsigned peers[kRsRounds];
#pragma unroll
  for (int r = 0; r < kRsRounds; r++) {
    const size_t idx = base + (size_t)r * 32 + lane;
    const bool ok = idx < n;
    unsigned pm = __ballot_sync(0xffffffffu, ok);
    const uint32_t d = ok ? rs_digit<SEGDIG, BITS>(k[r], v[r], shift, seg, nseg) : 0u;
#pragma unroll
    for (int b = 0; b < BITS; b++) {
      const bool bit = (d >> b) & 1u;
      const unsigned m = __ballot_sync(0xffffffffu, bit);
      pm &= bit ? m : ~m;
    }
    dg[r] = d;
    peers[r] = ok ? pm : 0u;
    if (ok && lane == __ffs(pm) - 1) wc[w][d] += __popc(pm);
    __syncwarp();
  }
  __syncthreads();
  // warp start offsets: global tile offset + counts of earlier warps
  for (int d = threadIdx.x; d < kBins; d += kRsThreads) {
    uint32_t run = offs[(size_t)d * ntiles + blockIdx.x];
#pragma unroll
    for (int q = 0; q < kRsWarps; q++) {
      uint32_t c = wc[q][d];
      wc[q][d] = run;
      run += c;
    }
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < kRsRounds; r++) {
    const bool ok = peers[r] != 0u;
    const uint32_t d = dg[r];
    uint32_t pos = 0;
    if (ok) pos = wc[w][d] + __popc(peers[r] & lt);
    __syncwarp();
    if (ok) {
      kout[pos] = k[r];
      vout[pos] = v[r];
      if (lane == __ffs(peers[r]) - 1) wc[w][d] += __popc(peers[r]);
    }
    __syncwarp();
  }
}

}  // namespace

// One stable counting pass (BITS-bit key digit at `shift`, or SEGDIG: segment
// of the value) from (k0, v0) into (k1, v1).
template <bool SEGDIG, int BITS>
static srt_status sort_pass(srt_ctx *ctx, const uint32_t *k0, const uint32_t *v0,
                            uint32_t *k1, uint32_t *v1, size_t n, int shift,
                            const uint32_t *seg, int nseg) {
  cudaStream_t st = ctx->stream;
  const uint32_t ntiles = (uint32_t)((n + kRsTile - 1) / kRsTile);
  uint32_t *hist = ctx->s_hist.as<uint32_t>();
  rs_hist_kernel<SEGDIG, BITS><<<ntiles, kRsThreads, 0, st>>>(k0, v0, n, shift, hist, ntiles,
                                                              seg, nseg);
  ctx->launches++;
  srt_status s = cuda_status(cudaGetLastError(), "rs_hist");
  if (s != SRT_OK) return s;
  s = exclusive_scan(ctx, hist, hist, (size_t)(1u << BITS) * ntiles);
  if (s != SRT_OK) return s;
  rs_scatter_kernel<SEGDIG, BITS><<<ntiles, kRsThreads, 0, st>>>(k0, v0, k1, v1, n, shift,
                                                                 hist, ntiles, seg, nseg);
  ctx->launches++;
  return cuda_status(cudaGetLastError(), "rs_scatter");
}

static srt_status sort_scratch(srt_ctx *ctx, size_t n) {
  const uint32_t ntiles = (uint32_t)((n + kRsTile - 1) / kRsTile);
  cudaError_t e;
  if ((e = ctx->s_keys2.ensure(n * 4)) != cudaSuccess) return cuda_status(e, "sort");
  if ((e = ctx->s_vals2.ensure(n * 4)) != cudaSuccess) return cuda_status(e, "sort");
  if ((e = ctx->s_hist.ensure((size_t)kRsMaxBins * ntiles * 4)) != cudaSuccess)
    return cuda_status(e, "sort");
  return SRT_OK;
}

// Stable LSD sort of (keys, vals) by key; result lands back in keys/vals.
// identity_vals: vals are 0..n-1 on entry (not read).  key_bits <= 30: one
// 10-bit pass per 10 bits (three for Morton codes), otherwise four 8-bit
// passes; either way the order is the stable order by key.  With nseg > 1 a last pass groups the
// result by the segment of each value (the segment offsets `seg` are global
// indices), i.e. the order is (segment, key, value).
srt_status sort_pairs_seg(srt_ctx *ctx, uint32_t *keys, uint32_t *vals, size_t n,
                          bool identity_vals, const uint32_t *seg, int nseg, int key_bits) {
  if (n == 0) return SRT_OK;
  srt_status s = sort_scratch(ctx, n);
  if (s != SRT_OK) return s;
  uint32_t *k0 = keys, *v0 = vals, *k1 = ctx->s_keys2.as<uint32_t>(),
           *v1 = ctx->s_vals2.as<uint32_t>();
  const bool narrow = key_bits <= 30;
  const int passes = narrow ? (key_bits < 1 ? 1 : (key_bits + 9) / 10) : 4;
  for (int pass = 0; pass < passes; pass++) {
    const uint32_t *vin = (pass == 0 && identity_vals) ? nullptr : v0;
    s = narrow ? sort_pass<false, 10>(ctx, k0, vin, k1, v1, n, pass * 10, nullptr, 0)
               : sort_pass<false, 8>(ctx, k0, vin, k1, v1, n, pass * 8, nullptr, 0);
    if (s != SRT_OK) return s;
    std::swap(k0, k1);
    std::swap(v0, v1);
  }
  if (nseg > 1) {
    s = sort_pass<true, 8>(ctx, k0, v0, k1, v1, n, 0, seg, nseg);
    if (s != SRT_OK) return s;
    std::swap(k0, k1);
    std::swap(v0, v1);
  }
  if (k0 != keys) {  // an odd number of passes ends in the scratch
    cudaError_t e = cudaMemcpyAsync(keys, k0, n * 4, cudaMemcpyDeviceToDevice, ctx->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(vals, v0, n * 4, cudaMemcpyDeviceToDevice, ctx->stream);
    if (e != cudaSuccess) return cuda_status(e, "sort copy");
  }
  return SRT_OK;
}

srt_status sort_pairs(srt_ctx *ctx, uint32_t *keys, uint32_t *vals, size_t n,
                      bool identity_vals, int key_bits) {
  return sort_pairs_seg(ctx, keys, vals, n, identity_vals, nullptr, 1, key_bits);
}

namespace {
// ------------------------------------------------------------------ 4. Karras
// Delta30 (render/render_prefix_tree_util.cc:501-526).
__device__ __forceinline__ int kdelta(const uint32_t *__restrict__ c, int i, int j,
                                      int n) {
  if (j < 0 || j >= n) return -1;
  uint32_t a = __ldg(&c[i]), b = __ldg(&c[j]);
  if (a == b) return 32 + __clz((uint32_t)i ^ (uint32_t)j);
  return __clz(a ^ b);
}

// ConstructBinaryRadixTree30 for every internal node; also records ranges
// and parent links for the bottom-up pass.
__global__ void karras_kernel(const uint32_t *__restrict__ codes, int n,
                              uint32_t *__restrict__ kchild, uint8_t *__restrict__ kflags,
                              uint2 *__restrict__ krange, uint32_t *__restrict__ kparent,
                              uint32_t *__restrict__ lparent,
                              unsigned long long *__restrict__ ticket = nullptr,
                              uint8_t *__restrict__ kprefix = nullptr) {
  // the tile counter of level_scan_kernel, which follows on the stream
  if (ticket && blockIdx.x == 0 && threadIdx.x == 0) *ticket = 0ull;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n - 1;
       i += gridDim.x * blockDim.x) {
    int d = (kdelta(codes, i, i + 1, n) - kdelta(codes, i, i - 1, n)) >= 0 ? 1 : -1;
    int dmin = kdelta(codes, i, i - d, n);
    int lmax = 2;
    while (kdelta(codes, i, i + lmax * d, n) > dmin) lmax *= 2;
    int l = 0;
    for (int t = lmax / 2; t >= 1; t /= 2)
      if (kdelta(codes, i, i + (l + t) * d, n) > dmin) l += t;
    int j = i + l * d;
    int dnode = kdelta(codes, i, j, n);
    int s = 0;
    for (int k = 2;; k *= 2) {  // t = ceil(l/2), ceil(l/4), ..., 1
      int t = (l + k - 1) / k;
      if (t <= 0) break;
      if (kdelta(codes, i, i + (s + t) * d, n) > dnode) s += t;
      if (t == 1) break;
    }
    int g = i + s * d + (d < 0 ? d : 0);
    int lo = i < j ? i : j, hi = i < j ? j : i;
    bool lleaf = (lo == g), rleaf = (hi == g + 1);
    if (kchild) kchild[i] = (uint32_t)g;
    kflags[i] = (uint8_t)((lleaf ? 1 : 0) | (rleaf ? 2 : 0));
    if (kprefix) kprefix[i] = (uint8_t)dnode;  // <= 64
    if (krange) krange[i] = make_uint2((uint32_t)lo, (uint32_t)hi);
    if (kparent) {
      if (!lleaf) kparent[g] = (uint32_t)i;
      else if (lparent) lparent[g] = (uint32_t)i;
      if (!rleaf) kparent[g + 1] = (uint32_t)i;
      else if (lparent) lparent[g + 1] = (uint32_t)i;
      if (i == 0) kparent[0] = kNone;
    }
  }
}

// ------------------------------------------------------------------ 5. refit
// Leaf-ordered primitive cache: thread per sorted position j gathers the
// primitive's vertices (or centre and radius) once.
template <int KIND>
__global__ void cache_kernel(const float *__restrict__ v, const uint32_t *__restrict__ f,
                             const float *__restrict__ radius, float constr,
                             const uint32_t *__restrict__ sidx, int n,
                             float4 *__restrict__ prims) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    const uint32_t p = sidx[j];
    if (KIND == SRT_TRIANGLES) {
      const size_t a = f[3 * (size_t)p], b = f[3 * (size_t)p + 1], c = f[3 * (size_t)p + 2];
      prims[3 * (size_t)j + 0] = make_float4(v[3 * a], v[3 * a + 1], v[3 * a + 2],
                                             __uint_as_float(p));
      prims[3 * (size_t)j + 1] = make_float4(v[3 * b], v[3 * b + 1], v[3 * b + 2], 0.0f);
      prims[3 * (size_t)j + 2] = make_float4(v[3 * c], v[3 * c + 1], v[3 * c + 2], 0.0f);
    } else if (KIND == SRT_TETRAHEDRA) {
      float x[12];
#pragma unroll
      for (int c = 0; c < 4; c++) {
        const size_t q = f[4 * (size_t)p + c];
        x[3 * c] = v[3 * q];
        x[3 * c + 1] = v[3 * q + 1];
        x[3 * c + 2] = v[3 * q + 2];
      }
      prims[3 * (size_t)j + 0] = make_float4(x[0], x[1], x[2], x[3]);
      prims[3 * (size_t)j + 1] = make_float4(x[4], x[5], x[6], x[7]);
      prims[3 * (size_t)j + 2] = make_float4(x[8], x[9], x[10], x[11]);
    } else {
      const float r = radius ? radius[p] : constr;
      prims[j] = make_float4(v[3 * (size_t)p], v[3 * (size_t)p + 1], v[3 * (size_t)p + 2], r);
    }
  }
}

// Box of the sorted primitive range [lo, hi] in order -- ComputeBoundingBox30
// (render/render_accel_triangle.cc:661-709): the first value seen wins ties,
// as the left-first merges of MergeBoundingBox do.
template <int KIND, typename P = float4>
__device__ __forceinline__ Box range_box(const P *__restrict__ prims, uint32_t lo,
                                         uint32_t hi, float keps) {
  // groups of four primitives: their loads are issued together
  constexpr int kGroup = 4;
  Box b = cache_box<KIND>(prims, lo, keps);
  for (uint32_t j = lo + 1; j <= hi; j += kGroup) {
    Box bx[kGroup];
#pragma unroll
    for (int q = 0; q < kGroup; q++)
      if (j + q <= hi) bx[q] = cache_box<KIND>(prims, j + q, keps);
#pragma unroll
    for (int q = 0; q < kGroup; q++)
      if (j + q <= hi) b = box_merge(b, bx[q]);
  }
  return b;
}

// Internal-node boxes of the build: 32 bytes each, two 16-byte words
// (lo.x, lo.y, lo.z, hi.x), (hi.y, hi.z, -, -).
struct __align__(16) BoxP {
  float4 a, b;
};
__device__ __forceinline__ BoxP box_pack(const Box &x) {
  BoxP p;
  p.a = make_float4(x.lo[0], x.lo[1], x.lo[2], x.hi[0]);
  p.b = make_float4(x.hi[1], x.hi[2], 0.0f, 0.0f);
  return p;
}
__device__ __forceinline__ Box box_unpack(const float4 a, const float4 b) {
  Box x;
  x.lo[0] = a.x; x.lo[1] = a.y; x.lo[2] = a.z;
  x.hi[0] = a.w; x.hi[1] = b.x; x.hi[2] = b.y;
  return x;
}
// A box written by another thread of the running kernel (after the acquire
// of the arrival counter): read through L2.
__device__ __forceinline__ Box ibox_load(const BoxP *__restrict__ ibox, uint32_t c) {
  const float4 *q = reinterpret_cast<const float4 *>(ibox + c);
  return box_unpack(__ldcg(q), __ldcg(q + 1));
}
__device__ __forceinline__ void ibox_store(BoxP *__restrict__ ibox, uint32_t c, const Box &x) {
  const BoxP p = box_pack(x);
  float4 *q = reinterpret_cast<float4 *>(ibox + c);
  __stcg(q, p.a);
  __stcg(q + 1, p.b);
}
// Arrival at a node's two-child counter: release this thread's box stores,
// acquire the other child's; returns the count before this arrival.
__device__ __forceinline__ uint32_t arrive(uint32_t *counter) {
  uint32_t old;
  asm volatile("atom.add.acq_rel.gpu.global.u32 %0, [%1], 1;"
               : "=r"(old) : "l"(counter) : "memory");
  return old;
}

// Boxes of the emitted tree only.  Thread per emitted branch (Karras internal
// node i = kidx[slot]): children that become leaves of the emitted
// tree get their box here -- a Karras leaf from the cache, a collapsed
// subtree c by range_box into ibox[c] -- and branch boxes are merged bottom
// up, left first, by the second of the two children to finish (arrival
// counter per node), each climb carrying its own box and reading only the
// sibling's.  Ancestors of an emitted branch are emitted branches.
template <int KIND, typename P = float4>
__global__ void __launch_bounds__(256)
refit_kernel(const uint32_t *__restrict__ kchild, const uint8_t *__restrict__ kflags,
             const uint2 *__restrict__ krange, const uint32_t *__restrict__ kparent,
             const uint32_t *__restrict__ flag, const uint32_t *__restrict__ kidx, int n,
             const SceneInfo *__restrict__ scene, const P *__restrict__ prims,
             uint32_t *__restrict__ counter, BoxP *__restrict__ ibox,
             uint32_t *__restrict__ err) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= scene->nbranches) return;
  const uint32_t i = __ldg(&kidx[t]);  // the emitted branches are dense in slot order
  const float keps = scene->keps;
  const uint32_t g = __ldg(&kchild[i]);
  const uint8_t fl = __ldg(&kflags[i]);
  bool leafside[2];
  Box lb[2];
#pragma unroll
  for (int side = 0; side < 2; side++) {
    const uint32_t c = g + side;
    const bool kleaf = fl & (1 << side);
    leafside[side] = kleaf || !__ldg(&flag[c]);
    if (kleaf) {
      lb[side] = cache_box<KIND>(prims, c, keps);
    } else if (leafside[side]) {  // collapsed subtree: one emitted leaf
      const uint2 r = __ldg(&krange[c]);
      lb[side] = range_box<KIND, P>(prims, r.x, r.y, keps);
      ibox_store(ibox, c, lb[side]);  // for the emission, and a sibling's climb
    }
  }
  if (!leafside[0] && !leafside[1]) return;  // two branch children climb here
  Box mine;
  if (leafside[0] && leafside[1]) {
    mine = box_merge(lb[0], lb[1]);
  } else {
    // one leaf child (a collapsed subtree's box is in its own slot already; a
    // Karras leaf's is read from the cache by whoever merges): meet the
    // branch child's climb
    const int ls = leafside[0] ? 0 : 1;
    const Box lbox = ls == 0 ? lb[0] : lb[1];
    if (arrive(&counter[i]) == 0) return;
    const Box bb = ibox_load(ibox, g + (1 - ls));
    mine = ls == 0 ? box_merge(lbox, bb) : box_merge(bb, lbox);
  }
  // climb: per level one arrival and one sibling-box read; the parent's
  // parent and split are loaded ahead, alongside the arrival
  uint32_t node = i;
  uint32_t q = node == 0 ? kNone : __ldg(&kparent[node]);
  for (int guard = 0; guard < 64; guard++) {
    ibox_store(ibox, node, mine);
    if (node == 0 || q == kNone) return;
    const uint32_t gq = __ldg(&kchild[q]);
    const uint8_t fq = __ldg(&kflags[q]);
    const uint32_t qnext = q == 0 ? kNone : __ldg(&kparent[q]);
    if (arrive(&counter[q]) == 0) return;
    const bool left = (gq == node) && !(fq & 1);
    const uint32_t sib = left ? gq + 1 : gq;
    const bool sib_kleaf = left ? (fq & 2) : (fq & 1);
    const Box sb = sib_kleaf ? cache_box<KIND>(prims, sib, keps) : ibox_load(ibox, sib);
    mine = left ? box_merge(mine, sb) : box_merge(sb, mine);
    node = q;
    q = qnext;
  }
  atomicOr(err, kErrTree);
}

// ------------------------------------------------------------------ 6. levels
// flag[i] = 1 iff Karras internal node i is emitted as a branch: its range
// holds more than max_leaf + 1 keys and it lies at level <= 23 (the root is
// always split).
// The same flags, their exclusive prefix sum (the emitted branches' node slots, in Karras index
// order), the inverse map kidx (slot -> Karras node) and the branch count,
// in one pass: tiles of
// 1024 nodes in ticket order, each adding the flagged counts of earlier tiles
// by look-back (64-bit words: epoch, flag bits 30-31, count).  Also zeroes
// the refit's arrival counters.  Waits are bounded (kErrSortWait).
constexpr int kLsThreads = 256;
constexpr int kLsItems = 4;
constexpr int kLsTile = kLsThreads * kLsItems;

__global__ void __launch_bounds__(kLsThreads)
level_scan_kernel(const uint2 *__restrict__ krange, const uint32_t *__restrict__ kparent,
                  const uint8_t *__restrict__ kprefix, int n, int max_leaf,
                  uint32_t *__restrict__ flag,
                  uint32_t *__restrict__ slot, uint32_t *__restrict__ kidx,
                  uint32_t *__restrict__ counter,
                  unsigned long long *__restrict__ status, unsigned long long *__restrict__ ticket,
                  uint32_t epoch, SceneInfo *__restrict__ scene, uint32_t *__restrict__ err) {
  __shared__ uint32_t s_tile, s_prefix, s_warp[kLsThreads / 32];
  if (threadIdx.x == 0) s_tile = (uint32_t)atomicAdd(ticket, 1ull);
  __syncthreads();
  const uint32_t tile = s_tile;
  if (tile >= gridDim.x) {  // a counter left over from a failed launch
    if (threadIdx.x == 0) atomicOr(err, kErrSortWait);
    return;
  }
  const uint32_t m = (uint32_t)n - 1u;
  const uint32_t base = tile * (uint32_t)kLsTile + threadIdx.x * (uint32_t)kLsItems;
  // Each level down a root path lengthens the common prefix of the range's
  // (code, index) keys by at least one bit, so a node's depth is at most its
  // prefix length minus the root's: within the level cap there, no parent
  // walk is needed.
  const int root_prefix = __ldg(&kprefix[0]);
  uint32_t f[kLsItems];
#pragma unroll
  for (int q = 0; q < kLsItems; q++) {
    const uint32_t i = base + q;
    f[q] = 0;
    if (i >= m) continue;
    counter[i] = 0;
    const uint2 r = __ldg(&krange[i]);
    if (i == 0) {
      f[q] = 1;  // Build32 always splits the root
    } else if (r.y - r.x > (uint32_t)max_leaf) {
      if ((int)__ldg(&kprefix[i]) - root_prefix <= kMaxLevel) {
        f[q] = 1u;
      } else {
        int lvl = 0;
        uint32_t x = i;
        while (x != 0 && lvl <= kMaxLevel) {
          x = __ldg(&kparent[x]);
          lvl++;
        }
        f[q] = (lvl <= kMaxLevel) ? 1u : 0u;
      }
    }
  }
  // exclusive scan within the tile
  uint32_t x[kLsItems], sum = 0;
#pragma unroll
  for (int q = 0; q < kLsItems; q++) {
    x[q] = sum;
    sum += f[q];
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  uint32_t inc = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += y;
  }
  if (lane == 31) s_warp[w] = inc;
  __syncthreads();
  uint32_t wbase = 0, total = 0;
#pragma unroll
  for (int k = 0; k < kLsThreads / 32; k++) {
    const uint32_t v = s_warp[k];
    if (k < w) wbase += v;
    total += v;
  }
  if (threadIdx.x == 0) {
    const unsigned long long ep = (unsigned long long)epoch << 32;
    constexpr uint32_t kAgg = 1u << 30, kInc = 2u << 30, kCnt = (1u << 30) - 1u;
    unsigned long long *mine = status + tile;
    uint32_t prefix = 0;
    if (tile == 0) {
      asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(mine), "l"(ep | kInc | total)
                   : "memory");
    } else {
      asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(mine), "l"(ep | kAgg | total)
                   : "memory");
      int j = (int)tile - 1;
      uint32_t spins = 0;
      while (j >= 0) {
        unsigned long long v;
        asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(status + j)
                     : "memory");
        if ((uint32_t)(v >> 32) != epoch) {
          if (++spins > (1u << 22)) {
            atomicOr(err, kErrSortWait);
            break;
          }
          __nanosleep(64);
          continue;
        }
        prefix += (uint32_t)v & kCnt;
        if ((uint32_t)v & kInc) break;
        j--;
      }
      asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(mine),
                   "l"(ep | kInc | ((prefix + total) & kCnt)) : "memory");
    }
    s_prefix = prefix;
    if (tile == gridDim.x - 1) scene->nbranches = prefix + total;
  }
  __syncthreads();
  const uint32_t off = s_prefix + wbase + inc - sum;
#pragma unroll
  for (int q = 0; q < kLsItems; q++) {
    const uint32_t i = base + q;
    if (i < m) {
      flag[i] = f[q];
      slot[i] = off + x[q];
      if (f[q]) kidx[off + x[q]] = i;  // emitted branches in slot order
    }
  }
}

// ------------------------------------------------------------------ 7. emission
template <int KIND, typename P = float4>
__device__ __forceinline__ void child_info(uint32_t c, bool kleaf,
                                           const uint2 *__restrict__ krange,
                                           const uint32_t *__restrict__ flag,
                                           const uint32_t *__restrict__ slot,
                                           const BoxP *__restrict__ ibox,
                                           const P *__restrict__ prims, float keps,
                                           Box &box, bool &is_branch, uint32_t &ref,
                                           uint32_t &count) {
  if (kleaf) {
    box = cache_box<KIND>(prims, c, keps);
    is_branch = false;
    ref = c;
    count = 1;
    return;
  }
  box = box_unpack(__ldg(&ibox[c].a), __ldg(&ibox[c].b));
  if (flag[c]) {
    is_branch = true;
    ref = slot[c];
    count = 0;
  } else {
    uint2 r = krange[c];
    is_branch = false;
    ref = r.x;
    count = r.y - r.x + 1;
  }
}

template <int KIND>
__global__ void emit_node2_kernel(const uint32_t *__restrict__ codes,
                                  const uint32_t *__restrict__ kchild,
                                  const uint8_t *__restrict__ kflags,
                                  const uint2 *__restrict__ krange,
                                  const uint32_t *__restrict__ flag,
                                  const uint32_t *__restrict__ slot,
                                  const BoxP *__restrict__ ibox,
                                  const float4 *__restrict__ prims,
                                  const SceneInfo *__restrict__ scene,
                                  const uint32_t *__restrict__ kidx,
                                  Node2 *__restrict__ nodes, uint32_t *__restrict__ err) {
  const float keps = scene->keps;
  const uint32_t nb = scene->nbranches;
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < nb;
       t += gridDim.x * blockDim.x) {
    const uint32_t i = __ldg(&kidx[t]);
    uint32_t g = kchild[i];
    uint8_t fl = kflags[i];
    Box b0, b1;
    bool br0, br1;
    uint32_t r0, r1, c0, c1;
    child_info<KIND>(g, fl & 1, krange, flag, slot, ibox, prims, keps, b0, br0, r0, c0);
    child_info<KIND>(g + 1, fl & 2, krange, flag, slot, ibox, prims, keps, b1, br1, r1, c1);
    if (c0 > kCountMask || c1 > kCountMask) atomicOr(err, kErrTree);
    uint32_t axis = (uint32_t)split_axis(codes[i]);
    Node2 nd;
    nd.a = make_float4(b0.lo[0], b0.lo[1], b0.lo[2], b0.hi[0]);
    nd.b = make_float4(b0.hi[1], b0.hi[2], b1.lo[0], b1.lo[1]);
    nd.c = make_float4(b1.lo[2], b1.hi[0], b1.hi[1], b1.hi[2]);
    nd.d = make_uint4(r0, r1, (c0 & kCountMask) | (axis << 30), c1 & kCountMask);
    nodes[t] = nd;  // slot[i] == t
  }
}

__device__ __forceinline__ NodeT make_tet_node(const Box &b, uint32_t meta, uint32_t ref) {
  NodeT t;
  t.a = make_float4(b.lo[0], b.lo[1], b.lo[2], __uint_as_float(meta));
  t.b = make_float4(b.hi[0], b.hi[1], b.hi[2], __uint_as_float(ref));
  return t;
}

template <typename P = float4>
__global__ void emit_tet_kernel(const uint32_t *__restrict__ codes,
                                const uint32_t *__restrict__ kchild,
                                const uint8_t *__restrict__ kflags,
                                const uint2 *__restrict__ krange,
                                const uint32_t *__restrict__ flag,
                                const uint32_t *__restrict__ slot,
                                const BoxP *__restrict__ ibox,
                                const P *__restrict__ prims,
                                const SceneInfo *__restrict__ scene,
                                const uint32_t *__restrict__ kidx,
                                NodeT *__restrict__ nodes, uint32_t *__restrict__ err) {
  const float keps = scene->keps;
  const uint32_t nb = scene->nbranches;
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < nb;
       t += gridDim.x * blockDim.x) {
    const uint32_t i = __ldg(&kidx[t]);
    const uint32_t s = t;  // slot[i]
    if (i == 0)
      nodes[0] = make_tet_node(box_unpack(__ldg(&ibox[0].a), __ldg(&ibox[0].b)),
                               (uint32_t)split_axis(codes[0]), 1u);
    uint32_t g = kchild[i];
    uint8_t fl = kflags[i];
#pragma unroll
    for (int side = 0; side < 2; side++) {
      uint32_t c = g + side;
      Box b;
      bool br;
      uint32_t ref, cnt;
      child_info<SRT_TETRAHEDRA, P>(c, fl & (1 << side), krange, flag, slot, ibox, prims,
                                 keps, b, br, ref, cnt);
      uint32_t meta, r;
      if (br) {
        meta = (uint32_t)split_axis(codes[c]);
        r = 1u + 2u * ref;
      } else {
        if (cnt > kCountMask) atomicOr(err, kErrTree);
        meta = kLeafBit | cnt;
        r = ref;
      }
      nodes[1 + 2 * (size_t)s + side] = make_tet_node(b, meta, r);
    }
  }
}


// Scene box and Morton codes.  With `hist` (3 x 1024 words) and `tickets`,
// also the digit histograms of sort_codes30's passes (hist_ready).
template <int KIND>
srt_status launch_bbox_morton(srt_ctx *ctx, const float *v, const uint32_t *f,
                              const float *radius, float constr, size_t n,
                              SceneInfo *scene, uint32_t *codes, uint32_t *index,
                              uint32_t *hist = nullptr,
                              unsigned long long *tickets = nullptr) {
  cudaStream_t st = ctx->stream;
  int gb = grid_for(n, kBlock, ctx->num_sms * (n > (4u << 20) ? 4 : 1));
  cudaError_t e = ctx->s_partial.ensure((size_t)gb * sizeof(Box));
  if (e != cudaSuccess) return cuda_status(e, "bbox scratch");
  Box *partial = ctx->s_partial.as<Box>();
  bbox_partial_kernel<KIND><<<gb, kBlock, 0, st>>>(v, f, radius, constr, n, partial, hist,
                                                   tickets);
  ctx->launches++;
  if (hist) {
    const int gm = grid_for(n, kBlock, ctx->num_sms * 8);
    morton_hist_kernel<KIND><<<gm, kBlock, 0, st>>>(v, f, n, partial, gb, scene, codes, hist);
    ctx->launches++;
    return cuda_status(cudaGetLastError(), "bbox/morton");
  }
  bbox_final_kernel<KIND><<<1, 32, 0, st>>>(partial, gb, scene);
  ctx->launches++;
  int gm = grid_for(n, kBlock, ctx->num_sms * 16);
  morton_kernel<KIND><<<gm, kBlock, 0, st>>>(v, f, n, scene, codes, index);
  ctx->launches++;
  return cuda_status(cudaGetLastError(), "bbox/morton");
}

constexpr size_t kOneSweepMax = (size_t)1 << 18;

template <int KIND>
srt_status build_kind(srt_accel *a, const float *v, const uint32_t *f,
                      const float *radius, float constr, size_t n) {
  srt_ctx *ctx = a->ctx;
  cudaStream_t st = ctx->stream;
  cudaError_t e;
  const int in = (int)n;
  const size_t m = n - 1;  // internal nodes
#define ENSURE(buf, bytes)                                   \
  do {                                                       \
    if ((e = (buf).ensure(bytes)) != cudaSuccess)            \
      return cuda_status(e, "build allocation " #buf);       \
  } while (0)
  ENSURE(a->codes, n * 4);
  ENSURE(a->indices, n * 4);
  ENSURE(a->prims, n * sizeof(float4) * PrimTraits<KIND>::kCacheF4);
  ENSURE(a->scene, sizeof(SceneInfo));
  size_t max_nodes = (KIND == SRT_TETRAHEDRA) ? (2 * m + 1) : m;
  ENSURE(a->nodes, max_nodes * (KIND == SRT_TETRAHEDRA ? sizeof(NodeT) : sizeof(Node2)));

  ENSURE(ctx->s_kchild, m * 4);
  ENSURE(ctx->s_kflags, m);
  ENSURE(ctx->s_krange, m * sizeof(uint2));
  ENSURE(ctx->s_kparent, m * 4);
  ENSURE(ctx->s_counter, m * 4);
  ENSURE(ctx->s_ibox, (m + 1) * sizeof(BoxP));
  ENSURE(ctx->s_kidx, m * 4);
  ENSURE(ctx->s_kprefix, m);
  ENSURE(ctx->s_flag, m * 4);
  ENSURE(ctx->s_slot, m * 4);
#undef ENSURE
#define ENSURE2(buf, bytes)                                  \
  do {                                                       \
    if ((e = (buf).ensure(bytes)) != cudaSuccess)            \
      return cuda_status(e, "build allocation " #buf);       \
  } while (0)
  SceneInfo *scene = a->scene.as<SceneInfo>();
  uint32_t *codes = a->codes.as<uint32_t>();
  uint32_t *idx = a->indices.as<uint32_t>();
  // Morton codes, then their stable sort: up to kOneSweepMax keys with one
  // look-back kernel per digit pass (the Morton kernel fills its digit
  // histograms), larger arrays with the histogram / scan / scatter passes,
  // which keep more of the GPU busy per pass at those sizes (measured)
  srt_status s;
  if (n <= kOneSweepMax) {
    uint32_t *hist = nullptr;
    unsigned long long *tickets = nullptr;
    s = sort_codes30_scratch(ctx, n, &hist, &tickets);
    if (s != SRT_OK) return s;
    s = launch_bbox_morton<KIND>(ctx, v, f, radius, constr, n, scene, codes, nullptr, hist,
                                 tickets);
    if (s != SRT_OK) return s;
    s = sort_codes30(ctx, codes, idx, n, true, true);
  } else {
    s = launch_bbox_morton<KIND>(ctx, v, f, radius, constr, n, scene, codes, nullptr);
    if (s != SRT_OK) return s;
    s = sort_pairs(ctx, codes, idx, n, true, 30);
  }
  if (s != SRT_OK) return s;
  uint32_t *kchild = ctx->s_kchild.as<uint32_t>();
  uint8_t *kflags = ctx->s_kflags.as<uint8_t>();
  uint2 *krange = ctx->s_krange.as<uint2>();
  uint32_t *kparent = ctx->s_kparent.as<uint32_t>();
  uint32_t *counter = ctx->s_counter.as<uint32_t>();
  BoxP *ibox = ctx->s_ibox.as<BoxP>();
  uint32_t *kidx = ctx->s_kidx.as<uint32_t>();
  uint32_t *flag = ctx->s_flag.as<uint32_t>();
  uint32_t *slot = ctx->s_slot.as<uint32_t>();
  // level-scan look-back words (ticket + one per tile; zero when allocated)
  const uint32_t ltiles = (uint32_t)((m + kLsTile - 1) / kLsTile);
  const size_t lbytes = 256 + (size_t)ltiles * 8;
  if (lbytes > ctx->s_lscan.cap || !ctx->s_lscan.p) {
    ENSURE2(ctx->s_lscan, lbytes);
    if ((e = cudaMemsetAsync(ctx->s_lscan.p, 0, ctx->s_lscan.cap, st)) != cudaSuccess)
      return cuda_status(e, "level scan");
  }
  unsigned long long *lticket = ctx->s_lscan.as<unsigned long long>();
  unsigned long long *lstatus =
      reinterpret_cast<unsigned long long *>(ctx->s_lscan.as<char>() + 256);
  int gk = grid_for(m, kBlock, ctx->num_sms * 16);
  uint8_t *kprefix = ctx->s_kprefix.as<uint8_t>();
  karras_kernel<<<gk, kBlock, 0, st>>>(codes, in, kchild, kflags, krange, kparent, nullptr,
                                       lticket, kprefix);
  const uint32_t lepoch = ++ctx->os_epoch == 0 ? ++ctx->os_epoch : ctx->os_epoch;
  level_scan_kernel<<<ltiles, kLsThreads, 0, st>>>(krange, kparent, kprefix, in,
                                                   PrimTraits<KIND>::kMaxLeaf, flag, slot,
                                                   kidx, counter, lstatus, lticket, lepoch,
                                                   scene, ctx->d_err);
  cache_kernel<KIND><<<grid_for(n, kBlock, ctx->num_sms * 16), kBlock, 0, st>>>(
      v, f, radius, constr, idx, in, a->prims.as<float4>());
  refit_kernel<KIND><<<(unsigned)((m + kBlock - 1) / kBlock), kBlock, 0, st>>>(
      kchild, kflags, krange, kparent, flag, kidx, in, scene, a->prims.as<float4>(), counter,
      ibox, ctx->d_err);
  ctx->launches += 4;
  s = cuda_status(cudaGetLastError(), "karras/level/cache/refit");
  if (s != SRT_OK) return s;
  if (KIND == SRT_TETRAHEDRA) {
    emit_tet_kernel<<<gk, kBlock, 0, st>>>(codes, kchild, kflags, krange, flag, slot, ibox,
                                           a->prims.as<float4>(), scene, kidx,
                                           a->nodes.as<NodeT>(), ctx->d_err);
    ctx->launches++;
  } else {
    emit_node2_kernel<KIND><<<gk, kBlock, 0, st>>>(codes, kchild, kflags, krange, flag,
                                                   slot, ibox, a->prims.as<float4>(),
                                                   scene, kidx, a->nodes.as<Node2>(),
                                                   ctx->d_err);
    ctx->launches++;
  }
#undef ENSURE2
  return cuda_status(cudaGetLastError(), "emit");
}

}  // namespace

// Build32 of tetrahedra with double-precision positions (the reference's
// isDoublePrecisionPos, render/render_accel_tetra.cc:1621-1660): the scene
// box pads each double coordinate in double and rounds to float, the Morton
// codes take the positions rounded to float (CalculateMortonCodesTetraDouble30
// builds real3 from them), leaf boxes pad the doubles again, and the
// primitive cache keeps the doubles for the Pluecker tests.  vf (3 * nverts
// floats) receives the rounded positions.
srt_status build_tet_double(srt_accel *a, const double *dv, size_t nverts, const uint32_t *f,
                            size_t n, float *vf) {
  srt_ctx *ctx = a->ctx;
  cudaStream_t st = ctx->stream;
  cudaError_t e;
  const size_t m = n - 1;
  if ((e = a->codes.ensure(n * 4)) != cudaSuccess || (e = a->indices.ensure(n * 4)) != cudaSuccess ||
      (e = a->prims.ensure(n * 6 * sizeof(double2))) != cudaSuccess ||
      (e = a->scene.ensure(sizeof(SceneInfo))) != cudaSuccess ||
      (e = a->nodes.ensure((2 * m + 1) * sizeof(NodeT))) != cudaSuccess ||
      (e = ctx->s_ibox.ensure((m + 1) * sizeof(BoxP))) != cudaSuccess)
    return cuda_status(e, "build allocation");
  SceneInfo *scene = a->scene.as<SceneInfo>();
  uint32_t *codes = a->codes.as<uint32_t>(), *idx = a->indices.as<uint32_t>();
  round_vertices_kernel<<<grid_for(3 * nverts, kBlock, ctx->num_sms * 16), kBlock, 0, st>>>(
      dv, 3 * nverts, vf);
  const int gb = grid_for(n, kBlock, ctx->num_sms * (n > (4u << 20) ? 4 : 1));
  if ((e = ctx->s_partial.ensure((size_t)gb * sizeof(Box))) != cudaSuccess)
    return cuda_status(e, "bbox scratch");
  Box *partial = ctx->s_partial.as<Box>();
  bbox_partial_tet_d_kernel<<<gb, kBlock, 0, st>>>(dv, f, n, partial);
  bbox_final_kernel<SRT_TETRAHEDRA><<<1, 32, 0, st>>>(partial, gb, scene);
  morton_kernel<SRT_TETRAHEDRA><<<grid_for(n, kBlock, ctx->num_sms * 16), kBlock, 0, st>>>(
      vf, f, n, scene, codes, nullptr);
  ctx->launches += 4;
  srt_status s = cuda_status(cudaGetLastError(), "bbox/morton");
  if (s != SRT_OK) return s;
  if ((s = sort_pairs(ctx, codes, idx, n, true, 30)) != SRT_OK) return s;
  Topology T;
  if ((s = stage_topology(ctx, codes, n, PrimTraits<SRT_TETRAHEDRA>::kMaxLeaf, scene, T)) !=
      SRT_OK)
    return s;
  double2 *prims = a->prims.as<double2>();
  BoxP *ibox = ctx->s_ibox.as<BoxP>();
  cache_tet_d_kernel<<<grid_for(n, kBlock, ctx->num_sms * 16), kBlock, 0, st>>>(dv, f, idx,
                                                                               (int)n, prims);
  refit_kernel<SRT_TETRAHEDRA, double2><<<(unsigned)((m + kBlock - 1) / kBlock), kBlock, 0, st>>>(
      T.kchild, T.kflags, T.krange, T.kparent, T.flag, T.kidx, (int)n, scene, prims, T.counter,
      ibox, ctx->d_err);
  const int gk = grid_for(m, kBlock, ctx->num_sms * 16);
  emit_tet_kernel<double2><<<gk, kBlock, 0, st>>>(codes, T.kchild, T.kflags, T.krange, T.flag,
                                                  T.slot, ibox, prims, scene, T.kidx,
                                                  a->nodes.as<NodeT>(), ctx->d_err);
  ctx->launches += 3;
  return cuda_status(cudaGetLastError(), "tetrahedra (double)");
}

namespace {

}  // namespace

namespace {
// =================================================================== batches
// Many scenes in one build: primitives of scene s are the global range
// [foff[s], foff[s+1]); its Karras internal nodes the global range
// [ioff[s], ioff[s+1]) with ioff[s] = foff[s] - s.  Every stage runs once
// over all scenes and computes exactly the per-scene build: boxes, Morton
// codes and trees use each scene's own box and local key positions.

__device__ __forceinline__ int f2o(float f) {  // order-preserving float -> int
  const int i = __float_as_int(f);
  return i >= 0 ? i : i ^ 0x7fffffff;
}
__device__ __forceinline__ float o2f(int i) { return __int_as_float(i >= 0 ? i : i ^ 0x7fffffff); }

// Block-wide box reduction; the result is valid in thread 0.
__device__ Box block_reduce_box(Box b) {
  __shared__ Box sh[32];
#pragma unroll
  for (int k = 0; k < 3; k++) {
    for (int o = 16; o > 0; o >>= 1) {
      b.lo[k] = fmin_ref(b.lo[k], __shfl_down_sync(0xffffffffu, b.lo[k], o));
      b.hi[k] = fmax_ref(b.hi[k], __shfl_down_sync(0xffffffffu, b.hi[k], o));
    }
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) sh[w] = b;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int i = 1; i < (int)(blockDim.x >> 5); i++) b = box_merge(b, sh[i]);
  }
  __syncthreads();
  return b;
}

__global__ void seg_bbox_init_kernel(int *__restrict__ acc, int nseg) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < 6 * nseg; i += gridDim.x * blockDim.x)
    acc[i] = (i % 6) < 3 ? INT_MAX : INT_MIN;
}

constexpr int kSegTile = 2048;

template <int KIND>
__global__ void seg_bbox_kernel(const float *__restrict__ v, const uint32_t *__restrict__ f,
                                const uint32_t *__restrict__ foff, int nseg, uint32_t N,
                                int *__restrict__ acc) {
  const uint32_t t0 = blockIdx.x * kSegTile;
  if (t0 >= N) return;
  const uint32_t t1 = min(N, t0 + kSegTile);
  const int s0 = seg_of(foff, nseg, t0), s1 = seg_of(foff, nseg, t1 - 1);
  const float e = (KIND == SRT_TRIANGLES) ? 0.0f : FLT_EPSILON * 16;
  const int nv = (KIND == SRT_TRIANGLES) ? 3 : 4;
  for (int sg = s0; sg <= s1; sg++) {
    const uint32_t lo = max(t0, __ldg(&foff[sg])), hi = min(t1, __ldg(&foff[sg + 1]));
    Box b;
    box_init(b);
    for (uint32_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
      for (int c = 0; c < nv; c++) {
        const size_t vi = f[(size_t)nv * i + c];
        box_add(b, v[3 * vi], v[3 * vi + 1], v[3 * vi + 2], e);
      }
    }
    b = block_reduce_box(b);
    if (threadIdx.x == 0 && lo < hi) {
      for (int k = 0; k < 3; k++) {
        atomicMin(&acc[6 * sg + k], f2o(b.lo[k]));
        atomicMax(&acc[6 * sg + 3 + k], f2o(b.hi[k]));
      }
    }
  }
}

template <int KIND>
__global__ void seg_finalize_kernel(const int *__restrict__ acc, int nseg,
                                    SceneInfo *__restrict__ scenes) {
  const int sg = blockIdx.x * blockDim.x + threadIdx.x;
  if (sg >= nseg) return;
  SceneInfo si;
  float lo[3], hi[3];
  for (int k = 0; k < 3; k++) {
    lo[k] = o2f(acc[6 * sg + k]);
    hi[k] = o2f(acc[6 * sg + 3 + k]);
    si.lo[k] = lo[k];
    si.hi[k] = hi[k];
    si.inv[k] = 1024.0f / (hi[k] - lo[k]);
  }
  if (KIND == SRT_TRIANGLES) {
    double es = (double)(hi[0] - lo[0]);
    if (es < (double)(hi[1] - lo[1])) es = (double)(hi[1] - lo[1]);
    if (es < (double)(hi[2] - lo[2])) es = (double)(hi[2] - lo[2]);
    si.eps_scale = es;
    si.keps = FLT_EPSILON * (float)es;
  } else {
    si.eps_scale = 16.0;
    si.keps = FLT_EPSILON * 16;
  }
  si.nbranches = 0;
  si.pad = 0;
  scenes[sg] = si;
}

template <int KIND>
__global__ void seg_morton_kernel(const float *__restrict__ v, const uint32_t *__restrict__ f,
                                  const uint32_t *__restrict__ foff, int nseg, uint32_t N,
                                  const SceneInfo *__restrict__ scenes,
                                  uint32_t *__restrict__ codes) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    const SceneInfo &sc = scenes[seg_of(foff, nseg, i)];
    float cx, cy, cz;
    if (KIND == SRT_TRIANGLES) {
      const float third = 1.0f / 3.0f;
      const size_t a = f[3 * (size_t)i], b = f[3 * (size_t)i + 1], c = f[3 * (size_t)i + 2];
      cx = third * ((v[3 * a] + v[3 * b]) + v[3 * c]);
      cy = third * ((v[3 * a + 1] + v[3 * b + 1]) + v[3 * c + 1]);
      cz = third * ((v[3 * a + 2] + v[3 * b + 2]) + v[3 * c + 2]);
    } else {
      const float fourth = 1.0f / 4.0f;
      const size_t a = f[4 * (size_t)i], b = f[4 * (size_t)i + 1], c = f[4 * (size_t)i + 2],
                   d = f[4 * (size_t)i + 3];
      cx = fourth * (((v[3 * a] + v[3 * b]) + v[3 * c]) + v[3 * d]);
      cy = fourth * (((v[3 * a + 1] + v[3 * b + 1]) + v[3 * c + 1]) + v[3 * d + 1]);
      cz = fourth * (((v[3 * a + 2] + v[3 * b + 2]) + v[3 * c + 2]) + v[3 * d + 2]);
    }
    const uint32_t qx = f2u32_x86((cx - sc.lo[0]) * sc.inv[0]);
    const uint32_t qy = f2u32_x86((cy - sc.lo[1]) * sc.inv[1]);
    const uint32_t qz = f2u32_x86((cz - sc.lo[2]) * sc.inv[2]);
    codes[i] = (spread10(qx) << 2) | (spread10(qy) << 1) | spread10(qz);
  }
}

__global__ void seg_karras_kernel(const uint32_t *__restrict__ codes,
                                  const uint32_t *__restrict__ foff,
                                  const uint32_t *__restrict__ ioff, int nseg, uint32_t M,
                                  uint32_t *__restrict__ kchild, uint8_t *__restrict__ kflags,
                                  uint2 *__restrict__ krange, uint32_t *__restrict__ kparent,
                                  uint32_t *__restrict__ lparent) {
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < M; g += gridDim.x * blockDim.x) {
    const int sg = seg_of(ioff, nseg, g);
    const uint32_t fb = __ldg(&foff[sg]), ib = __ldg(&ioff[sg]);
    const int n = (int)(__ldg(&foff[sg + 1]) - fb);
    const int i = (int)(g - ib);
    const uint32_t *c = codes + fb;
    int d = (kdelta(c, i, i + 1, n) - kdelta(c, i, i - 1, n)) >= 0 ? 1 : -1;
    int dmin = kdelta(c, i, i - d, n);
    int lmax = 2;
    while (kdelta(c, i, i + lmax * d, n) > dmin) lmax *= 2;
    int l = 0;
    for (int t = lmax / 2; t >= 1; t /= 2)
      if (kdelta(c, i, i + (l + t) * d, n) > dmin) l += t;
    const int j = i + l * d;
    const int dnode = kdelta(c, i, j, n);
    int s = 0;
    for (int k = 2;; k *= 2) {
      const int t = (l + k - 1) / k;
      if (t <= 0) break;
      if (kdelta(c, i, i + (s + t) * d, n) > dnode) s += t;
      if (t == 1) break;
    }
    const int gm = i + s * d + (d < 0 ? d : 0);
    const int lo = i < j ? i : j, hi = i < j ? j : i;
    const bool lleaf = (lo == gm), rleaf = (hi == gm + 1);
    kchild[g] = (uint32_t)gm;
    kflags[g] = (uint8_t)((lleaf ? 1 : 0) | (rleaf ? 2 : 0));
    krange[g] = make_uint2((uint32_t)lo, (uint32_t)hi);
    if (lleaf) lparent[fb + gm] = g; else kparent[ib + gm] = g;
    if (rleaf) lparent[fb + gm + 1] = g; else kparent[ib + gm + 1] = g;
    if (i == 0) kparent[g] = kNone;
  }
}

template <int KIND>
__global__ void seg_refit_kernel(const float *__restrict__ v, const uint32_t *__restrict__ f,
                                 const uint32_t *__restrict__ sidx,
                                 const uint32_t *__restrict__ foff,
                                 const uint32_t *__restrict__ ioff, int nseg, uint32_t N,
                                 const SceneInfo *__restrict__ scenes,
                                 const uint32_t *__restrict__ lparent,
                                 const uint32_t *__restrict__ kparent,
                                 const uint32_t *__restrict__ kchild,
                                 const uint8_t *__restrict__ kflags,
                                 uint32_t *__restrict__ counter, Box *__restrict__ ibox,
                                 float4 *__restrict__ prims, uint32_t *__restrict__ err) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= N) return;
  const int sg = seg_of(foff, nseg, j);
  const uint32_t fb = __ldg(&foff[sg]), ib = __ldg(&ioff[sg]);
  const float keps = scenes[sg].keps;
  const uint32_t p = sidx[j];
  Box mine;
  box_init(mine);
  if (KIND == SRT_TRIANGLES) {
    const size_t a = f[3 * (size_t)p], b = f[3 * (size_t)p + 1], c = f[3 * (size_t)p + 2];
    const float4 p0 = make_float4(v[3 * a], v[3 * a + 1], v[3 * a + 2], __uint_as_float(p - fb));
    const float4 p1 = make_float4(v[3 * b], v[3 * b + 1], v[3 * b + 2], 0.0f);
    const float4 p2 = make_float4(v[3 * c], v[3 * c + 1], v[3 * c + 2], 0.0f);
    prims[3 * (size_t)j + 0] = p0;
    prims[3 * (size_t)j + 1] = p1;
    prims[3 * (size_t)j + 2] = p2;
    box_add(mine, p0.x, p0.y, p0.z, keps);
    box_add(mine, p1.x, p1.y, p1.z, keps);
    box_add(mine, p2.x, p2.y, p2.z, keps);
  }
  uint32_t cur = j;
  bool cur_leaf = true;
  uint32_t node = lparent[j];
  for (uint32_t guard = 0; guard < 2 * N + 64; guard++) {
    __threadfence();
    if (atomicAdd(&counter[node], 1u) == 0) return;
    __threadfence();
    const uint32_t gl = __ldcg(&kchild[node]);
    const uint8_t fl = __ldcg(&kflags[node]);
    const bool lleaf = fl & 1, rleaf = fl & 2;
    const uint32_t left = lleaf ? fb + gl : ib + gl;
    const uint32_t right = rleaf ? fb + gl + 1 : ib + gl + 1;
    const bool i_am_left = (cur == left) && (cur_leaf == lleaf);
    const uint32_t sib = i_am_left ? right : left;
    const bool sib_leaf = i_am_left ? rleaf : lleaf;
    Box sb;
    if (sib_leaf) {
      sb = cache_box<KIND>(prims, sib, keps);
    } else {
      const float *src = reinterpret_cast<const float *>(&ibox[sib]);
      sb.lo[0] = __ldcg(src + 0); sb.lo[1] = __ldcg(src + 1); sb.lo[2] = __ldcg(src + 2);
      sb.hi[0] = __ldcg(src + 3); sb.hi[1] = __ldcg(src + 4); sb.hi[2] = __ldcg(src + 5);
    }
    mine = i_am_left ? box_merge(mine, sb) : box_merge(sb, mine);
    ibox[node] = mine;
    if (node == ib) return;  // scene root
    cur = node;
    cur_leaf = false;
    node = __ldcg(&kparent[node]);
    if (node == kNone) return;
  }
  atomicOr(err, kErrTree);
}

__global__ void seg_level_kernel(const uint2 *__restrict__ krange,
                                 const uint32_t *__restrict__ kparent,
                                 const uint32_t *__restrict__ ioff, int nseg, uint32_t M,
                                 int max_leaf, uint32_t *__restrict__ flag) {
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < M; g += gridDim.x * blockDim.x) {
    const uint32_t root = __ldg(&ioff[seg_of(ioff, nseg, g)]);
    const uint2 r = krange[g];
    uint32_t fl = 0;
    if (g == root) {
      fl = 1;
    } else if (r.y - r.x > (uint32_t)max_leaf) {
      int lvl = 0;
      uint32_t x = g;
      while (x != root && lvl <= kMaxLevel) {
        x = kparent[x];
        lvl++;
      }
      fl = (lvl <= kMaxLevel) ? 1u : 0u;
    }
    flag[g] = fl;
  }
}

template <int KIND>
__global__ void seg_emit_node2_kernel(const uint32_t *__restrict__ codes,
                                      const uint32_t *__restrict__ kchild,
                                      const uint8_t *__restrict__ kflags,
                                      const uint2 *__restrict__ krange,
                                      const uint32_t *__restrict__ flag,
                                      const uint32_t *__restrict__ slot,
                                      const Box *__restrict__ ibox,
                                      const float4 *__restrict__ prims,
                                      const SceneInfo *__restrict__ scenes,
                                      const uint32_t *__restrict__ foff,
                                      const uint32_t *__restrict__ ioff, int nseg, uint32_t M,
                                      Node2 *__restrict__ nodes, uint32_t *__restrict__ err) {
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < M; g += gridDim.x * blockDim.x) {
    if (!flag[g]) continue;
    const int sg = seg_of(ioff, nseg, g);
    const uint32_t fb = __ldg(&foff[sg]), ib = __ldg(&ioff[sg]);
    const float keps = scenes[sg].keps;
    const uint32_t gl = kchild[g];
    const uint8_t fl = kflags[g];
    Box bx[2];
    uint32_t ref[2], cnt[2];
    for (int side = 0; side < 2; side++) {
      const uint32_t cl = gl + side;
      if (fl & (1 << side)) {
        bx[side] = cache_box<KIND>(prims, fb + cl, keps);
        ref[side] = fb + cl;
        cnt[side] = 1;
      } else {
        const uint32_t cg = ib + cl;
        bx[side] = ibox[cg];
        if (flag[cg]) {
          ref[side] = slot[cg];
          cnt[side] = 0;
        } else {
          const uint2 r = krange[cg];
          ref[side] = fb + r.x;
          cnt[side] = r.y - r.x + 1;
        }
      }
      if (cnt[side] > kCountMask) atomicOr(err, kErrTree);
    }
    const uint32_t axis = (uint32_t)split_axis(codes[fb + (g - ib)]);
    Node2 nd;
    nd.a = make_float4(bx[0].lo[0], bx[0].lo[1], bx[0].lo[2], bx[0].hi[0]);
    nd.b = make_float4(bx[0].hi[1], bx[0].hi[2], bx[1].lo[0], bx[1].lo[1]);
    nd.c = make_float4(bx[1].lo[2], bx[1].hi[0], bx[1].hi[1], bx[1].hi[2]);
    nd.d = make_uint4(ref[0], ref[1], (cnt[0] & kCountMask) | (axis << 30), cnt[1] & kCountMask);
    nodes[slot[g]] = nd;
  }
}

__global__ void seg_roots_kernel(const uint32_t *__restrict__ slot,
                                 const uint32_t *__restrict__ flag,
                                 const uint32_t *__restrict__ ioff, int nseg, uint32_t M,
                                 uint32_t *__restrict__ roots) {
  const int sg = blockIdx.x * blockDim.x + threadIdx.x;
  if (sg < nseg) roots[sg] = slot[ioff[sg]];
  if (sg == 0) roots[nseg] = slot[M - 1] + flag[M - 1];  // total branch nodes
}

}  // namespace

// Batched triangle build: see the block comment above seg_bbox_kernel.
// h_foff: host copy of the nseg+1 primitive offsets (each scene >= 2 faces).
srt_status build_batch(srt_ctx *ctx, BatchTree &bt, const float *v, const uint32_t *f,
                       const uint32_t *h_foff, int nseg) {
  constexpr int KIND = SRT_TRIANGLES;
  cudaStream_t st = ctx->stream;
  const uint32_t N = h_foff[nseg];
  const uint32_t M = N - (uint32_t)nseg;
  cudaError_t e;
#define ENSURE(buf, bytes)                                   \
  do {                                                       \
    if ((e = (buf).ensure(bytes)) != cudaSuccess)            \
      return cuda_status(e, "batch allocation " #buf);       \
  } while (0)
  ENSURE(bt.codes, (size_t)N * 4);
  ENSURE(bt.indices, (size_t)N * 4);
  ENSURE(bt.prims, (size_t)N * 3 * sizeof(float4));
  ENSURE(bt.nodes, (size_t)M * sizeof(Node2));
  ENSURE(bt.scenes, (size_t)nseg * sizeof(SceneInfo));
  ENSURE(bt.roots, (size_t)(nseg + 1) * 4);
  ENSURE(bt.acc, (size_t)nseg * 6 * 4);
  ENSURE(ctx->s_kchild, (size_t)M * 4);
  ENSURE(ctx->s_kflags, M);
  ENSURE(ctx->s_krange, (size_t)M * sizeof(uint2));
  ENSURE(ctx->s_kparent, (size_t)M * 4);
  ENSURE(ctx->s_lparent, (size_t)N * 4);
  ENSURE(ctx->s_counter, (size_t)M * 4);
  ENSURE(ctx->s_ibox, (size_t)M * sizeof(Box));
  ENSURE(ctx->s_flag, (size_t)M * 4);
  ENSURE(ctx->s_slot, (size_t)M * 4);
#undef ENSURE
  srt_status s = sort_scratch(ctx, N);
  if (s != SRT_OK) return s;
  {
    size_t need = 64;
    for (size_t t = ((size_t)kRsMaxBins * ((N + kRsTile - 1) / kRsTile) + kScanTile - 1) / kScanTile;
         t > 1; t = (t + kScanTile - 1) / kScanTile)
      need += t + 1;
    for (size_t t = (M + kScanTile - 1) / kScanTile; t > 1; t = (t + kScanTile - 1) / kScanTile)
      need += t + 1;
    if ((e = ctx->s_scan.ensure(need * 4)) != cudaSuccess) return cuda_status(e, "scan scratch");
  }
  const uint32_t *foff = bt.foff.as<uint32_t>();
  const uint32_t *ioff = bt.ioff.as<uint32_t>();
  SceneInfo *scenes = bt.scenes.as<SceneInfo>();
  uint32_t *codes = bt.codes.as<uint32_t>();
  uint32_t *idx = bt.indices.as<uint32_t>();
  int *acc = bt.acc.as<int>();
  const int gsm = ctx->num_sms * 16;
  seg_bbox_init_kernel<<<1, 256, 0, st>>>(acc, nseg);
  seg_bbox_kernel<KIND><<<(N + kSegTile - 1) / kSegTile, 256, 0, st>>>(v, f, foff, nseg, N, acc);
  seg_finalize_kernel<KIND><<<(nseg + 63) / 64, 64, 0, st>>>(acc, nseg, scenes);
  seg_morton_kernel<KIND><<<grid_for(N, kBlock, gsm), kBlock, 0, st>>>(v, f, foff, nseg, N,
                                                                       scenes, codes);
  ctx->launches += 4;
  s = cuda_status(cudaGetLastError(), "batch bbox/morton");
  if (s != SRT_OK) return s;
  s = sort_pairs_seg(ctx, codes, idx, N, true, foff, nseg, 30);
  if (s != SRT_OK) return s;
  uint32_t *kchild = ctx->s_kchild.as<uint32_t>();
  uint8_t *kflags = ctx->s_kflags.as<uint8_t>();
  uint2 *krange = ctx->s_krange.as<uint2>();
  uint32_t *kparent = ctx->s_kparent.as<uint32_t>();
  uint32_t *lparent = ctx->s_lparent.as<uint32_t>();
  uint32_t *counter = ctx->s_counter.as<uint32_t>();
  Box *ibox = ctx->s_ibox.as<Box>();
  uint32_t *flag = ctx->s_flag.as<uint32_t>();
  uint32_t *slot = ctx->s_slot.as<uint32_t>();
  seg_karras_kernel<<<grid_for(M, kBlock, gsm), kBlock, 0, st>>>(codes, foff, ioff, nseg, M,
                                                               kchild, kflags, krange, kparent,
                                                               lparent);
  if ((e = cudaMemsetAsync(counter, 0, (size_t)M * 4, st)) != cudaSuccess)
    return cuda_status(e, "refit counters");
  seg_refit_kernel<KIND><<<(N + kBlock - 1) / kBlock, kBlock, 0, st>>>(
      v, f, idx, foff, ioff, nseg, N, scenes, lparent, kparent, kchild, kflags, counter, ibox,
      bt.prims.as<float4>(), ctx->d_err);
  seg_level_kernel<<<grid_for(M, kBlock, gsm), kBlock, 0, st>>>(krange, kparent, ioff, nseg, M,
                                                              PrimTraits<KIND>::kMaxLeaf, flag);
  ctx->launches += 3;
  s = cuda_status(cudaGetLastError(), "batch karras/refit/level");
  if (s != SRT_OK) return s;
  s = exclusive_scan(ctx, flag, slot, M);
  if (s != SRT_OK) return s;
  seg_emit_node2_kernel<KIND><<<grid_for(M, kBlock, gsm), kBlock, 0, st>>>(
      codes, kchild, kflags, krange, flag, slot, ibox, bt.prims.as<float4>(), scenes, foff, ioff,
      nseg, M, bt.nodes.as<Node2>(), ctx->d_err);
  seg_roots_kernel<<<(nseg + 63) / 64, 64, 0, st>>>(slot, flag, ioff, nseg, M,
                                                   bt.roots.as<uint32_t>());
  ctx->launches += 2;
  return cuda_status(cudaGetLastError(), "batch emit");
}

namespace {
// Sorted Morton codes of a loaded tree: the code of each sorted primitive.
__global__ void gather_codes_kernel(const uint32_t *__restrict__ codes,
                                    const uint32_t *__restrict__ sidx, size_t n,
                                    uint32_t *__restrict__ out) {
  for (size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x; j < n;
       j += (size_t)gridDim.x * blockDim.x)
    out[j] = codes[sidx[j]];
}

__global__ void set_branches_kernel(SceneInfo *__restrict__ scene, uint32_t nb) {
  scene->nbranches = nb;
}

// An accel from a tree read from a file: the scene box and codes as the build
// computes them, the given sorted order and nodes, the primitive cache.
template <int KIND>
srt_status load_kind(srt_accel *a, const float *v, const uint32_t *f, const float *radius,
                     float constr, size_t n, const void *h_nodes, size_t nnodes,
                     uint32_t nbranches, const uint32_t *h_idx) {
  srt_ctx *ctx = a->ctx;
  cudaStream_t st = ctx->stream;
  cudaError_t e;
  const size_t node_bytes = (KIND == SRT_TETRAHEDRA) ? sizeof(NodeT) : sizeof(Node2);
  if ((e = a->codes.ensure(n * 4)) != cudaSuccess ||
      (e = a->indices.ensure(n * 4)) != cudaSuccess ||
      (e = a->prims.ensure(n * sizeof(float4) * PrimTraits<KIND>::kCacheF4)) != cudaSuccess ||
      (e = a->scene.ensure(sizeof(SceneInfo))) != cudaSuccess ||
      (e = a->nodes.ensure(nnodes * node_bytes)) != cudaSuccess ||
      (e = ctx->s_keys2.ensure(n * 4)) != cudaSuccess)
    return cuda_status(e, "load allocation");
  SceneInfo *scene = a->scene.as<SceneInfo>();
  uint32_t *tmp = ctx->s_keys2.as<uint32_t>();
  srt_status s = launch_bbox_morton<KIND>(ctx, v, f, radius, constr, n, scene, tmp, nullptr);
  if (s != SRT_OK) return s;
  uint32_t *idx = a->indices.as<uint32_t>();
  e = cudaMemcpyAsync(idx, h_idx, n * 4, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(a->nodes.p, h_nodes, nnodes * node_bytes, cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return cuda_status(e, "load upload");
  const int g = grid_for(n, kBlock, ctx->num_sms * 16);
  gather_codes_kernel<<<g, kBlock, 0, st>>>(tmp, idx, n, a->codes.as<uint32_t>());
  cache_kernel<KIND><<<g, kBlock, 0, st>>>(v, f, radius, constr, idx, (int)n,
                                           a->prims.as<float4>());
  set_branches_kernel<<<1, 1, 0, st>>>(scene, nbranches);
  ctx->launches += 3;
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_status(e, "load");
  // the host arrays are the caller's until the copies are done
  return cuda_status(cudaStreamSynchronize(st), "load");
}
}  // namespace

srt_status load_accel(srt_accel *a, const float *v, const uint32_t *f, const float *radius,
                      float constr, size_t n, const void *h_nodes, size_t nnodes,
                      uint32_t nbranches, const uint32_t *h_idx) {
  a->host_scene_valid = false;
  switch (a->kind) {
    case SRT_TRIANGLES:
      return load_kind<SRT_TRIANGLES>(a, v, f, radius, constr, n, h_nodes, nnodes, nbranches,
                                      h_idx);
    case SRT_TETRAHEDRA:
      return load_kind<SRT_TETRAHEDRA>(a, v, f, radius, constr, n, h_nodes, nnodes, nbranches,
                                       h_idx);
    case SRT_SPHERES:
      return load_kind<SRT_SPHERES>(a, v, f, radius, constr, n, h_nodes, nnodes, nbranches,
                                    h_idx);
  }
  return SRT_ERR_INVALID;
}

srt_status build_accel(srt_accel *a, const float *v, const uint32_t *f,
                       const float *radius, float constr, size_t n) {
  a->host_scene_valid = false;
  switch (a->kind) {
    case SRT_TRIANGLES:
      return build_kind<SRT_TRIANGLES>(a, v, f, radius, constr, n);
    case SRT_TETRAHEDRA:
      return build_kind<SRT_TETRAHEDRA>(a, v, f, radius, constr, n);
    case SRT_SPHERES:
      return build_kind<SRT_SPHERES>(a, v, f, radius, constr, n);
  }
  return SRT_ERR_INVALID;
}

srt_status stage_morton(srt_ctx *ctx, srt_kind kind, const float *v, const uint32_t *f,
                        const float *radius, float constr, size_t n, uint32_t *codes,
                        SceneInfo *scene) {
  switch (kind) {
    case SRT_TRIANGLES:
      return launch_bbox_morton<SRT_TRIANGLES>(ctx, v, f, radius, constr, n, scene, codes,
                                               nullptr);
    case SRT_TETRAHEDRA:
      return launch_bbox_morton<SRT_TETRAHEDRA>(ctx, v, f, radius, constr, n, scene, codes,
                                                nullptr);
    case SRT_SPHERES:
      return launch_bbox_morton<SRT_SPHERES>(ctx, v, f, radius, constr, n, scene, codes,
                                             nullptr);
  }
  return SRT_ERR_INVALID;
}

srt_status stage_topology(srt_ctx *ctx, const uint32_t *codes, size_t n, int max_leaf,
                          SceneInfo *info, Topology &t) {
  if (n < 2) return SRT_ERR_INVALID;
  cudaStream_t st = ctx->stream;
  cudaError_t e;
  const size_t m = n - 1;
  if ((e = ctx->s_kchild.ensure(m * 4)) != cudaSuccess ||
      (e = ctx->s_kflags.ensure(m)) != cudaSuccess ||
      (e = ctx->s_krange.ensure(m * sizeof(uint2))) != cudaSuccess ||
      (e = ctx->s_kparent.ensure(m * 4)) != cudaSuccess ||
      (e = ctx->s_counter.ensure(m * 4)) != cudaSuccess ||
      (e = ctx->s_kidx.ensure(m * 4)) != cudaSuccess ||
      (e = ctx->s_kprefix.ensure(m)) != cudaSuccess ||
      (e = ctx->s_flag.ensure(m * 4)) != cudaSuccess ||
      (e = ctx->s_slot.ensure(m * 4)) != cudaSuccess)
    return cuda_status(e, "topology scratch");
  const uint32_t ltiles = (uint32_t)((m + kLsTile - 1) / kLsTile);
  const size_t lbytes = 256 + (size_t)ltiles * 8;
  if (lbytes > ctx->s_lscan.cap || !ctx->s_lscan.p) {
    if ((e = ctx->s_lscan.ensure(lbytes)) != cudaSuccess ||
        (e = cudaMemsetAsync(ctx->s_lscan.p, 0, ctx->s_lscan.cap, st)) != cudaSuccess)
      return cuda_status(e, "level scan");
  }
  unsigned long long *lticket = ctx->s_lscan.as<unsigned long long>();
  unsigned long long *lstatus =
      reinterpret_cast<unsigned long long *>(ctx->s_lscan.as<char>() + 256);
  t.kchild = ctx->s_kchild.as<uint32_t>();
  t.kflags = ctx->s_kflags.as<uint8_t>();
  t.krange = ctx->s_krange.as<uint2>();
  t.kparent = ctx->s_kparent.as<uint32_t>();
  t.counter = ctx->s_counter.as<uint32_t>();
  t.kidx = ctx->s_kidx.as<uint32_t>();
  t.flag = ctx->s_flag.as<uint32_t>();
  t.slot = ctx->s_slot.as<uint32_t>();
  uint8_t *kprefix = ctx->s_kprefix.as<uint8_t>();
  const int gk = grid_for(m, kBlock, ctx->num_sms * 16);
  karras_kernel<<<gk, kBlock, 0, st>>>(codes, (int)n, ctx->s_kchild.as<uint32_t>(),
                                       ctx->s_kflags.as<uint8_t>(), ctx->s_krange.as<uint2>(),
                                       ctx->s_kparent.as<uint32_t>(), nullptr, lticket, kprefix);
  const uint32_t lepoch = ++ctx->os_epoch == 0 ? ++ctx->os_epoch : ctx->os_epoch;
  level_scan_kernel<<<ltiles, kLsThreads, 0, st>>>(
      ctx->s_krange.as<uint2>(), ctx->s_kparent.as<uint32_t>(), kprefix, (int)n, max_leaf,
      ctx->s_flag.as<uint32_t>(), ctx->s_slot.as<uint32_t>(), ctx->s_kidx.as<uint32_t>(),
      ctx->s_counter.as<uint32_t>(), lstatus, lticket, lepoch, info, ctx->d_err);
  ctx->launches += 2;
  return cuda_status(cudaGetLastError(), "topology");
}

srt_status stage_karras(srt_ctx *ctx, const uint32_t *codes, size_t n, uint32_t *child,
                        uint8_t *flags) {
  int gk = grid_for(n - 1, kBlock, ctx->num_sms * 16);
  karras_kernel<<<gk, kBlock, 0, ctx->stream>>>(codes, (int)n, child, flags, nullptr,
                                                nullptr, nullptr);
  ctx->launches++;
  return cuda_status(cudaGetLastError(), "karras");
}

}  // namespace srt
