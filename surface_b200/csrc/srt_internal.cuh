// srt_internal.cuh -- shared device/host internals of libsurface_rt.
//
// Floating point: the whole library is compiled with --fmad=false and without
// fast-math, so every float/double expression rounds exactly like the
// reference's x86-64 g++ build (SSE2, no contraction).  Division and sqrt are
// IEEE round-to-nearest.
#pragma once

#include <cuda_runtime.h>
#include <float.h>
#include <limits.h>
#include <stdint.h>

#include <atomic>
#include <string>
#include <vector>

#include "surface_rt.h"

namespace srt {

// ---------------------------------------------------------------- limits
constexpr int kMaxLevel = 23;        // reference depth > 22 forces a leaf;
                                     // root = level 0, its children level 1
constexpr int kStack = 32;           // traversal stack (tree depth <= 24)
constexpr uint32_t kCountMask = 0x3fffffffu;
constexpr uint32_t kLeafBit = 0x80000000u;
constexpr uint32_t kNone = 0xffffffffu;

// device error word bits (set by kernels, reported by srt_ctx_synchronize)
constexpr uint32_t kErrStack = 1u;
constexpr uint32_t kErrIter = 2u;
constexpr uint32_t kErrTree = 4u;
constexpr uint32_t kErrSortWait = 8u;  // a sort pass gave up waiting on a tile

// ---------------------------------------------------------------- layouts
// Two-child node (triangles, spheres): 64 bytes, the reference's
// TriangleNode/ParticleNode information with leaves folded into the parent:
//   a = (c0.lo.x, c0.lo.y, c0.lo.z, c0.hi.x)
//   b = (c0.hi.y, c0.hi.z, c1.lo.x, c1.lo.y)
//   c = (c1.lo.z, c1.hi.x, c1.hi.y, c1.hi.z)
//   d = (ref0, ref1, meta0, meta1)
// meta_k & kCountMask = leaf primitive count of child k (0: child k is a
// branch and ref_k its node index; else ref_k = first sorted primitive);
// meta0 >> 30 = this node's split axis.
struct __align__(16) Node2 {
  float4 a, b, c;
  uint4 d;
};

// Own-box node (tetrahedra): 32 bytes, the reference's TetraNode.
//   a = (lo.x, lo.y, lo.z, meta)  meta: leaf -> kLeafBit | count, branch -> axis
//   b = (hi.x, hi.y, hi.z, ref)   ref:  leaf -> first sorted primitive,
//                                       branch -> left child (right = ref + 1)
struct __align__(16) NodeT {
  float4 a, b;
};

// Scene box and derived build constants (one per build, device resident).
struct SceneInfo {
  float lo[3], hi[3];
  float inv[3];      // 1024 / (hi - lo)
  float keps;        // leaf box padding
  double eps_scale;  // triangles: max scene extent
  uint32_t nbranches;
  uint32_t pad;
};

struct Box {
  float lo[3], hi[3];
};

// ---------------------------------------------------------------- device math
// std::min / std::max with the reference's tie behaviour (first operand kept).
__device__ __forceinline__ float fmin_ref(float a, float b) { return (b < a) ? b : a; }
__device__ __forceinline__ float fmax_ref(float a, float b) { return (a < b) ? b : a; }

// (uint32_t)x as g++ emits it on x86-64: a 64-bit truncating convert whose low
// 32 bits are kept; NaN and |x| >= 2^63 give 0.
// (int)x as x86-64 converts it: truncation, INT_MIN for NaN and for values
// outside the int range.
__device__ __forceinline__ int f2i_x86(float x) {
  return (x >= -2147483648.0f && x < 2147483648.0f) ? (int)x : INT_MIN;
}
__device__ __forceinline__ int d2i_x86(double x) {
  return (x > -2147483649.0 && x < 2147483648.0) ? (int)x : INT_MIN;
}

// fasterfloorf (render/render_texture.cc:108-121), the repeat wrap's floor.
__device__ __forceinline__ int floor_ref(float x) {
  if (x >= 0) return f2i_x86(x);
  int y = f2i_x86(x);
  if (fabsf(x - (float)y) <= FLT_EPSILON) {
  } else {
    y = y - 1;
  }
  return y;
}

__device__ __forceinline__ uint32_t f2u32_x86(float x) {
  if (!(fabsf(x) < 9.2233720368547758e18f)) return 0u;
  return (uint32_t)(long long)x;
}

__device__ __forceinline__ uint32_t spread10(uint32_t v) {
  v &= 0x3ffu;
  v = (v | (v << 16)) & 0x030000ffu;
  v = (v | (v << 8)) & 0x0300f00fu;
  v = (v | (v << 4)) & 0x030c30c3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}

// Segment (scene) of global index x: the largest s with off[s] <= x.
__device__ __forceinline__ int seg_of(const uint32_t *__restrict__ off, int nseg, uint32_t x) {
  int lo = 0, hi = nseg - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(&off[mid]) <= x) lo = mid; else hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ int split_axis(uint32_t code) {
  return (__clz(code) - 2) % 3;  // __clz(0) = 32
}

// Spherical (u, v) of a sphere hit's unit normal n, the values ParticleAccel's
// BuildIntersection stores in Intersection::u / v
// (render/render_accel_particle.cc:3013-3014): u = (atan2(n.x, n.z) + pi) *
// 0.5 * (1 / pi), v = acos(n.y) / pi, all in double and rounded to float at
// the end.  The reference's build evaluates the angles with the C library's
// double atan2 / acos; CUDA's double atan2 / acos may differ from those in the
// last bit or two of the double, which changes the float result only when it
// lies within a few double ulps of a float rounding boundary.
constexpr double kPi = 3.14159265358979323846;
__device__ __forceinline__ void sphere_uv(const float n[3], float &u, float &v) {
  u = (float)((atan2((double)n[0], (double)n[2]) + kPi) * 0.5 * (1.0 / kPi));
  v = (float)(acos((double)n[1]) / kPi);
}

// ---------------------------------------------------------------- host side
// Bumped whenever any DevBuf frees memory; a captured CUDA graph that holds
// scratch pointers is valid only while the epoch it was captured at holds.
extern std::atomic<uint64_t> g_buffer_epoch;

struct DevBuf {
  void *p = nullptr;
  size_t cap = 0;
  DevBuf() = default;
  DevBuf(const DevBuf &) = delete;
  DevBuf &operator=(const DevBuf &) = delete;
  ~DevBuf() { release(); }
  cudaError_t ensure(size_t bytes);
  void release();
  template <typename T>
  T *as() const {
    return static_cast<T *>(p);
  }
};

}  // namespace srt

struct srt_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t own_stream = nullptr;
  uint32_t *d_err = nullptr;  // device error word
  uint32_t *h_err = nullptr;  // pinned mirror
  int num_sms = 148;
  uint64_t launches = 0;  // kernels launched by this context
  // scratch shared by the builds of this context (stream ordered)
  srt::DevBuf s_keys2, s_vals2, s_hist, s_scan, s_kchild, s_kflags, s_krange,
      s_kparent, s_lparent, s_counter, s_ibox, s_flag, s_slot, s_partial,
      s_stage_in, s_stage_out, s_stage_aux, s_stage_sub, s_stage_scal, s_stage_norm,
      s_defer, s_spawn, s_rkey, s_rorder, s_isect_sub, s_stage_isect, s_keys3, s_vals3,
      s_status, s_lscan, s_rays_in, s_kidx, s_kprefix;
  uint32_t os_epoch = 0;  // look-back epoch of the last sort pass (srt_sort.cu)
  // recorded after a build's host inputs were copied; the next staged ray
  // array waits for it (inputs_pending)
  cudaEvent_t ev_inputs = nullptr;
  bool inputs_pending = false;
  // side stream that copies a page-locked host ray array to the device while
  // earlier work (a build) still runs on the context stream; ev_copy: copy
  // done, ev_free: the last trace that read s_rays_in is done
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t ev_copy = nullptr, ev_free = nullptr;
  bool ev_free_recorded = false;
};

struct srt_accel {
  srt_ctx *ctx = nullptr;
  srt_kind kind = SRT_TRIANGLES;
  size_t n = 0;
  size_t nnodes_cap = 0;
  bool built = false;
  srt::DevBuf nodes, indices, codes, prims, scene;
  srt::DevBuf in_verts, in_faces, in_radius;  // device copies of host inputs
  // primitive arrays the tree was built from (owned copies of host inputs,
  // or the caller's device arrays, borrowed like the reference's mesh_)
  const float *src_verts = nullptr;
  const uint32_t *src_faces = nullptr;
  // tetrahedra with double-precision positions: the primitive cache holds
  // doubles (six double2 per tetrahedron); src_verts the positions rounded
  // to float; in_dverts a device copy of host positions
  bool dbl = false;
  srt::DevBuf in_dverts;
  // host-side cache of the device SceneInfo (valid after a sync)
  srt::SceneInfo host_scene;
  bool host_scene_valid = false;
};

namespace srt {
// Synchronises the context stream and reports kernel limit flags
// (SRT_ERR_LIMIT) raised since the last report (srt_capi.cu).
srt_status check_device_errors(srt_ctx *ctx);

// Many triangle scenes built as one forest (srt_batch).
struct BatchTree {
  DevBuf nodes, indices, codes, prims, scenes, roots, acc, foff, ioff, roff;
  int nseg = 0;
  size_t nprims = 0, nrays = 0;
};

void set_error(const std::string &msg);
srt_status cuda_status(cudaError_t e, const char *what);
// pointer classification
bool is_device_ptr(const void *p);

// build pipeline pieces (srt_build.cu)
// Build32 of tetrahedra with double-precision positions (srt_build.cu);
// vf receives the positions rounded to float.
srt_status build_tet_double(srt_accel *a, const double *dv, size_t nverts, const uint32_t *f,
                            size_t n, float *vf);
srt_status build_accel(srt_accel *a, const float *d_verts, const uint32_t *d_faces,
                       const float *d_radius, float const_radius, size_t n);
// An accel from a tree read from a file (srt_cache.cu): host nodes in the
// device layout (nnodes records, nbranches branches) and host sorted order.
srt_status load_accel(srt_accel *a, const float *d_verts, const uint32_t *d_faces,
                      const float *d_radius, float const_radius, size_t n,
                      const void *h_nodes, size_t nnodes, uint32_t nbranches,
                      const uint32_t *h_idx);
srt_status stage_morton(srt_ctx *ctx, srt_kind kind, const float *d_verts,
                        const uint32_t *d_faces, const float *d_radius,
                        float const_radius, size_t n, uint32_t *d_codes,
                        SceneInfo *d_scene);
// Top level of a scene (RenderGraph): a node of the reference's BVHTree
// (render/render_bvh_tree.h:28-43) over the elements' world boxes.
struct TopNode {
  double bmin[3], bmax[3];
  int32_t child[2];  // 0: none
  int32_t axis, leaf;
  uint32_t id;       // element of a leaf
  uint32_t pad;
};
// Scene element kinds beyond srt_kind: line and solid accels.
constexpr int32_t kSceneLines = 3, kSceneSolids = 4;
// SceneElem.aux bit of a solid element with double-precision positions,
// and of a tetrahedron element with them.
constexpr int32_t kSolidAuxDouble = 256;
constexpr int32_t kTetAuxDouble = 512;
// One element of a scene: a built accel and its transforms, 4x4 doubles in
// the reference's Matrixd layout (m[row][col], p' = p m + m[3]).  Line and
// solid elements keep their device nodes in nodes and records in prims;
// aux: the line accel's cap flag, the solid accel's vertices per solid (|
// kSolidAuxDouble for double-precision positions).
struct SceneElem {
  int32_t kind;
  uint32_t nprims;
  int32_t aux;
  const void *nodes;
  const float4 *prims;
  const uint32_t *sidx;
  const SceneInfo *scene;
  double T[16], invT[16], invT33[16];
};
// Device arrays of one scene trace (srt_trace.cu): per ray its candidates
// (kRoundCand slots of entry distance and element) and running nearest
// world distance; the dense sort keys (element rank in kind order, nelem
// for none) and values of the two phases -- phase 0: one per ray (its first
// candidate), phase 1: kRoundCand - 1 per ray (its later candidates) --;
// the per-(ray, slot) results of phase 1 and the list of rays with more
// candidates than slots.  counters: [2] overflow rays, [4 + 3p + k] warp
// fetch and [10 + 3p + k] deferred items of phase p, kind k; bounds [2][4]:
// each kind's range of a phase's sorted keys (kinds are rank ranges
// rank_start[k] .. rank_start[k + 1]).
constexpr int kRoundCand = 8;
constexpr int kSceneCounters = 16;
// A ray (or scene item) whose front-to-back pass was not conclusive.
struct Deferred {
  uint32_t ray;
  uint32_t full;  // 1: the reference's walk from the pass's bound; 0: replay the tie at m
  double m;
};
struct SceneWork {
  const SceneElem *elems;
  const uint32_t *elem_rank;  // element id -> rank in kind order
  uint32_t nelem;
  uint32_t rank_start[4];     // first rank of triangles, tetrahedra, spheres, loop-only kinds
  const srt_ray *rays;
  const uint32_t *prev_element;
  const float *prev_normals;
  srt_hit *hits;
  uint32_t *element;
  double *cand_t;
  uint32_t *cand_e;
  uint8_t *ncand;
  float *tnear;
  uint32_t *keys0, *vals0, *keys1, *vals1;
  float4 *res;
  Deferred *dlist;  // per phase, kind k's deferred items from bounds[k] on
  uint32_t *counters, *bounds;
  uint32_t *ovf;
  size_t n;
  uint32_t max_iter;
  unsigned long long *stats;
  uint32_t *err;
};
// Side streams of a scene's trace: one per element kind and one for the
// rays with more candidates than slots, forked from and joined to the
// context stream with events (also inside a graph capture).
struct SceneStreams {
  cudaStream_t side[4] = {};
  cudaEvent_t fork[3] = {};  // top level done, phase 0 items ready, phase 1 items ready
  cudaEvent_t join[4] = {};  // each side stream's latest work
};
// BVHTree::BuildTree on the host over n boxes (srt_scene.cu): node 0 is
// the root, TopNode.id of a leaf is its box's index.
void build_top_tree(const double *bmin, const double *bmax, size_t n,
                    std::vector<TopNode> &out);
// kinds: bit k set when the scene holds elements of kind k; deep_lines: a
// line or solid element's tree is deeper than 62 levels.
srt_status launch_scene_trace(srt_ctx *ctx, const TopNode *top, SceneWork W, uint32_t kinds,
                              bool deep_lines, const SceneStreams &ss);
// Coherent traversal order of n rays (srt_raysort.cu): *order is a device
// array in context scratch, valid until the context's next sort.
srt_status ray_order(srt_ctx *ctx, const srt_ray *rays, size_t n, const uint32_t **order);
// The same for the rays of a batch (ray offsets roff over nseg scenes, on
// the device), kept grouped by scene, ordered within a scene by the top
// mbits of their Morton code: keys (n + 16 words of scratch) and order (n).
srt_status batch_ray_order(srt_ctx *ctx, const srt_ray *rays, size_t n, const uint32_t *roff,
                           int nseg, int mbits, uint32_t *keys, uint32_t *order);
// Device bytes held by a line or solid accel (srt_line.cu, srt_solid.cu).
uint64_t line_accel_bytes(const srt_line_accel *a);
uint64_t solid_accel_bytes(const srt_solid_accel *a);
// A built line or solid accel as a scene element: its context, device
// nodes and records, element count, aux (cap flag / vertices per solid)
// and tree depth (lines) or whether the tree is deeper than 62 levels
// (solids).  False when the accel is not built.
bool line_scene_view(const srt_line_accel *a, srt_ctx **ctx, SceneElem &e, int &depth);
bool solid_scene_view(const srt_solid_accel *a, srt_ctx **ctx, SceneElem &e, bool &deep);
// Exclusive prefix sum of n uint32 on the context's stream (out may alias in).
srt_status scan_exclusive(srt_ctx *ctx, const uint32_t *in, uint32_t *out, size_t n);
// Stable sort of (key, value) pairs by key; key_bits: how many low bits of
// the keys can be non-zero (30 for Morton codes).
srt_status sort_pairs(srt_ctx *ctx, uint32_t *d_keys, uint32_t *d_vals,
                      size_t n, bool identity_vals, int key_bits = 32);
// The same order for 30-bit keys (Morton codes) with one kernel per 10-bit
// pass (srt_sort.cu); n < 2^30.
srt_status sort_codes30(srt_ctx *ctx, uint32_t *d_keys, uint32_t *d_vals, size_t n,
                        bool identity_vals, bool hist_ready = false);
// Its scratch for n keys: the digit histograms (3 x 1024 words, to be filled
// before a hist_ready sort) and the three passes' tile counters (zeroed).
srt_status sort_codes30_scratch(srt_ctx *ctx, size_t n, uint32_t **hist,
                                unsigned long long **tickets);
// The Karras tree of n >= 2 sorted codes and its emitted branches
// (srt_build.cu): an internal node is a branch iff it is the root, or its
// range holds more than max_leaf + 1 keys and it lies at level <= kMaxLevel
// (BuildTreeRecursive32's leaf rule).  Device arrays in the context's
// scratch, valid until the context's next build: per internal node i its
// split kchild[i] (children kchild[i] and kchild[i] + 1), kflags[i] (bit s:
// child s is a single key), krange[i] (first and last key), kparent[i]
// (internal parent; none for the root), flag[i] (branch), slot[i] (the
// branch's index among the branches in node order) and a zeroed arrival
// counter; kidx[slot] inverts slot.  info->nbranches receives the branch
// count.
struct Topology {
  const uint32_t *kchild, *kparent, *flag, *slot, *kidx;
  const uint8_t *kflags;
  const uint2 *krange;
  uint32_t *counter;
};
srt_status stage_topology(srt_ctx *ctx, const uint32_t *codes, size_t n, int max_leaf,
                          SceneInfo *info, Topology &t);
srt_status stage_karras(srt_ctx *ctx, const uint32_t *d_codes, size_t n,
                        uint32_t *d_child, uint8_t *d_flags);
srt_status build_batch(srt_ctx *ctx, BatchTree &bt, const float *v, const uint32_t *f,
                       const uint32_t *h_foff, int nseg);
// stack_depth: 24, 32 or 48 entries; order: NULL or a batch_ray_order.
srt_status launch_trace_batch(srt_ctx *ctx, BatchTree &bt, const srt_ray *rays,
                              srt_hit *hits, int block, int rays_per_thread,
                              unsigned long long *stats, int stack_depth = 32,
                              const uint32_t *order = nullptr);

// traversal (srt_trace.cu); max_iter 0 = the default walk cap
srt_status launch_trace(srt_accel *a, const srt_ray *d_rays, size_t n,
                        srt_hit *d_hits, const float *d_prev_normals,
                        uint32_t *d_subface, const float *d_vertex_scalar,
                        float *d_scalar_out, float *d_normal_out,
                        unsigned long long *d_stats, uint32_t flags,
                        uint32_t max_iter = 0);
// shading records of n traced rays (srt_isect.cu): BuildIntersection per hit;
// d_subface is required for tetrahedra
srt_status launch_isect(srt_accel *a, const srt_ray *d_rays, size_t n,
                        const srt_hit *d_hits, const uint32_t *d_subface,
                        srt_isect *d_isect);
}  // namespace srt
