// srt_line.cu -- LineAccel (render/render_accel_line.cc) on the GPU: capped
// cylinders between segment end points, closest hit.
//
// Build (LineAccel::BuildTree, :167-296) runs on the host like the
// reference's: top-down over an index array, a leaf below min_leaf lines or
// at max_depth, else a cut at the spatial median of the node box's longest
// axis (the position formed in double and stored as float), then the other
// axes in turn, with the two-ended partition of std::partition on the
// segment midpoints, and the object median when no axis separates them.
// Nodes are emitted in pre-order; the device copy packs each into 32 bytes.
// The lines are gathered in leaf order into 64-byte records holding the
// per-line terms of CylinderIsect (end points, max radius, |d|^2, the cap
// plane normal and offsets), computed with the reference's float operations.
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
#include <thread>
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
  size_t nlines = 0;
  int depth = 0, cap = 1;
  std::vector<LineNodeH> nodes;  // reference layout (Dump, export)
  std::vector<uint32_t> idx;
  srt::DevBuf dnodes, drecs;
};

namespace {

using srt::DevBuf;

// ------------------------------------------------------------------ build
struct LineInputs {
  const float *pos;
  const float *rad;  // per vertex, or null
  float constr;
  const uint32_t *seg;
};

inline float vrad(const LineInputs &in, uint32_t v) { return in.rad ? in.rad[v] : in.constr; }

// GetBoundingBoxOfLine (:83-116).
void line_box(const LineInputs &in, uint32_t i, float bmin[3], float bmax[3]) {
  const uint32_t a = in.seg[2 * i], b = in.seg[2 * i + 1];
  const float r0 = vrad(in, a), r1 = vrad(in, b);
  float pt[4][3];
  for (int k = 0; k < 3; k++) {
    pt[0][k] = in.pos[3 * a + k] - r0;
    pt[1][k] = in.pos[3 * a + k] + r0;
    pt[2][k] = in.pos[3 * b + k] - r1;
    pt[3][k] = in.pos[3 * b + k] + r1;
  }
  for (int k = 0; k < 3; k++) bmin[k] = bmax[k] = pt[0][k];
  for (int q = 1; q < 4; q++)
    for (int k = 0; k < 3; k++) {
      bmin[k] = (bmin[k] < pt[q][k]) ? bmin[k] : pt[q][k];
      bmax[k] = (bmax[k] > pt[q][k]) ? bmax[k] : pt[q][k];
    }
  const float eps = FLT_EPSILON * 16.0f;
  for (int k = 0; k < 3; k++) {
    bmin[k] -= bmin[k] * eps;
    bmax[k] += bmax[k] * eps;
  }
}

struct Builder {
  const std::vector<float> &box;  // 6 floats per line
  const std::vector<float> &mid;  // 3 floats per line: (p0 + p1) * 0.5
  std::vector<uint32_t> &idx;
  std::vector<LineNodeH> &nodes;
  int min_leaf, max_depth, depth_seen = 0;

  // ComputeBoundingBox (:142-163): min/max over the lines' boxes, in order.
  void range_box(size_t l, size_t r, float bmin[3], float bmax[3]) const {
    const float *b0 = &box[6 * idx[l]];
    for (int k = 0; k < 3; k++) {
      bmin[k] = b0[k];
      bmax[k] = b0[3 + k];
    }
    for (size_t i = l; i < r; i++) {
      const float *b = &box[6 * idx[i]];
      for (int k = 0; k < 3; k++) {
        bmin[k] = (bmin[k] < b[k]) ? bmin[k] : b[k];
        bmax[k] = (bmax[k] > b[3 + k]) ? bmax[k] : b[3 + k];
      }
    }
  }

  // std::partition's two-ended scan: lines whose midpoint lies below pos
  // first.
  size_t partition(size_t first, size_t last, int axis, float pos) {
    for (;;) {
      while (first != last && mid[3 * idx[first] + axis] < pos) first++;
      if (first == last) return first;
      last--;
      while (first != last && !(mid[3 * idx[last] + axis] < pos)) last--;
      if (first == last) return first;
      std::swap(idx[first], idx[last]);
      first++;
    }
  }

  // The cut of [l, r) (idx partitioned in place): the split and its axis.
  size_t cut(size_t l, size_t r, const float bmin[3], const float bmax[3], int &axis) {
    float bsize[3];
    for (int k = 0; k < 3; k++) bsize[k] = bmax[k] - bmin[k];
    int longest = 0;
    float m = bsize[0];
    if (m < bsize[1]) {
      m = bsize[1];
      longest = 1;
    }
    if (m < bsize[2]) longest = 2;
    size_t split = l;
    for (int t = 0; t < 3; t++) {
      axis = (longest + t) % 3;
      const float pos = (float)((double)bmin[axis] + 0.5 * (double)bsize[axis]);
      split = partition(l, r, axis, pos);
      if (split != l && split != r) break;
      split = l + ((r - l) >> 1);
    }
    return split;
  }

  size_t build(size_t l, size_t r, int depth) {
    const size_t off = nodes.size();
    nodes.push_back(LineNodeH{});
    depth_seen = std::max(depth_seen, depth);
    float bmin[3], bmax[3];
    range_box(l, r, bmin, bmax);
    const size_t n = r - l;
    if (n < (size_t)min_leaf || depth >= max_depth) {
      LineNodeH &nd = nodes[off];
      std::memcpy(nd.bmin, bmin, sizeof(bmin));
      std::memcpy(nd.bmax, bmax, sizeof(bmax));
      nd.flag = 1;
      nd.data[0] = (uint32_t)n;
      nd.data[1] = (uint32_t)l;
      return off;
    }
    int axis = 0;
    const size_t split = cut(l, r, bmin, bmax, axis);
    nodes[off].axis = axis;
    const size_t left = build(l, split, depth + 1);
    const size_t right = build(split, r, depth + 1);
    LineNodeH &nd = nodes[off];
    nd.data[0] = (uint32_t)left;
    nd.data[1] = (uint32_t)right;
    std::memcpy(nd.bmin, bmin, sizeof(bmin));
    std::memcpy(nd.bmax, bmax, sizeof(bmax));
    return off;
  }
};

// The same tree with the top `par` levels' subtrees built on their own
// threads (their idx ranges are disjoint) into local arrays, then laid out
// in pre-order: the node, its left subtree, its right subtree, child indices
// moved by the subtrees' offsets.
void build_par(const std::vector<float> &box, const std::vector<float> &mid,
               std::vector<uint32_t> &idx, int min_leaf, int max_depth, size_t l, size_t r,
               int depth, int par, std::vector<LineNodeH> &out, int &depth_seen) {
  Builder B{box, mid, idx, out, min_leaf, max_depth};
  const size_t n = r - l;
  if (par <= 0 || n < (size_t)min_leaf || depth >= max_depth || n < 4096) {
    B.depth_seen = depth;
    B.build(l, r, depth);
    depth_seen = std::max(depth_seen, B.depth_seen);
    return;
  }
  out.push_back(LineNodeH{});
  depth_seen = std::max(depth_seen, depth);
  float bmin[3], bmax[3];
  B.range_box(l, r, bmin, bmax);
  int axis = 0;
  const size_t split = B.cut(l, r, bmin, bmax, axis);
  std::vector<LineNodeH> L, R;
  int dl = 0, dr = 0;
  std::thread t([&] {
    build_par(box, mid, idx, min_leaf, max_depth, l, split, depth + 1, par - 1, L, dl);
  });
  build_par(box, mid, idx, min_leaf, max_depth, split, r, depth + 1, par - 1, R, dr);
  t.join();
  depth_seen = std::max(depth_seen, std::max(dl, dr));
  LineNodeH &root = out[0];
  std::memcpy(root.bmin, bmin, sizeof(bmin));
  std::memcpy(root.bmax, bmax, sizeof(bmax));
  root.axis = axis;
  root.data[0] = 1;
  root.data[1] = (uint32_t)(1 + L.size());
  out.reserve(1 + L.size() + R.size());
  for (const auto *sub : {&L, &R}) {
    const uint32_t shift = (uint32_t)out.size();
    for (LineNodeH nd : *sub) {
      if (!nd.flag) {
        nd.data[0] += shift;
        nd.data[1] += shift;
      }
      out.push_back(nd);
    }
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

// A host copy of an input that may live on the device.
template <typename T>
srt_status host_copy(const T *p, size_t count, std::vector<T> &buf, const T **out) {
  if (!p || !srt::is_device_ptr(p)) {
    *out = p;
    return SRT_OK;
  }
  buf.resize(count ? count : 1);
  cudaError_t e = cudaMemcpy(buf.data(), p, count * sizeof(T), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return srt::cuda_status(e, "line input copy");
  *out = buf.data();
  return SRT_OK;
}

}  // namespace

namespace srt {
uint64_t line_accel_bytes(const srt_line_accel *a) { return a->dnodes.cap + a->drecs.cap; }
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
  std::vector<float> hp, hr;
  std::vector<uint32_t> hs;
  const float *pos, *rad;
  const uint32_t *seg;
  srt_status s = host_copy(positions, nverts * 3, hp, &pos);
  if (s == SRT_OK) s = host_copy(radius, radius ? nverts : 0, hr, &rad);
  if (s == SRT_OK) s = host_copy(segments, nlines * 2, hs, &seg);
  if (s != SRT_OK) return s;
  for (size_t i = 0; i < 2 * nlines; i++)
    if (seg[i] >= nverts) {
      set_error("srt_line_build: a segment names a vertex beyond nverts");
      return SRT_ERR_INVALID;
    }
  const LineInputs in{pos, rad, constant_radius, seg};
  std::vector<float> box(6 * nlines), mid(3 * nlines);
  for (size_t i = 0; i < nlines; i++) {
    line_box(in, (uint32_t)i, &box[6 * i], &box[6 * i + 3]);
    const uint32_t p = seg[2 * i], q = seg[2 * i + 1];
    for (int k = 0; k < 3; k++) mid[3 * i + k] = (pos[3 * p + k] + pos[3 * q + k]) * 0.5f;
  }
  a->built = false;
  a->idx.resize(nlines);
  for (size_t i = 0; i < nlines; i++) a->idx[i] = (uint32_t)i;
  a->nodes.clear();
  int depth_seen = 0;
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  int par = 0;
  while ((1u << (par + 1)) <= std::min(hw, 16u)) par++;
  build_par(box, mid, a->idx, min_leaf, max_depth, 0, nlines, 0, par, a->nodes, depth_seen);
  if (a->nodes.size() >= (1u << 29)) {
    set_error("srt_line_build: more than 2^29 nodes");
    return SRT_ERR_INVALID;
  }
  std::vector<LNode> dn(a->nodes.size());
  for (size_t i = 0; i < a->nodes.size(); i++) {
    const LineNodeH &h = a->nodes[i];
    LNode &d = dn[i];
    for (int k = 0; k < 3; k++) {
      d.bmin[k] = h.bmin[k];
      d.bmax[k] = h.bmax[k];
    }
    if (h.flag) {
      d.w0 = h.data[1];
      d.w1 = kLineLeaf | h.data[0];
    } else {
      d.w0 = h.data[0];
      d.w1 = h.data[1] | ((uint32_t)h.axis << 29);
    }
  }
  cudaError_t e;
  if ((e = a->dnodes.ensure(dn.size() * sizeof(LNode))) != cudaSuccess ||
      (e = a->drecs.ensure(nlines * sizeof(LineRec))) != cudaSuccess)
    return cuda_status(e, "line accel");
  e = cudaMemcpyAsync(a->dnodes.p, dn.data(), dn.size() * sizeof(LNode),
                      cudaMemcpyHostToDevice, ctx->stream);
  if (e != cudaSuccess) return cuda_status(e, "line nodes");
  DevBuf sp, sr, ss, so;
  const void *dp, *dr, *ds;
  if ((s = line_view(ctx, positions, nverts * 12, sp, &dp)) != SRT_OK) return s;
  if ((s = line_view(ctx, radius, radius ? nverts * 4 : 0, sr, &dr)) != SRT_OK) return s;
  if ((s = line_view(ctx, segments, nlines * 8, ss, &ds)) != SRT_OK) return s;
  if ((e = so.ensure(nlines * 4)) != cudaSuccess) return cuda_status(e, "line order");
  e = cudaMemcpyAsync(so.p, a->idx.data(), nlines * 4, cudaMemcpyHostToDevice, ctx->stream);
  if (e != cudaSuccess) return cuda_status(e, "line order");
  const unsigned grid = (unsigned)std::min<size_t>((nlines + 255) / 256, 4096);
  line_rec_kernel<<<grid, 256, 0, ctx->stream>>>(
      static_cast<const float *>(dp), static_cast<const float *>(dr), constant_radius,
      static_cast<const uint32_t *>(ds), so.as<uint32_t>(), nlines, a->drecs.as<LineRec>());
  ctx->launches++;
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_status(e, "line records");
  // the staged inputs are freed on return: finish with them first
  if ((e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess)
    return cuda_status(e, "line build");
  a->nlines = nlines;
  a->depth = depth_seen;
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
    bmin[k] = a->nodes[0].bmin[k];
    bmax[k] = a->nodes[0].bmax[k];
  }
  return SRT_OK;
}

SRT_API srt_status srt_line_info(srt_line_accel *a, uint64_t *nlines, uint64_t *nnodes,
                                 int32_t *depth) {
  if (!a) return SRT_ERR_INVALID;
  if (nlines) *nlines = a->built ? a->nlines : 0;
  if (nnodes) *nnodes = a->built ? a->nodes.size() : 0;
  if (depth) *depth = a->built ? a->depth : 0;
  return SRT_OK;
}

SRT_API srt_status srt_line_export(srt_line_accel *a, void *nodes, uint32_t *indices) {
  if (!a || !a->built) return SRT_ERR_INVALID;
  if (nodes) std::memcpy(nodes, a->nodes.data(), a->nodes.size() * sizeof(LineNodeH));
  if (indices) std::memcpy(indices, a->idx.data(), a->idx.size() * sizeof(uint32_t));
  return SRT_OK;
}

SRT_API srt_status srt_line_dump(srt_line_accel *a, const char *path) {
  if (!a || !path || !a->built) return SRT_ERR_INVALID;
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
