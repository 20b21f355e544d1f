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
    for (int qi = 0; qi < len; qi++)
      solid_test<NV>(recs, queue[qi][threadIdx.x], prev, dorg, ddir, jax, t, prim, bp, bn);
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
bool solid_scene_view(const srt_solid_accel *a, srt_ctx **ctx, SceneElem &e) {
  if (!a || !a->built) return false;
  *ctx = a->ctx;
  e.kind = kSceneSolids;
  e.nprims = (uint32_t)a->n;
  e.aux = a->nv;
  e.nodes = a->dnodes.p;
  e.prims = a->drecs.as<float4>();
  e.sidx = nullptr;
  e.scene = nullptr;
  return true;
}
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
