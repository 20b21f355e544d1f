// srt_capi.cu -- the extern "C" surface of libsurface_rt (include/surface_rt.h).
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include <type_traits>

#include "srt_internal.cuh"

namespace srt {

static thread_local std::string g_last_error;

void set_error(const std::string &msg) { g_last_error = msg; }

srt_status cuda_status(cudaError_t e, const char *what) {
  if (e == cudaSuccess) return SRT_OK;
  set_error(std::string(what) + ": " + cudaGetErrorString(e));
  return e == cudaErrorMemoryAllocation ? SRT_ERR_NO_MEMORY : SRT_ERR_CUDA;
}

std::atomic<uint64_t> g_buffer_epoch{0};

cudaError_t DevBuf::ensure(size_t bytes) {
  if (bytes <= cap && p) return cudaSuccess;
  release();
  size_t want = bytes < 256 ? 256 : bytes;
  cudaError_t e = cudaMalloc(&p, want);
  if (e != cudaSuccess) {
    p = nullptr;
    cap = 0;
    cudaGetLastError();
    return e;
  }
  cap = want;
  return cudaSuccess;
}

void DevBuf::release() {
  if (p) {
    cudaFree(p);
    g_buffer_epoch.fetch_add(1, std::memory_order_relaxed);
  }
  p = nullptr;
  cap = 0;
}

bool is_device_ptr(const void *p) {
  if (!p) return false;
  cudaPointerAttributes at;
  cudaError_t e = cudaPointerGetAttributes(&at, p);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

// A page-locked host array that the device reaches through unified
// addressing (cudaHostAlloc / cudaHostRegister memory is mapped): the device
// address to write it directly, else null (pageable memory).
static void *mapped_ptr(void *p) {
  if (!p) return nullptr;
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return at.type == cudaMemoryTypeHost ? at.devicePointer : nullptr;
}

// Device view of a caller array: the pointer itself, or a copy into `stage`.
static srt_status device_view(srt_ctx *ctx, const void *p, size_t bytes, DevBuf &stage,
                              const void **out) {
  if (!p || bytes == 0) {
    *out = p;
    return SRT_OK;
  }
  if (is_device_ptr(p)) {
    *out = p;
    return SRT_OK;
  }
  cudaError_t e = stage.ensure(bytes);
  if (e != cudaSuccess) return cuda_status(e, "staging allocation");
  e = cudaMemcpyAsync(stage.p, p, bytes, cudaMemcpyHostToDevice, ctx->stream);
  if (e != cudaSuccess) return cuda_status(e, "host to device copy");
  *out = stage.p;
  return SRT_OK;
}

// Waits for the context stream and reports (then clears) the kernels' limit
// flags.
srt_status check_device_errors(srt_ctx *ctx) {
  cudaError_t e = cudaMemcpyAsync(ctx->h_err, ctx->d_err, 4, cudaMemcpyDeviceToHost,
                                  ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return cuda_status(e, "synchronize");
  uint32_t flags = *ctx->h_err;
  if (flags) {
    cudaMemsetAsync(ctx->d_err, 0, 4, ctx->stream);
    cudaStreamSynchronize(ctx->stream);
    std::string m = "kernel limit hit:";
    if (flags & kErrStack) m += " traversal stack overflow;";
    if (flags & kErrIter) m += " traversal iteration cap;";
    if (flags & kErrTree) m += " malformed tree / leaf too large;";
    if (flags & kErrSortWait) m += " sort pass gave up waiting on an earlier tile;";
    set_error(m);
    return SRT_ERR_LIMIT;
  }
  return SRT_OK;
}

static srt_status read_scene(srt_accel *a) {
  if (!a->built) {
    set_error("accel not built");
    return SRT_ERR_INVALID;
  }
  if (!a->host_scene_valid) {
    cudaError_t e = cudaMemcpyAsync(&a->host_scene, a->scene.p, sizeof(SceneInfo),
                                    cudaMemcpyDeviceToHost, a->ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(a->ctx->stream);
    if (e != cudaSuccess) return cuda_status(e, "read scene info");
    a->host_scene_valid = true;
  }
  return SRT_OK;
}

static size_t node_count(const srt_accel *a) {
  size_t nb = a->host_scene.nbranches;
  return a->kind == SRT_TETRAHEDRA ? 2 * nb + 1 : nb;
}

static srt_status build_common(srt_accel *a, const float *verts, size_t nverts,
                               const uint32_t *prims, size_t nprims, int per_prim,
                               const float *radius, float constr) {
  if (!a || !verts) {
    set_error("NULL argument");
    return SRT_ERR_INVALID;
  }
  if (nprims < 2 || nprims >= (1u << 30)) {
    set_error("primitive count must be in [2, 2^30)");
    return SRT_ERR_INVALID;
  }
  if (per_prim > 0 && (!prims || nverts == 0)) {
    set_error("NULL primitive index array");
    return SRT_ERR_INVALID;
  }
  srt_ctx *ctx = a->ctx;
  if (cudaSetDevice(ctx->device) != cudaSuccess) return cuda_status(cudaGetLastError(), "device");
  const void *dv = nullptr, *df = nullptr, *dr = nullptr;
  size_t vbytes = (per_prim > 0 ? nverts : nprims) * 3 * sizeof(float);
  srt_status s = device_view(ctx, verts, vbytes, a->in_verts, &dv);
  if (s != SRT_OK) return s;
  if (per_prim > 0) {
    s = device_view(ctx, prims, nprims * per_prim * sizeof(uint32_t), a->in_faces, &df);
    if (s != SRT_OK) return s;
  }
  if (radius) {
    s = device_view(ctx, radius, nprims * sizeof(float), a->in_radius, &dr);
    if (s != SRT_OK) return s;
  }
  if (dv != verts || (df && df != prims) || (dr && dr != radius)) {
    // host inputs were copied: a ray array staged next (prestage_rays) waits
    // for these copies, so the build's inputs cross the host link first
    cudaError_t e = cudaSuccess;
    if (!ctx->ev_inputs) e = cudaEventCreateWithFlags(&ctx->ev_inputs, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventRecord(ctx->ev_inputs, ctx->stream);
    if (e != cudaSuccess) return cuda_status(e, "input copy event");
    ctx->inputs_pending = true;
  }
  a->n = nprims;
  a->dbl = false;
  a->src_verts = static_cast<const float *>(dv);
  a->src_faces = static_cast<const uint32_t *>(df);
  s = build_accel(a, static_cast<const float *>(dv), static_cast<const uint32_t *>(df),
                  static_cast<const float *>(dr), constr, nprims);
  a->built = (s == SRT_OK);
  return s;
}

// Tetrahedra with double-precision positions.
static srt_status build_tet_d(srt_accel *a, const double *verts, size_t nverts,
                              const uint32_t *tets, size_t ntets) {
  if (!a || !verts || !tets || nverts == 0) {
    set_error("NULL argument");
    return SRT_ERR_INVALID;
  }
  if (a->kind != SRT_TETRAHEDRA) {
    set_error("accel kind is not tetrahedra");
    return SRT_ERR_INVALID;
  }
  if (ntets < 2 || ntets >= (1u << 30)) {
    set_error("primitive count must be in [2, 2^30)");
    return SRT_ERR_INVALID;
  }
  srt_ctx *ctx = a->ctx;
  if (cudaSetDevice(ctx->device) != cudaSuccess) return cuda_status(cudaGetLastError(), "device");
  const void *dv = nullptr, *df = nullptr;
  srt_status s = device_view(ctx, verts, nverts * 3 * sizeof(double), a->in_dverts, &dv);
  if (s != SRT_OK) return s;
  if ((s = device_view(ctx, tets, ntets * 4 * sizeof(uint32_t), a->in_faces, &df)) != SRT_OK)
    return s;
  if (dv != verts || df != tets) {  // as build_common: staged rays wait for these copies
    cudaError_t e = cudaSuccess;
    if (!ctx->ev_inputs) e = cudaEventCreateWithFlags(&ctx->ev_inputs, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventRecord(ctx->ev_inputs, ctx->stream);
    if (e != cudaSuccess) return cuda_status(e, "input copy event");
    ctx->inputs_pending = true;
  }
  cudaError_t e = a->in_verts.ensure(nverts * 3 * sizeof(float));
  if (e != cudaSuccess) return cuda_status(e, "rounded positions");
  a->n = ntets;
  a->dbl = true;
  a->host_scene_valid = false;
  a->src_verts = a->in_verts.as<float>();
  a->src_faces = static_cast<const uint32_t *>(df);
  s = build_tet_double(a, static_cast<const double *>(dv), nverts,
                       static_cast<const uint32_t *>(df), ntets, a->in_verts.as<float>());
  a->built = (s == SRT_OK);
  return s;
}

}  // namespace srt

using namespace srt;

extern "C" {

SRT_API const char *srt_last_error(void) { return g_last_error.c_str(); }

SRT_API uint64_t srt_ctx_launch_count(srt_ctx *ctx) { return ctx ? ctx->launches : 0; }

SRT_API srt_status srt_ctx_create(int device, srt_ctx **out) {
  if (!out) return SRT_ERR_INVALID;
  *out = nullptr;
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    set_error("no CUDA device available");
    return SRT_ERR_CUDA;
  }
  if (device < 0 || device >= ndev) {
    set_error("device index out of range");
    return SRT_ERR_INVALID;
  }
  if ((e = cudaSetDevice(device)) != cudaSuccess) return cuda_status(e, "cudaSetDevice");
  srt_ctx *c = new (std::nothrow) srt_ctx();
  if (!c) return SRT_ERR_NO_MEMORY;
  c->device = device;
  cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device);
  if ((e = cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking)) != cudaSuccess) {
    delete c;
    return cuda_status(e, "stream");
  }
  c->stream = c->own_stream;
  if ((e = cudaMalloc(&c->d_err, 4)) != cudaSuccess ||
      (e = cudaMallocHost(&c->h_err, 4)) != cudaSuccess) {
    srt_ctx_destroy(c);
    return cuda_status(e, "error word");
  }
  cudaMemset(c->d_err, 0, 4);
  *c->h_err = 0;
  *out = c;
  return SRT_OK;
}

SRT_API srt_status srt_ctx_destroy(srt_ctx *c) {
  if (!c) return SRT_OK;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  DevBuf *bufs[] = {&c->s_keys2, &c->s_vals2, &c->s_hist, &c->s_scan, &c->s_kchild,
                    &c->s_kflags, &c->s_krange, &c->s_kparent, &c->s_lparent,
                    &c->s_counter, &c->s_ibox, &c->s_flag, &c->s_slot, &c->s_partial,
                    &c->s_stage_in, &c->s_stage_out, &c->s_stage_aux, &c->s_stage_sub,
                    &c->s_stage_scal, &c->s_stage_norm, &c->s_defer, &c->s_spawn, &c->s_rkey,
                    &c->s_rorder, &c->s_isect_sub, &c->s_stage_isect, &c->s_keys3,
                    &c->s_vals3, &c->s_status, &c->s_lscan, &c->s_rays_in,
                    &c->s_kidx, &c->s_kprefix};
  if (c->copy_stream) cudaStreamSynchronize(c->copy_stream);
  for (DevBuf *b : bufs) b->release();
  if (c->ev_copy) cudaEventDestroy(c->ev_copy);
  if (c->ev_inputs) cudaEventDestroy(c->ev_inputs);
  if (c->ev_free) cudaEventDestroy(c->ev_free);
  if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
  if (c->d_err) cudaFree(c->d_err);
  if (c->h_err) cudaFreeHost(c->h_err);
  if (c->own_stream) cudaStreamDestroy(c->own_stream);
  delete c;
  return SRT_OK;
}

SRT_API srt_status srt_ctx_set_stream(srt_ctx *c, void *stream) {
  if (!c) return SRT_ERR_INVALID;
  c->stream = stream ? static_cast<cudaStream_t>(stream) : c->own_stream;
  return SRT_OK;
}

SRT_API void *srt_ctx_get_stream(srt_ctx *c) { return c ? (void *)c->stream : nullptr; }

SRT_API srt_status srt_ctx_synchronize(srt_ctx *c) {
  if (!c) return SRT_ERR_INVALID;
  cudaSetDevice(c->device);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_status(e, "pending error");
  return check_device_errors(c);
}

SRT_API srt_status srt_accel_create(srt_ctx *ctx, srt_kind kind, srt_accel **out) {
  if (!ctx || !out || kind < SRT_TRIANGLES || kind > SRT_SPHERES) {
    set_error("invalid accel arguments");
    return SRT_ERR_INVALID;
  }
  srt_accel *a = new (std::nothrow) srt_accel();
  if (!a) return SRT_ERR_NO_MEMORY;
  a->ctx = ctx;
  a->kind = kind;
  *out = a;
  return SRT_OK;
}

SRT_API srt_status srt_accel_destroy(srt_accel *a) {
  if (!a) return SRT_OK;
  cudaSetDevice(a->ctx->device);
  cudaStreamSynchronize(a->ctx->stream);
  DevBuf *bufs[] = {&a->nodes, &a->indices, &a->codes, &a->prims, &a->scene,
                    &a->in_verts, &a->in_faces, &a->in_radius};
  for (DevBuf *b : bufs) b->release();
  delete a;
  return SRT_OK;
}

SRT_API srt_status srt_accel_build_triangles(srt_accel *a, const float *vertices,
                                             size_t nvertices, const uint32_t *faces,
                                             size_t nfaces) {
  if (a && a->kind != SRT_TRIANGLES) {
    set_error("accel kind is not triangles");
    return SRT_ERR_INVALID;
  }
  return build_common(a, vertices, nvertices, faces, nfaces, 3, nullptr, 0.0f);
}

SRT_API srt_status srt_accel_build_tetrahedra(srt_accel *a, const float *vertices,
                                              size_t nvertices, const uint32_t *tets,
                                              size_t ntets) {
  if (a && a->kind != SRT_TETRAHEDRA) {
    set_error("accel kind is not tetrahedra");
    return SRT_ERR_INVALID;
  }
  return build_common(a, vertices, nvertices, tets, ntets, 4, nullptr, 0.0f);
}

SRT_API srt_status srt_accel_build_tetrahedra_double(srt_accel *a, const double *vertices,
                                                     size_t nvertices, const uint32_t *tets,
                                                     size_t ntets) {
  return build_tet_d(a, vertices, nvertices, tets, ntets);
}

SRT_API srt_status srt_accel_build_spheres(srt_accel *a, const float *centers,
                                           const float *radius, float constant_radius,
                                           size_t n) {
  if (a && a->kind != SRT_SPHERES) {
    set_error("accel kind is not spheres");
    return SRT_ERR_INVALID;
  }
  return build_common(a, centers, n, nullptr, n, 0, radius, constant_radius);
}

static srt_status create_and_build(srt_ctx *ctx, srt_kind kind, srt_accel **out,
                                   const float *v, size_t nv, const uint32_t *f,
                                   size_t n, const float *rad, float cr) {
  if (!out) return SRT_ERR_INVALID;
  srt_accel *a = nullptr;
  srt_status s = srt_accel_create(ctx, kind, &a);
  if (s != SRT_OK) return s;
  if (kind == SRT_TRIANGLES)
    s = srt_accel_build_triangles(a, v, nv, f, n);
  else if (kind == SRT_TETRAHEDRA)
    s = srt_accel_build_tetrahedra(a, v, nv, f, n);
  else
    s = srt_accel_build_spheres(a, v, rad, cr, n);
  if (s != SRT_OK) {
    srt_accel_destroy(a);
    return s;
  }
  *out = a;
  return SRT_OK;
}

SRT_API srt_status srt_build_triangles(srt_ctx *ctx, const float *vertices, size_t nv,
                                       const uint32_t *faces, size_t nfaces,
                                       srt_accel **out) {
  return create_and_build(ctx, SRT_TRIANGLES, out, vertices, nv, faces, nfaces, nullptr, 0);
}

SRT_API srt_status srt_build_tetrahedra(srt_ctx *ctx, const float *vertices, size_t nv,
                                        const uint32_t *tets, size_t ntets,
                                        srt_accel **out) {
  return create_and_build(ctx, SRT_TETRAHEDRA, out, vertices, nv, tets, ntets, nullptr, 0);
}

SRT_API srt_status srt_build_spheres(srt_ctx *ctx, const float *centers,
                                     const float *radius, float constant_radius, size_t n,
                                     srt_accel **out) {
  return create_and_build(ctx, SRT_SPHERES, out, centers, n, nullptr, n, radius,
                          constant_radius);
}

SRT_API srt_status srt_accel_info_get(srt_accel *a, srt_accel_info *info) {
  if (!a || !info) return SRT_ERR_INVALID;
  srt_status s = read_scene(a);
  if (s != SRT_OK) return s;
  memset(info, 0, sizeof(*info));
  info->kind = a->kind;
  info->node_bytes = a->kind == SRT_TETRAHEDRA ? (int)sizeof(NodeT) : (int)sizeof(Node2);
  info->num_prims = a->n;
  info->num_nodes = node_count(a);
  info->num_branches = a->host_scene.nbranches;
  info->num_leaves = a->host_scene.nbranches + 1;  // full binary tree
  for (int k = 0; k < 3; k++) {
    info->scene_min[k] = a->host_scene.lo[k];
    info->scene_max[k] = a->host_scene.hi[k];
  }
  info->eps_scale = a->host_scene.eps_scale;
  return SRT_OK;
}

SRT_API srt_status srt_accel_export(srt_accel *a, void *nodes, uint32_t *indices,
                                    uint32_t *codes) {
  if (!a) return SRT_ERR_INVALID;
  srt_status s = read_scene(a);
  if (s != SRT_OK) return s;
  cudaStream_t st = a->ctx->stream;
  size_t nb = node_count(a) * (a->kind == SRT_TETRAHEDRA ? sizeof(NodeT) : sizeof(Node2));
  cudaError_t e = cudaSuccess;
  if (nodes) e = cudaMemcpyAsync(nodes, a->nodes.p, nb, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess && indices)
    e = cudaMemcpyAsync(indices, a->indices.p, a->n * 4, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess && codes)
    e = cudaMemcpyAsync(codes, a->codes.p, a->n * 4, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  return cuda_status(e, "export");
}

SRT_API srt_status srt_accel_bbox(srt_accel *a, double bmin[3], double bmax[3]) {
  if (!a || !bmin || !bmax) return SRT_ERR_INVALID;
  srt_status s = read_scene(a);
  if (s != SRT_OK) return s;
  float lo[3], hi[3];
  cudaStream_t st = a->ctx->stream;
  if (a->kind == SRT_TETRAHEDRA) {
    NodeT root;
    cudaError_t e = cudaMemcpyAsync(&root, a->nodes.p, sizeof(root), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_status(e, "bbox");
    lo[0] = root.a.x; lo[1] = root.a.y; lo[2] = root.a.z;
    hi[0] = root.b.x; hi[1] = root.b.y; hi[2] = root.b.z;
  } else {
    Node2 root;
    cudaError_t e = cudaMemcpyAsync(&root, a->nodes.p, sizeof(root), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_status(e, "bbox");
    // MergeBoundingBox of the two root slots (left first)
    const float c0l[3] = {root.a.x, root.a.y, root.a.z}, c0h[3] = {root.a.w, root.b.x, root.b.y};
    const float c1l[3] = {root.b.z, root.b.w, root.c.x}, c1h[3] = {root.c.y, root.c.z, root.c.w};
    for (int k = 0; k < 3; k++) {
      lo[k] = (c1l[k] < c0l[k]) ? c1l[k] : c0l[k];
      hi[k] = (c0h[k] < c1h[k]) ? c1h[k] : c0h[k];
    }
  }
  for (int k = 0; k < 3; k++) {
    bmin[k] = lo[k];
    bmax[k] = hi[k];
  }
  return SRT_OK;
}

// Reference Dump() records: TriangleNode (64 B: bmin[2][3], bmax[2][3], int
// flag, int axis, uint data[2]), TetraNode (40 B: bmin[3], bmax[3], int flag,
// int axis, uint data[2]), ParticleNode (60 B: bmin[2][3], bmax[2][3], uint
// data[2], short flag, short axis).  Nodes are written in depth-first order
// (left first), the order of the reference's sequential build; fields the
// reference leaves uninitialised (a leaf's second slot, its axis) are zero.
namespace {
struct DumpNode {
  float lo[2][3], hi[2][3];
  int32_t leaf, axis;
  uint32_t d0, d1;
};

void dump_node2(const Node2 *nd, uint32_t ni, std::vector<DumpNode> &out) {
  const Node2 &x = nd[ni];
  const float box[2][6] = {{x.a.x, x.a.y, x.a.z, x.a.w, x.b.x, x.b.y},
                           {x.b.z, x.b.w, x.c.x, x.c.y, x.c.z, x.c.w}};
  const uint32_t ref[2] = {x.d.x, x.d.y};
  const uint32_t cnt[2] = {x.d.z & kCountMask, x.d.w & kCountMask};
  size_t me = out.size();
  out.push_back(DumpNode());
  DumpNode &b = out[me];
  memset(&b, 0, sizeof(b));
  b.leaf = 0;
  b.axis = (int32_t)(x.d.z >> 30);
  for (int k = 0; k < 2; k++)
    for (int c = 0; c < 3; c++) {
      b.lo[k][c] = box[k][c];
      b.hi[k][c] = box[k][3 + c];
    }
  uint32_t child[2];
  for (int k = 0; k < 2; k++) {
    child[k] = (uint32_t)out.size();
    if (cnt[k] == 0) {
      dump_node2(nd, ref[k], out);
    } else {
      DumpNode l;
      memset(&l, 0, sizeof(l));
      l.leaf = 1;
      for (int c = 0; c < 3; c++) {
        l.lo[0][c] = box[k][c];
        l.hi[0][c] = box[k][3 + c];
      }
      l.d0 = cnt[k];
      l.d1 = ref[k];
      out.push_back(l);
    }
  }
  out[me].d0 = child[0];
  out[me].d1 = child[1];
}

void dump_tet(const NodeT *nd, uint32_t ni, std::vector<DumpNode> &out) {
  const NodeT &x = nd[ni];
  uint32_t meta, ref;
  memcpy(&meta, &x.a.w, 4);
  memcpy(&ref, &x.b.w, 4);
  size_t me = out.size();
  DumpNode b;
  memset(&b, 0, sizeof(b));
  b.lo[0][0] = x.a.x; b.lo[0][1] = x.a.y; b.lo[0][2] = x.a.z;
  b.hi[0][0] = x.b.x; b.hi[0][1] = x.b.y; b.hi[0][2] = x.b.z;
  if (meta & kLeafBit) {
    b.leaf = 1;
    b.d0 = meta & kCountMask;
    b.d1 = ref;
    out.push_back(b);
    return;
  }
  b.axis = (int32_t)(meta & 3u);
  out.push_back(b);
  uint32_t c0 = (uint32_t)out.size();
  dump_tet(nd, ref, out);
  uint32_t c1 = (uint32_t)out.size();
  dump_tet(nd, ref + 1, out);
  out[me].d0 = c0;
  out[me].d1 = c1;
}
}  // namespace

SRT_API srt_status srt_accel_dump(srt_accel *a, const char *path) {
  if (!a || !path) return SRT_ERR_INVALID;
  srt_accel_info info;
  srt_status s = srt_accel_info_get(a, &info);
  if (s != SRT_OK) return s;
  std::vector<unsigned char> raw(info.num_nodes * info.node_bytes);
  std::vector<uint32_t> idx(a->n);
  s = srt_accel_export(a, raw.data(), idx.data(), nullptr);
  if (s != SRT_OK) return s;
  std::vector<DumpNode> out;
  out.reserve(info.num_branches * 2 + 2);
  if (a->kind == SRT_TETRAHEDRA)
    dump_tet(reinterpret_cast<const NodeT *>(raw.data()), 0u, out);
  else
    dump_node2(reinterpret_cast<const Node2 *>(raw.data()), 0u, out);
  FILE *fp = fopen(path, "wb");
  if (!fp) {
    set_error(std::string("cannot write ") + path);
    return SRT_ERR_INVALID;
  }
  unsigned long long nn = out.size(), ni = idx.size();
  bool ok = fwrite(&nn, 8, 1, fp) == 1;
  for (const DumpNode &d : out) {
    unsigned char rec[64];
    size_t sz = 0;
    memset(rec, 0, sizeof(rec));
    if (a->kind == SRT_TRIANGLES) {
      memcpy(rec, d.lo, 24);
      memcpy(rec + 24, d.hi, 24);
      memcpy(rec + 48, &d.leaf, 4);
      memcpy(rec + 52, &d.axis, 4);
      memcpy(rec + 56, &d.d0, 4);
      memcpy(rec + 60, &d.d1, 4);
      sz = 64;
    } else if (a->kind == SRT_SPHERES) {
      memcpy(rec, d.lo, 24);
      memcpy(rec + 24, d.hi, 24);
      memcpy(rec + 48, &d.d0, 4);
      memcpy(rec + 52, &d.d1, 4);
      int16_t fl = (int16_t)d.leaf, ax = (int16_t)d.axis;
      memcpy(rec + 56, &fl, 2);
      memcpy(rec + 58, &ax, 2);
      sz = 60;
    } else {
      memcpy(rec, d.lo[0], 12);
      memcpy(rec + 12, d.hi[0], 12);
      memcpy(rec + 24, &d.leaf, 4);
      memcpy(rec + 28, &d.axis, 4);
      memcpy(rec + 32, &d.d0, 4);
      memcpy(rec + 36, &d.d1, 4);
      sz = 40;
    }
    ok = ok && fwrite(rec, 1, sz, fp) == sz;
  }
  ok = ok && fwrite(&ni, 8, 1, fp) == 1;
  ok = ok && fwrite(idx.data(), 4, idx.size(), fp) == idx.size();
  ok = (fclose(fp) == 0) && ok;
  if (!ok) {
    set_error(std::string("short write to ") + path);
    return SRT_ERR_INVALID;
  }
  return SRT_OK;
}

// ---------------------------------------------------------------- zero copy
// Device-visible address of page-locked host memory (cudaMallocHost /
// cudaHostAlloc memory is mapped into the device's address space under
// unified addressing), or nullptr for device or pageable memory.
static void *mapped_host(const void *p) {
  if (!p) return nullptr;
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  if (at.type != cudaMemoryTypeHost || !at.devicePointer) return nullptr;
  return at.devicePointer;
}

// A large page-locked host ray array is copied to the device on the
// context's side stream, which starts at once: the copy overlaps whatever
// the context stream is still running (typically the build that precedes a
// trace), and the context stream waits for it before the trace.  Small
// arrays are read in place over the host link (*out unchanged).
#ifndef SRT_PRESTAGE_MIN_BYTES
#define SRT_PRESTAGE_MIN_BYTES ((size_t)1 << 20)
#endif
static srt_status prestage_rays(srt_ctx *ctx, const srt_ray *rays, size_t n,
                                const srt_ray **out) {
  const size_t bytes = n * sizeof(srt_ray);
  if (bytes < SRT_PRESTAGE_MIN_BYTES) return SRT_OK;
  cudaError_t e;
  if (!ctx->copy_stream) {
    if ((e = cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking)) !=
            cudaSuccess ||
        (e = cudaEventCreateWithFlags(&ctx->ev_copy, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&ctx->ev_free, cudaEventDisableTiming)) != cudaSuccess)
      return cuda_status(e, "ray staging stream");
  }
  if (bytes > ctx->s_rays_in.cap) {
    // a reallocation: nothing of the old buffer may still be read
    if (ctx->ev_free_recorded && (e = cudaEventSynchronize(ctx->ev_free)) != cudaSuccess)
      return cuda_status(e, "ray staging");
    if ((e = ctx->s_rays_in.ensure(bytes)) != cudaSuccess) return cuda_status(e, "ray staging");
  }
  if (ctx->ev_free_recorded &&
      (e = cudaStreamWaitEvent(ctx->copy_stream, ctx->ev_free, 0)) != cudaSuccess)
    return cuda_status(e, "ray staging");
  if (ctx->inputs_pending) {
    if ((e = cudaStreamWaitEvent(ctx->copy_stream, ctx->ev_inputs, 0)) != cudaSuccess)
      return cuda_status(e, "ray staging");
    ctx->inputs_pending = false;
  }
  if ((e = cudaMemcpyAsync(ctx->s_rays_in.p, rays, bytes, cudaMemcpyHostToDevice,
                           ctx->copy_stream)) != cudaSuccess ||
      (e = cudaEventRecord(ctx->ev_copy, ctx->copy_stream)) != cudaSuccess ||
      (e = cudaStreamWaitEvent(ctx->stream, ctx->ev_copy, 0)) != cudaSuccess)
    return cuda_status(e, "ray staging");
  *out = ctx->s_rays_in.as<srt_ray>();
  return SRT_OK;
}

// An optional array that the kernels can address directly: NULL, device
// memory, or page-locked host memory.  Sets ok = false for pageable memory.
static void *direct_view(const void *p, bool &ok) {
  if (!p) return nullptr;
  if (is_device_ptr(p)) return const_cast<void *>(p);
  void *m = mapped_host(p);
  if (!m) ok = false;
  return m;
}

SRT_API srt_status srt_trace_closest(srt_accel *a, const srt_ray *rays, size_t n,
                                     srt_hit *hits, const srt_trace_opts *opts) {
  if (!a || (!rays && n) || (!hits && n)) {
    set_error("NULL argument");
    return SRT_ERR_INVALID;
  }
  if (!a->built) {
    set_error("accel not built");
    return SRT_ERR_INVALID;
  }
  if (n == 0) return SRT_OK;
  srt_ctx *ctx = a->ctx;
  cudaSetDevice(ctx->device);
  srt_trace_opts o;
  memset(&o, 0, sizeof(o));
  if (opts) o = *opts;
  if (o.vertex_scalar && a->kind == SRT_TETRAHEDRA && !is_device_ptr(o.vertex_scalar)) {
    // vertex count is not stored; the scalar array is read only at hit
    // vertices, so a host array would have to be staged whole
    set_error("vertex_scalar must be device memory");
    return SRT_ERR_INVALID;
  }
  if (o.stats && !is_device_ptr(o.stats)) {
    set_error("stats must be device memory");
    return SRT_ERR_INVALID;
  }
  {
    // Page-locked host rays and hits: the kernels write the hits over the
    // host link while they traverse, and read small ray arrays the same way;
    // a large ray array is copied on the side stream as soon as the call is
    // made (prestage_rays), overlapping a build still running.  Either way
    // the transfers overlap GPU work instead of preceding and following it.
    // (a sorted trace reads the rays three times: those are staged instead)
    void *mr = mapped_host(rays), *mh = mapped_host(hits);
    if (mr && mh && !(o.flags & SRT_TRACE_SORT_RAYS)) {
      bool ok = true;
      void *pn = direct_view(o.prev_normals, ok), *sub = direct_view(o.subface, ok);
      void *scal = direct_view(o.scalar_out, ok), *norm = direct_view(o.normal_out, ok);
      void *isx = direct_view(o.isect, ok);
      if (ok) {
        if ((reinterpret_cast<uintptr_t>(mr) | reinterpret_cast<uintptr_t>(mh)) & 15u) {
          set_error("ray and hit arrays must be 16-byte aligned");
          return SRT_ERR_INVALID;
        }
        if (isx && !sub && a->kind == SRT_TETRAHEDRA) {
          // the shading pass needs each ray's entering face
          cudaError_t e = ctx->s_isect_sub.ensure(n * 4);
          if (e != cudaSuccess) return cuda_status(e, "entering faces");
          sub = ctx->s_isect_sub.p;
        }
        const srt_ray *trays = static_cast<const srt_ray *>(mr);
        srt_status s = prestage_rays(ctx, rays, n, &trays);
        if (s != SRT_OK) return s;
        s = launch_trace(
            a, trays, n, static_cast<srt_hit *>(mh),
            static_cast<const float *>(pn), static_cast<uint32_t *>(sub),
            a->kind == SRT_TETRAHEDRA ? o.vertex_scalar : nullptr, static_cast<float *>(scal),
            static_cast<float *>(norm), o.stats, o.flags, o.max_iter);
        if (s != SRT_OK) return s;
        if (isx) {
          s = launch_isect(a, trays, n, static_cast<const srt_hit *>(mh),
                           static_cast<uint32_t *>(sub), static_cast<srt_isect *>(isx));
          if (s != SRT_OK) return s;
        }
        if (trays != mr) {
          cudaError_t e = cudaEventRecord(ctx->ev_free, ctx->stream);
          if (e != cudaSuccess) return cuda_status(e, "ray staging event");
          ctx->ev_free_recorded = true;
        }
        return check_device_errors(ctx);
      }
    }
  }
  const void *drays = nullptr, *dpn = nullptr, *dvs = nullptr;
  srt_status s = device_view(ctx, rays, n * sizeof(srt_ray), ctx->s_stage_in, &drays);
  if (s != SRT_OK) return s;
  if (o.prev_normals) {
    s = device_view(ctx, o.prev_normals, n * 3 * sizeof(float), ctx->s_stage_aux, &dpn);
    if (s != SRT_OK) return s;
  }
  if (o.vertex_scalar && a->kind == SRT_TETRAHEDRA) {
    // vertex count is not stored; the scalar array is read only at hit
    // vertices, so a host array must be staged whole: require device memory
    if (!is_device_ptr(o.vertex_scalar)) {
      set_error("vertex_scalar must be device memory");
      return SRT_ERR_INVALID;
    }
    dvs = o.vertex_scalar;
  }
  // outputs: device pointers are written in place; page-locked host arrays
  // too, through their mapped addresses (the kernels' stores cross PCIe
  // while they run, instead of a copy after them); pageable ones via staging
  const bool hits_dev = is_device_ptr(hits);
  bool any_host = !hits_dev;
  srt_hit *dh = hits;
  cudaError_t e;
  if (!hits_dev) {
    dh = static_cast<srt_hit *>(mapped_ptr(hits));
    if (!dh) {
      if ((e = ctx->s_stage_out.ensure(n * sizeof(srt_hit))) != cudaSuccess)
        return cuda_status(e, "hit staging");
      dh = ctx->s_stage_out.as<srt_hit>();
    }
  }
  uint32_t *dsub = o.subface;
  float *dscal = o.scalar_out, *dnorm = o.normal_out;
  srt_isect *disx = o.isect;
  // a host output: its mapped address, else the staging buffer
  auto host_out = [&](auto *&d, DevBuf &stage, size_t bytes) -> cudaError_t {
    using P = std::remove_reference_t<decltype(d)>;
    if (!d || is_device_ptr(d)) return cudaSuccess;
    any_host = true;
    if (void *m = mapped_ptr(d)) {
      d = static_cast<P>(m);
      return cudaSuccess;
    }
    cudaError_t err = stage.ensure(bytes);
    if (err == cudaSuccess) d = stage.as<std::remove_pointer_t<P>>();
    return err;
  };
  if ((e = host_out(dsub, ctx->s_stage_sub, n * 4)) != cudaSuccess)
    return cuda_status(e, "staging");
  uint32_t *isub = dsub;  // entering faces for the shading pass
  if (disx && !isub && a->kind == SRT_TETRAHEDRA) {
    if ((e = ctx->s_isect_sub.ensure(n * 4)) != cudaSuccess)
      return cuda_status(e, "entering faces");
    isub = ctx->s_isect_sub.as<uint32_t>();
  }
  if ((e = host_out(disx, ctx->s_stage_isect, n * sizeof(srt_isect))) != cudaSuccess ||
      (e = host_out(dscal, ctx->s_stage_scal, n * 4)) != cudaSuccess ||
      (e = host_out(dnorm, ctx->s_stage_norm, n * 12)) != cudaSuccess)
    return cuda_status(e, "staging");
  if ((reinterpret_cast<uintptr_t>(drays) | reinterpret_cast<uintptr_t>(dh)) & 15u) {
    set_error("ray and hit arrays must be 16-byte aligned");
    return SRT_ERR_INVALID;
  }
  if (o.stats && !is_device_ptr(o.stats)) {
    set_error("stats must be device memory");
    return SRT_ERR_INVALID;
  }
  s = launch_trace(a, static_cast<const srt_ray *>(drays), n, dh,
                   static_cast<const float *>(dpn), isub, static_cast<const float *>(dvs),
                   dscal, dnorm, o.stats, o.flags, o.max_iter);
  if (s != SRT_OK) return s;
  if (disx) {
    s = launch_isect(a, static_cast<const srt_ray *>(drays), n, dh, isub, disx);
    if (s != SRT_OK) return s;
  }
  cudaStream_t st = ctx->stream;
  // staged outputs come back by copies (mapped ones were written in place)
  if (disx != o.isect && disx == ctx->s_stage_isect.as<srt_isect>())
    cudaMemcpyAsync(o.isect, disx, n * sizeof(srt_isect), cudaMemcpyDeviceToHost, st);
  if (dh == ctx->s_stage_out.as<srt_hit>() && dh != hits)
    cudaMemcpyAsync(hits, dh, n * sizeof(srt_hit), cudaMemcpyDeviceToHost, st);
  if (dsub != o.subface && dsub == ctx->s_stage_sub.as<uint32_t>())
    cudaMemcpyAsync(o.subface, dsub, n * 4, cudaMemcpyDeviceToHost, st);
  if (dscal != o.scalar_out && dscal == ctx->s_stage_scal.as<float>())
    cudaMemcpyAsync(o.scalar_out, dscal, n * 4, cudaMemcpyDeviceToHost, st);
  if (dnorm != o.normal_out && dnorm == ctx->s_stage_norm.as<float>())
    cudaMemcpyAsync(o.normal_out, dnorm, n * 12, cudaMemcpyDeviceToHost, st);
  if (any_host || !is_device_ptr(rays)) return check_device_errors(ctx);
  return cuda_status(cudaGetLastError(), "trace");
}

// ---------------------------------------------------------------- stages
SRT_API srt_status srt_stage_morton(srt_ctx *ctx, srt_kind kind, const float *vertices,
                                    size_t nvertices, const uint32_t *prims,
                                    const float *radius, float constant_radius, size_t n,
                                    uint32_t *codes, float scene_box[6]) {
  if (!ctx || !vertices || !codes || n == 0) return SRT_ERR_INVALID;
  cudaSetDevice(ctx->device);
  int per = kind == SRT_TRIANGLES ? 3 : (kind == SRT_TETRAHEDRA ? 4 : 0);
  if (per && !prims) return SRT_ERR_INVALID;
  DevBuf sv, sf, sr, sc, ss;
  const void *dv, *df = nullptr, *dr = nullptr;
  srt_status s = device_view(ctx, vertices, (per ? nvertices : n) * 12, sv, &dv);
  if (s != SRT_OK) return s;
  if (per && (s = device_view(ctx, prims, n * per * 4, sf, &df)) != SRT_OK) return s;
  if (radius && (s = device_view(ctx, radius, n * 4, sr, &dr)) != SRT_OK) return s;
  cudaError_t e;
  if ((e = sc.ensure(n * 4)) != cudaSuccess) return cuda_status(e, "stage");
  if ((e = ss.ensure(sizeof(SceneInfo))) != cudaSuccess) return cuda_status(e, "stage");
  s = stage_morton(ctx, kind, static_cast<const float *>(dv), static_cast<const uint32_t *>(df),
                   static_cast<const float *>(dr), constant_radius, n, sc.as<uint32_t>(),
                   ss.as<SceneInfo>());
  if (s != SRT_OK) return s;
  SceneInfo si;
  e = cudaMemcpyAsync(codes, sc.p, n * 4, cudaMemcpyDefault, ctx->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&si, ss.p, sizeof(si), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return cuda_status(e, "stage morton");
  if (scene_box)
    for (int k = 0; k < 3; k++) {
      scene_box[k] = si.lo[k];
      scene_box[3 + k] = si.hi[k];
    }
  return SRT_OK;
}

SRT_API srt_status srt_stage_sort_pairs(srt_ctx *ctx, uint32_t *codes, uint32_t *indices,
                                        size_t n) {
  if (!ctx || !codes || !indices) return SRT_ERR_INVALID;
  if (n == 0) return SRT_OK;
  cudaSetDevice(ctx->device);
  DevBuf k, v;
  cudaError_t e;
  if ((e = k.ensure(n * 4)) != cudaSuccess || (e = v.ensure(n * 4)) != cudaSuccess)
    return cuda_status(e, "stage sort");
  cudaMemcpyAsync(k.p, codes, n * 4, cudaMemcpyDefault, ctx->stream);
  cudaMemcpyAsync(v.p, indices, n * 4, cudaMemcpyDefault, ctx->stream);
  srt_status s = sort_pairs(ctx, k.as<uint32_t>(), v.as<uint32_t>(), n, false);
  if (s != SRT_OK) return s;
  cudaMemcpyAsync(codes, k.p, n * 4, cudaMemcpyDefault, ctx->stream);
  cudaMemcpyAsync(indices, v.p, n * 4, cudaMemcpyDefault, ctx->stream);
  return check_device_errors(ctx);
}

SRT_API srt_status srt_stage_karras(srt_ctx *ctx, const uint32_t *codes, size_t n,
                                    uint32_t *child, uint8_t *left_leaf,
                                    uint8_t *right_leaf) {
  if (!ctx || !codes || !child || !left_leaf || !right_leaf || n < 2 || n >= (1u << 30))
    return SRT_ERR_INVALID;
  cudaSetDevice(ctx->device);
  DevBuf dc, dch, dfl;
  cudaError_t e;
  if ((e = dc.ensure(n * 4)) != cudaSuccess || (e = dch.ensure(n * 4)) != cudaSuccess ||
      (e = dfl.ensure(n)) != cudaSuccess)
    return cuda_status(e, "stage karras");
  cudaMemcpyAsync(dc.p, codes, n * 4, cudaMemcpyDefault, ctx->stream);
  srt_status s = stage_karras(ctx, dc.as<uint32_t>(), n, dch.as<uint32_t>(), dfl.as<uint8_t>());
  if (s != SRT_OK) return s;
  std::vector<uint8_t> fl(n - 1);
  cudaMemcpyAsync(child, dch.p, (n - 1) * 4, cudaMemcpyDefault, ctx->stream);
  cudaMemcpyAsync(fl.data(), dfl.p, n - 1, cudaMemcpyDeviceToHost, ctx->stream);
  s = check_device_errors(ctx);
  if (s != SRT_OK) return s;
  for (size_t i = 0; i + 1 < n; i++) {
    left_leaf[i] = fl[i] & 1;
    right_leaf[i] = (fl[i] >> 1) & 1;
  }
  return SRT_OK;
}

}  // extern "C"
