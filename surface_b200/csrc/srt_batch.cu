// srt_batch.cu -- many triangle scenes built and traced as one forest.
//
// Every build stage runs once over all scenes (srt_build.cu, build_batch)
// and all rays are traced by one persistent kernel (srt_trace.cu,
// launch_trace_batch).  The first call runs eagerly and autotunes the
// traversal (timed with CUDA events, one axis at a time from the default
// point): block size x rays per grab, then the traversal stack depth (24, 32
// or 48 entries; a depth the trees overflow is dropped), then the ray order
// (array order, or sorted within each scene by the top 12 or 22 bits of a
// Morton code over origin and direction, the sort timed with the trace).
// The second identical call captures the whole sequence in a CUDA graph,
// later identical calls replay it with one graph launch.
#include <cstring>
#include <vector>

#include "srt_internal.cuh"

using namespace srt;

struct srt_batch {
  srt_ctx *ctx = nullptr;
  BatchTree bt;
  std::vector<uint64_t> fo, ro;
  const float *verts = nullptr;
  const uint32_t *faces = nullptr;
  const srt_ray *rays = nullptr;
  srt_hit *hits = nullptr;
  int block = 128, R = 1, depth = 32, sort_bits = 0;
  DevBuf rkey, rorder;  // batch ray order (sort_bits > 0)
  bool tuned = false, pinned = false;  // pinned: set by srt_batch_set_tuning
  int same_calls = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  uint64_t kernels_per_call = 0;
  uint64_t epoch = 0;  // g_buffer_epoch when the graph was captured

  void drop_graph() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec = nullptr;
    graph = nullptr;
  }
};

namespace {

// Upload the per-scene offsets as uint32 (global primitive, internal node
// and ray offsets).
srt_status upload_offsets(srt_batch *b) {
  const int ns = (int)b->fo.size() - 1;
  std::vector<uint32_t> f(ns + 1), in(ns + 1), r(ns + 1);
  for (int s = 0; s <= ns; s++) {
    f[s] = (uint32_t)b->fo[s];
    in[s] = (uint32_t)(b->fo[s] - (uint64_t)s);
    r[s] = (uint32_t)b->ro[s];
  }
  cudaError_t e;
  if ((e = b->bt.foff.ensure((ns + 1) * 4)) != cudaSuccess ||
      (e = b->bt.ioff.ensure((ns + 1) * 4)) != cudaSuccess ||
      (e = b->bt.roff.ensure((ns + 1) * 4)) != cudaSuccess)
    return cuda_status(e, "batch offsets");
  cudaStream_t st = b->ctx->stream;
  e = cudaMemcpyAsync(b->bt.foff.p, f.data(), (ns + 1) * 4, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(b->bt.ioff.p, in.data(), (ns + 1) * 4, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(b->bt.roff.p, r.data(), (ns + 1) * 4, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_status(e, "batch offsets");
  b->bt.nseg = ns;
  b->bt.nprims = b->fo[ns];
  b->bt.nrays = b->ro[ns];
  return SRT_OK;
}

// The traversal as tuned: the batch ray order (when sorting) and the trace.
srt_status trace_tuned(srt_batch *b, int block, int R, int depth, int sort_bits) {
  const uint32_t *order = nullptr;
  if (sort_bits > 0) {
    const size_t n = b->bt.nrays;
    cudaError_t e;
    if ((e = b->rkey.ensure(n * 4 + 64)) != cudaSuccess ||
        (e = b->rorder.ensure(n * 4)) != cudaSuccess)
      return cuda_status(e, "batch ray order");
    srt_status s = batch_ray_order(b->ctx, b->rays, n, b->bt.roff.as<uint32_t>(), b->bt.nseg,
                                   sort_bits, b->rkey.as<uint32_t>(), b->rorder.as<uint32_t>());
    if (s != SRT_OK) return s;
    order = b->rorder.as<uint32_t>();
  }
  return launch_trace_batch(b->ctx, b->bt, b->rays, b->hits, block, R, nullptr, depth, order);
}

srt_status build_and_trace(srt_batch *b, const uint32_t *h_foff) {
  srt_status s = build_batch(b->ctx, b->bt, b->verts, b->faces, h_foff, b->bt.nseg);
  if (s != SRT_OK) return s;
  return trace_tuned(b, b->block, b->R, b->depth, b->sort_bits);
}

// Reads and clears the kernels' limit word: whether a candidate's walks
// ran out of stack (their hits are then incomplete; the tuned trace that
// follows recomputes them all).
srt_status take_limit_flag(srt_ctx *ctx, bool &hit) {
  uint32_t h = 0;
  cudaError_t e = cudaMemcpyAsync(&h, ctx->d_err, 4, cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e == cudaSuccess && h) e = cudaMemsetAsync(ctx->d_err, 0, 4, ctx->stream);
  if (e != cudaSuccess) return cuda_status(e, "autotune limit flag");
  hit = h != 0;
  return SRT_OK;
}

// Time the traversal over the tuning axes, one at a time from the default
// point (block 128, one grab of 32 rays, depth 32, array order), and keep
// the fastest point.
srt_status autotune(srt_batch *b) {
  static const int blocks[] = {64, 128, 256};
  static const int Rs[] = {1, 2, 4};
  static const int depths[] = {24, 32, 48};
  static const int sorts[] = {0, 12, 22};
  srt_ctx *ctx = b->ctx;
  cudaStream_t st = ctx->stream;
  bool pending = false;  // a limit raised before tuning (the build's) stays for the caller
  {
    uint32_t h = 0;
    cudaError_t e = cudaMemcpyAsync(&h, ctx->d_err, 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_status(e, "autotune");
    pending = h != 0;
  }
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  // ms of one candidate (second of two runs: the first warms caches); ok
  // false when its walks overflowed the stack
  auto time_point = [&](int blk, int r, int dep, int sb, float &ms, bool &ok) -> srt_status {
    ms = 0.0f;
    ok = true;
    for (int rep = 0; rep < 2; rep++) {
      cudaEventRecord(e0, st);
      srt_status s = trace_tuned(b, blk, r, dep, sb);
      cudaEventRecord(e1, st);
      if (s != SRT_OK) return s;
      cudaError_t e = cudaEventSynchronize(e1);
      if (e != cudaSuccess) return cuda_status(e, "autotune");
      if (rep > 0) cudaEventElapsedTime(&ms, e0, e1);
    }
    if (!pending) {
      bool hit = false;
      srt_status s = take_limit_flag(ctx, hit);
      if (s != SRT_OK) return s;
      ok = !hit;
    }
    return SRT_OK;
  };
  int bb = 128, br = 1, bd = 32, bs = 0;
  float best = 1e30f;
  srt_status s = SRT_OK;
  for (int blk : blocks)
    for (int r : Rs) {
      float ms;
      bool ok;
      if ((s = time_point(blk, r, bd, bs, ms, ok)) != SRT_OK) break;
      if (ok && ms < best) best = ms, bb = blk, br = r;
    }
  for (int dep : depths) {
    if (s != SRT_OK || dep == bd || (pending && dep < 32)) continue;
    float ms;
    bool ok;
    if ((s = time_point(bb, br, dep, bs, ms, ok)) != SRT_OK) break;
    if (ok && ms < best) best = ms, bd = dep;
  }
  for (int sb : sorts) {
    if (s != SRT_OK || sb == bs) continue;
    float ms;
    bool ok;
    if ((s = time_point(bb, br, bd, sb, ms, ok)) != SRT_OK) break;
    if (ok && ms < best) best = ms, bs = sb;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (s != SRT_OK) return s;
  b->block = bb;
  b->R = br;
  b->depth = bd;
  b->sort_bits = bs;
  b->tuned = true;
  return SRT_OK;
}

}  // namespace

extern "C" {

SRT_API srt_status srt_batch_create(srt_ctx *ctx, srt_batch **out) {
  if (!ctx || !out) return SRT_ERR_INVALID;
  srt_batch *b = new srt_batch();
  b->ctx = ctx;
  *out = b;
  return SRT_OK;
}

SRT_API srt_status srt_batch_destroy(srt_batch *b) {
  if (!b) return SRT_OK;
  cudaSetDevice(b->ctx->device);
  cudaStreamSynchronize(b->ctx->stream);
  b->drop_graph();
  delete b;
  return SRT_OK;
}

SRT_API srt_status srt_batch_config(srt_batch *b, int32_t *block, int32_t *rays_per_thread,
                                    int32_t *graph_captured, uint64_t *kernels_per_call) {
  if (!b) return SRT_ERR_INVALID;
  if (block) *block = b->block;
  if (rays_per_thread) *rays_per_thread = b->R;
  if (graph_captured) *graph_captured = b->exec ? 1 : 0;
  if (kernels_per_call) *kernels_per_call = b->kernels_per_call;
  return SRT_OK;
}

SRT_API srt_status srt_batch_tuning(srt_batch *b, int32_t *block, int32_t *rays_per_grab,
                                    int32_t *stack_depth, int32_t *sort_bits) {
  if (!b) return SRT_ERR_INVALID;
  if (block) *block = b->block;
  if (rays_per_grab) *rays_per_grab = b->R;
  if (stack_depth) *stack_depth = b->depth;
  if (sort_bits) *sort_bits = b->sort_bits;
  return SRT_OK;
}

SRT_API srt_status srt_batch_set_tuning(srt_batch *b, int32_t block, int32_t rays_per_grab,
                                        int32_t stack_depth, int32_t sort_bits) {
  if (!b || (block != 64 && block != 128 && block != 256) || rays_per_grab < 1 ||
      rays_per_grab > 8 || (stack_depth != 24 && stack_depth != 32 && stack_depth != 48) ||
      (sort_bits != 0 && sort_bits != 12 && sort_bits != 22)) {
    set_error("tuning: block 64/128/256, 1..8 grabs, depth 24/32/48, sort bits 0/12/22");
    return SRT_ERR_INVALID;
  }
  cudaSetDevice(b->ctx->device);
  cudaStreamSynchronize(b->ctx->stream);
  b->drop_graph();
  b->same_calls = 0;
  b->block = block;
  b->R = rays_per_grab;
  b->depth = stack_depth;
  b->sort_bits = sort_bits;
  b->tuned = true;
  b->pinned = true;
  return SRT_OK;
}

SRT_API srt_status srt_batch_build_trace(srt_batch *b, int32_t nscenes, const float *vertices,
                                         const uint32_t *faces, const uint64_t *face_offsets,
                                         const srt_ray *rays, const uint64_t *ray_offsets,
                                         srt_hit *hits) {
  if (!b || nscenes <= 0 || nscenes > 256 || !vertices || !faces || !face_offsets || !rays ||
      !ray_offsets || !hits) {
    set_error("invalid batch arguments");
    return SRT_ERR_INVALID;
  }
  srt_ctx *ctx = b->ctx;
  cudaSetDevice(ctx->device);
  if (face_offsets[0] != 0 || ray_offsets[0] != 0) {
    set_error("offsets must start at 0");
    return SRT_ERR_INVALID;
  }
  for (int s = 0; s < nscenes; s++) {
    if (face_offsets[s + 1] < face_offsets[s] + 2 || ray_offsets[s + 1] < ray_offsets[s]) {
      set_error("every scene needs at least 2 faces; offsets must not decrease");
      return SRT_ERR_INVALID;
    }
  }
  if (face_offsets[nscenes] >= (1ull << 30) || ray_offsets[nscenes] >= (1ull << 31)) {
    set_error("batch too large");
    return SRT_ERR_INVALID;
  }
  if (!is_device_ptr(vertices) || !is_device_ptr(faces) || !is_device_ptr(rays) ||
      !is_device_ptr(hits)) {
    set_error("batch arrays must be device memory");
    return SRT_ERR_INVALID;
  }
  if ((reinterpret_cast<uintptr_t>(rays) | reinterpret_cast<uintptr_t>(hits)) & 15u) {
    set_error("ray and hit arrays must be 16-byte aligned");
    return SRT_ERR_INVALID;
  }
  std::vector<uint64_t> fo(face_offsets, face_offsets + nscenes + 1);
  std::vector<uint64_t> ro(ray_offsets, ray_offsets + nscenes + 1);
  const bool same = fo == b->fo && ro == b->ro && vertices == b->verts && faces == b->faces &&
                    rays == b->rays && hits == b->hits;
  std::vector<uint32_t> h_foff(nscenes + 1);
  for (int s = 0; s <= nscenes; s++) h_foff[s] = (uint32_t)fo[s];
  srt_status s;
  if (!same) {
    const bool reshaped = fo != b->fo || ro != b->ro;
    b->drop_graph();
    b->fo = fo;
    b->ro = ro;
    b->verts = vertices;
    b->faces = faces;
    b->rays = rays;
    b->hits = hits;
    b->same_calls = 0;
    if (reshaped) {  // new scene sizes: new offsets, tune again (unless pinned)
      b->tuned = b->pinned;
      if ((s = upload_offsets(b)) != SRT_OK) return s;
    }
  }
  // graph replay, unless a scratch buffer it points into has been freed since
  if (b->exec && b->epoch != g_buffer_epoch.load(std::memory_order_relaxed)) {
    b->drop_graph();
    b->same_calls = 1;
  }
  if (b->exec) {
    cudaError_t e = cudaGraphLaunch(b->exec, ctx->stream);
    if (e != cudaSuccess) return cuda_status(e, "batch graph launch");
    ctx->launches += b->kernels_per_call;
    return SRT_OK;
  }
  // eager run (allocates, autotunes on the first call)
  const uint64_t l0 = ctx->launches;
  if ((s = build_batch(ctx, b->bt, vertices, faces, h_foff.data(), nscenes)) != SRT_OK) return s;
  const uint64_t lb = ctx->launches;
  if (!b->tuned && (s = autotune(b)) != SRT_OK) return s;
  const uint64_t lt = ctx->launches;
  if ((s = trace_tuned(b, b->block, b->R, b->depth, b->sort_bits)) != SRT_OK) return s;
  b->kernels_per_call = (lb - l0) + (ctx->launches - lt);
  b->same_calls++;
  // capture on the second identical call (the legacy and per-thread default
  // streams cannot be captured; those stay eager)
  if (b->same_calls >= 2 && ctx->stream != nullptr && ctx->stream != cudaStreamLegacy &&
      ctx->stream != cudaStreamPerThread) {
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_status(e, "batch sync");
    const uint64_t c0 = ctx->launches;
    e = cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return cuda_status(e, "batch capture");
    srt_status cs = build_and_trace(b, h_foff.data());
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(ctx->stream, &g);
    if (cs != SRT_OK || e != cudaSuccess || !g) {
      if (g) cudaGraphDestroy(g);
      cudaGetLastError();
      ctx->launches = c0;
      return SRT_OK;  // stay eager; results of this call are complete
    }
    b->kernels_per_call = ctx->launches - c0;
    ctx->launches = c0;
    b->graph = g;
    b->epoch = g_buffer_epoch.load(std::memory_order_relaxed);
    if (cudaGraphInstantiate(&b->exec, g, 0) != cudaSuccess) {
      cudaGetLastError();
      b->drop_graph();
    }
  }
  return cuda_status(cudaGetLastError(), "batch");
}

}  // extern "C"
