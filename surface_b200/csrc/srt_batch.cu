// srt_batch.cu -- many triangle scenes built and traced in one call.
//
// This first version runs the plain build + trace per scene on the
// context stream (the per-scene loop the batched workload is measured
// against); the scene table is read once from device memory.
#include <vector>

#include "srt_internal.cuh"

struct srt_batch {
  srt_ctx *ctx = nullptr;
  std::vector<srt_accel *> accels;
};

using namespace srt;

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
  for (srt_accel *a : b->accels) srt_accel_destroy(a);
  delete b;
  return SRT_OK;
}

SRT_API srt_status srt_batch_build_trace(srt_batch *b, int32_t nscenes,
                                         const float *vertices, const uint32_t *faces,
                                         const uint64_t *face_offsets,
                                         const srt_ray *rays, const uint64_t *ray_offsets,
                                         srt_hit *hits) {
  if (!b || nscenes <= 0 || !vertices || !faces || !face_offsets || !rays ||
      !ray_offsets || !hits)
    return SRT_ERR_INVALID;
  srt_ctx *ctx = b->ctx;
  cudaSetDevice(ctx->device);
  std::vector<uint64_t> fo(nscenes + 1), ro(nscenes + 1);
  cudaMemcpyAsync(fo.data(), face_offsets, fo.size() * 8, cudaMemcpyDefault, ctx->stream);
  cudaMemcpyAsync(ro.data(), ray_offsets, ro.size() * 8, cudaMemcpyDefault, ctx->stream);
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return cuda_status(e, "batch offsets");
  while ((int)b->accels.size() < nscenes) {
    srt_accel *a = nullptr;
    srt_status s = srt_accel_create(ctx, SRT_TRIANGLES, &a);
    if (s != SRT_OK) return s;
    b->accels.push_back(a);
  }
  for (int i = 0; i < nscenes; i++) {
    srt_accel *a = b->accels[i];
    // the vertex array is shared; each scene indexes into it
    srt_status s = srt_accel_build_triangles(a, vertices, 1, faces + 3 * fo[i],
                                             (size_t)(fo[i + 1] - fo[i]));
    if (s != SRT_OK) return s;
    s = srt_trace_closest(a, rays + ro[i], (size_t)(ro[i + 1] - ro[i]), hits + ro[i], nullptr);
    if (s != SRT_OK) return s;
  }
  return SRT_OK;
}

}  // extern "C"
