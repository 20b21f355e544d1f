// srt_spawn.cu -- secondary rays from closest hits (the particle workload's
// one jittered bounce per hit).
//
// In the reference a fragment shader makes the secondary ray and calls back
// trace() with the previous hit's primitive, distance and normal attached
// (gles/gles_glsl_runtime.cc:119-136: prev_prim_id, prev_hit_t,
// prev_hit_normal), which the sphere test uses for its self-hit rule
// (render/render_accel_particle.cc:2478-2489).  Here every hit ray spawns one
// ray at its hit point with a uniformly distributed direction on the
// hemisphere about the hit normal; rays that missed spawn nothing.  Output
// order is the input order of the hit rays (a prefix sum of the hit flags),
// so the result does not depend on scheduling.
#include "srt_internal.cuh"

namespace srt {
namespace {

// SplitMix64 output function (Steele, Lea and Flood, "Fast splittable
// pseudorandom number generators", OOPSLA 2014): a counter-based stream,
// one 64-bit draw per ray.
__device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

__global__ void hit_flags_kernel(const srt_hit *__restrict__ hits, size_t n,
                                 uint32_t *__restrict__ flags) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    flags[i] = hits[i].prim != kNone ? 1u : 0u;
}

__global__ void spawn_kernel(const srt_ray *__restrict__ rays, const srt_hit *__restrict__ hits,
                             const float *__restrict__ normals, size_t n, uint64_t seed,
                             const uint32_t *__restrict__ flags,
                             const uint32_t *__restrict__ slots, srt_ray *__restrict__ out,
                             float *__restrict__ out_normals) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    if (!flags[i]) continue;
    const srt_ray r = rays[i];
    const srt_hit h = hits[i];
    float nx = normals[3 * i], ny = normals[3 * i + 1], nz = normals[3 * i + 2];
    const float inv = 1.0f / sqrtf(nx * nx + ny * ny + nz * nz);
    nx *= inv;
    ny *= inv;
    nz *= inv;
    // two 24-bit uniforms in [0, 1)
    const uint64_t z = mix64(seed + 0x9e3779b97f4a7c15ull * (uint64_t)(i + 1));
    const float u1 = (float)(uint32_t)(z >> 40) * (1.0f / 16777216.0f);
    const float u2 = (float)(uint32_t)((z >> 16) & 0xffffffu) * (1.0f / 16777216.0f);
    // uniform hemisphere: cos(theta) uniform in [0, 1), phi uniform
    const float ct = u1, st = sqrtf(fmaxf(0.0f, 1.0f - ct * ct));
    float sp, cp;
    sincospif(2.0f * u2, &sp, &cp);
    const float lx = st * cp, ly = st * sp;
    // orthonormal basis about n (Duff et al., "Building an Orthonormal
    // Basis, Revisited", JCGT 2017)
    const float sg = copysignf(1.0f, nz);
    const float a = -1.0f / (sg + nz);
    const float b = nx * ny * a;
    const float b1x = 1.0f + sg * nx * nx * a, b1y = sg * b, b1z = -sg * nx;
    const float b2x = b, b2y = sg + ny * ny * a, b2z = -ny;
    srt_ray o;
    for (int k = 0; k < 3; k++) o.org[k] = r.org[k] + h.t * r.dir[k];
    o.dir[0] = lx * b1x + ly * b2x + ct * nx;
    o.dir[1] = lx * b1y + ly * b2y + ct * ny;
    o.dir[2] = lx * b1z + ly * b2z + ct * nz;
    o.prev_prim = h.prim;
    o.prev_t = h.t;
    const uint32_t k = slots[i];
    out[k] = o;
    out_normals[3 * (size_t)k] = nx;
    out_normals[3 * (size_t)k + 1] = ny;
    out_normals[3 * (size_t)k + 2] = nz;
  }
}

}  // namespace
}  // namespace srt

using namespace srt;

extern "C" SRT_API srt_status srt_spawn_secondary(srt_ctx *ctx, const srt_ray *rays,
                                                  const srt_hit *hits, const float *normals,
                                                  size_t n, uint64_t seed, srt_ray *out,
                                                  float *out_normals, uint32_t *count) {
  if (!ctx || !count || (n && (!rays || !hits || !normals || !out || !out_normals))) {
    set_error("NULL argument");
    return SRT_ERR_INVALID;
  }
  *count = 0;
  if (n == 0) return SRT_OK;
  if (n >= 0xffffffffull) {
    set_error("at most 2^32-2 rays per call");
    return SRT_ERR_INVALID;
  }
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_status(e, "set device");
  if (!is_device_ptr(rays) || !is_device_ptr(hits) || !is_device_ptr(normals) ||
      !is_device_ptr(out) || !is_device_ptr(out_normals)) {
    set_error("srt_spawn_secondary: all arrays must be device memory");
    return SRT_ERR_INVALID;
  }
  if ((e = ctx->s_spawn.ensure(2 * n * sizeof(uint32_t) + 16)) != cudaSuccess)
    return cuda_status(e, "spawn scratch");
  uint32_t *flags = ctx->s_spawn.as<uint32_t>();
  uint32_t *slots = flags + n;
  cudaStream_t st = ctx->stream;
  const int grid = ctx->num_sms * 8;
  hit_flags_kernel<<<grid, 256, 0, st>>>(hits, n, flags);
  ctx->launches++;
  srt_status s = cuda_status(cudaGetLastError(), "spawn flags");
  if (s != SRT_OK) return s;
  if ((s = scan_exclusive(ctx, flags, slots, n)) != SRT_OK) return s;
  spawn_kernel<<<grid, 256, 0, st>>>(rays, hits, normals, n, seed, flags, slots, out,
                                     out_normals);
  ctx->launches++;
  if ((s = cuda_status(cudaGetLastError(), "spawn")) != SRT_OK) return s;
  uint32_t last[2];
  e = cudaMemcpyAsync(&last[0], slots + n - 1, 4, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&last[1], flags + n - 1, 4, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_status(e, "spawn count");
  *count = last[0] + last[1];
  return SRT_OK;
}
