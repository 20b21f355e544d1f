// srt_raysort.cu -- coherent ray order for traversal (SRT_TRACE_SORT_RAYS).
//
// Rays that start close together and point the same way visit the same
// nodes; a warp of such rays diverges less.  The order is a Morton curve over
// the six ray coordinates (origin and direction), each quantized within the
// rays' own bounding range, with the 30 key bits shared among the
// coordinates that vary (an orthographic view orders by origin, a pinhole
// view by direction, bounce rays by both).  A stable sort of (key, ray
// index) gives the order; traversal reads ray order[k] in thread k and writes
// its hit at the ray's own index, so results do not depend on the order.
#include <climits>

#include "srt_internal.cuh"

namespace srt {
namespace {

__device__ __forceinline__ int ord_f(float f) {  // order-preserving float -> int
  const int i = __float_as_int(f);
  return i >= 0 ? i : i ^ 0x7fffffff;
}
__device__ __forceinline__ float ord_i(int i) { return __int_as_float(i >= 0 ? i : i ^ 0x7fffffff); }

// box[0..5]: min of o.xyz, d.xyz; box[6..11]: max
__global__ void ray_box_init_kernel(int *__restrict__ box) {
  const int k = threadIdx.x;
  if (k < 12) box[k] = k < 6 ? INT_MAX : INT_MIN;
}

__global__ void ray_box_kernel(const srt_ray *__restrict__ rays, size_t n, int *__restrict__ box) {
  float lo[6], hi[6];
#pragma unroll
  for (int a = 0; a < 6; a++) {
    lo[a] = FLT_MAX;
    hi[a] = -FLT_MAX;
  }
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const float4 *r4 = reinterpret_cast<const float4 *>(rays + i);
    const float4 a = __ldg(r4), b = __ldg(r4 + 1);
    const float x[6] = {a.x, a.y, a.z, b.x, b.y, b.z};
#pragma unroll
    for (int k = 0; k < 6; k++) {
      lo[k] = fminf(lo[k], x[k]);  // NaN coordinates are ignored
      hi[k] = fmaxf(hi[k], x[k]);
    }
  }
#pragma unroll
  for (int k = 0; k < 6; k++) {
    for (int o = 16; o > 0; o >>= 1) {
      lo[k] = fminf(lo[k], __shfl_down_sync(0xffffffffu, lo[k], o));
      hi[k] = fmaxf(hi[k], __shfl_down_sync(0xffffffffu, hi[k], o));
    }
  }
  if ((threadIdx.x & 31) == 0) {
#pragma unroll
    for (int k = 0; k < 6; k++) {
      atomicMin(&box[k], ord_f(lo[k]));
      atomicMax(&box[6 + k], ord_f(hi[k]));
    }
  }
}

// The rays' quantization: per coordinate its low end and scale, the
// coordinates that vary (dims[0..nd)) and the bits each gets (30 / nd).
struct RayQuant {
  float lo[6], scale[6];
  int dims[6], nd, bits;
  __device__ __forceinline__ explicit RayQuant(const int *__restrict__ box) {
    nd = 0;
#pragma unroll
    for (int k = 0; k < 6; k++) {
      lo[k] = ord_i(box[k]);
      const float ext = ord_i(box[6 + k]) - lo[k];
      scale[k] = ext > 0.0f ? 1.0f / ext : 0.0f;
      if (ext > 0.0f) dims[nd++] = k;
    }
    bits = nd ? 30 / nd : 0;  // bits per varying coordinate (<= 30 total)
  }
  // Morton code (up to 30 bits) of ray i
  __device__ __forceinline__ uint32_t key(const srt_ray *__restrict__ rays, size_t i) const {
    const float qmax = (float)((1u << bits) - 1u);
    const float4 *r4 = reinterpret_cast<const float4 *>(rays + i);
    const float4 a = __ldg(r4), b = __ldg(r4 + 1);
    const float x[6] = {a.x, a.y, a.z, b.x, b.y, b.z};
    uint32_t q[6];
    for (int c = 0; c < nd; c++) {
      const int k = dims[c];
      // fmaxf(NaN, 0) = 0: NaN coordinates land in cell 0
      const float v = fminf(fmaxf((x[k] - lo[k]) * scale[k] * (qmax + 1.0f), 0.0f), qmax);
      q[c] = (uint32_t)v;
    }
    uint32_t key = 0;
    for (int bit = bits - 1; bit >= 0; bit--)
      for (int c = 0; c < nd; c++) key = (key << 1) | ((q[c] >> bit) & 1u);
    return key;
  }
};

__global__ void ray_key_kernel(const srt_ray *__restrict__ rays, size_t n,
                               const int *__restrict__ box, uint32_t *__restrict__ keys) {
  const RayQuant Q(box);
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    keys[i] = Q.key(rays, i);
}

// Batch keys: the ray's scene above the top mbits of its Morton code, so
// that the order keeps every scene's rays together.
__global__ void batch_ray_key_kernel(const srt_ray *__restrict__ rays, size_t n,
                                     const int *__restrict__ box,
                                     const uint32_t *__restrict__ roff, int nseg, int mbits,
                                     uint32_t *__restrict__ keys) {
  const RayQuant Q(box);
  const int used = Q.nd * Q.bits;  // significant bits of a Morton code
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const uint32_t m = Q.key(rays, i);
    const uint32_t top = used > mbits ? m >> (used - mbits) : m << (mbits - used);
    keys[i] = ((uint32_t)seg_of(roff, nseg, (uint32_t)i) << mbits) | top;
  }
}

}  // namespace

srt_status batch_ray_order(srt_ctx *ctx, const srt_ray *rays, size_t n, const uint32_t *roff,
                           int nseg, int mbits, uint32_t *keys, uint32_t *order) {
  int segbits = 0;
  while ((1 << segbits) < nseg) segbits++;
  if (mbits < 1 || segbits + mbits > 30) {
    set_error("ray order: scene and Morton bits exceed 30");
    return SRT_ERR_INVALID;
  }
  int *box = reinterpret_cast<int *>(keys + n);  // 12 ints after the keys
  cudaStream_t st = ctx->stream;
  const int grid = ctx->num_sms * 4;
  ray_box_init_kernel<<<1, 32, 0, st>>>(box);
  ray_box_kernel<<<grid, 256, 0, st>>>(rays, n, box);
  batch_ray_key_kernel<<<grid, 256, 0, st>>>(rays, n, box, roff, nseg, mbits, keys);
  ctx->launches += 3;
  srt_status s = cuda_status(cudaGetLastError(), "batch ray keys");
  if (s != SRT_OK) return s;
  return sort_pairs(ctx, keys, order, n, true, segbits + mbits);
}

srt_status ray_order(srt_ctx *ctx, const srt_ray *rays, size_t n, const uint32_t **order) {
  cudaError_t e;
  if ((e = ctx->s_rkey.ensure(n * 4 + 64)) != cudaSuccess ||
      (e = ctx->s_rorder.ensure(n * 4)) != cudaSuccess)
    return cuda_status(e, "ray order scratch");
  uint32_t *keys = ctx->s_rkey.as<uint32_t>();
  int *box = reinterpret_cast<int *>(keys + n);  // 12 ints after the keys
  uint32_t *ord = ctx->s_rorder.as<uint32_t>();
  cudaStream_t st = ctx->stream;
  const int grid = ctx->num_sms * 4;
  ray_box_init_kernel<<<1, 32, 0, st>>>(box);
  ray_box_kernel<<<grid, 256, 0, st>>>(rays, n, box);
  ray_key_kernel<<<grid, 256, 0, st>>>(rays, n, box, keys);
  ctx->launches += 3;
  srt_status s = cuda_status(cudaGetLastError(), "ray keys");
  if (s != SRT_OK) return s;
  if ((s = sort_pairs(ctx, keys, ord, n, true, 30)) != SRT_OK) return s;
  *order = ord;
  return SRT_OK;
}

}  // namespace srt
