// srt_camera.cu -- eye rays and the framebuffer write of one frame, as
// RaytraceEngine::OnData does them on the CPU (gles/gles_raytrace_engine.cc:
// 547-879) for one sample per pixel.
//
//   frame      Camera::buildFrame (render/render_camera.cc:17-63): float
//              arithmetic, real3::normalize's reciprocal length in double
//              (render/render_common.h:69-83); computed once on the host.
//   pixels     loop pixels (x, y) of the render region in steps of `step`;
//              ViewportConversion (gles/gles_raytrace_engine.cc:530-544)
//              maps each to (px, py), and off-screen ones are skipped.
//              Conversion is monotone per axis, so the kept pixels are a
//              rectangle of the loop grid, found on the host.
//   rays       corner + (px + step/2) u + (py - step/2 + 1) v: the origin of
//              an orthographic ray, the end of a perspective ray from the
//              eye (:770-795); directions normalized as real3::normalize.
//   write      a hit fills the step x step block at (x + u, height - y - 1 +
//              v) with its colour (RGBA8 by clamp(), :50-58, or RGBA32F) and
//              depth t (:840-877); misses leave the framebuffer untouched.
//              Blocks whose rows fall outside the framebuffer are skipped
//              (the reference would write outside it).
#include <climits>
#include <cmath>

#include "srt_internal.cuh"

namespace srt {
namespace {

struct Frame {
  float corner[3], u[3], v[3], look[3], eye[3];
  int ortho, W, H, vx, vy, vw, vh, step;
  int xs, ys;  // first kept loop pixel
  int nx, ny;  // kept loop pixels per row / column
};

// real3::normalize (render/render_common.h:69-83); host and device.
__host__ __device__ inline void norm3(float v[3]) {
  const double l2 = (double)(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  double l = 0.0;
  if (fabs(l2) > 1.0e-30) l = 1.0 / sqrt(l2);
  for (int k = 0; k < 3; k++) v[k] = (float)((double)v[k] * l);
}

inline void cross3(const float a[3], const float b[3], float o[3]) {
  o[0] = a[1] * b[2] - a[2] * b[1];
  o[1] = a[2] * b[0] - a[0] * b[2];
  o[2] = a[0] * b[1] - a[1] * b[0];
}

// ViewportConversion of loop coordinate x along one axis: axis 0 subtracts
// the viewport offset (the camera's x is flipped), axis 1 adds it.
__host__ __device__ inline int viewport_px(int x, int axis, int size, int off, int vsize) {
  const float inv = 1.0f / (float)size;
  const float x01 = ((float)x + 0.5f) * inv;
  const float nd = 2.0f * (x01 - 0.5f);
  const float w = (nd + 1.0f) * (0.5f * (float)vsize);
  return axis == 0 ? (int)(w - (float)off) : (int)(w + (float)off);
}

void build_frame(const srt_camera &c, Frame &f) {
  float look[3], u[3], v[3];
  for (int k = 0; k < 3; k++) look[k] = c.lookat[k] - c.eye[k];
  cross3(look, c.up, u);
  norm3(u);
  cross3(look, u, v);
  norm3(v);
  norm3(look);
  const int W = c.width, H = c.height;
  if (c.ortho) {
    for (int k = 0; k < 3; k++) {
      u[k] = u[k] / (float)W;
      v[k] = v[k] / (float)H;
    }
    for (int k = 0; k < 3; k++) f.corner[k] = -(u[k] * (float)W + v[k] * (float)H);
    for (int k = 0; k < 3; k++) {
      u[k] = 2.0f * u[k];
      v[k] = 2.0f * v[k];
    }
  } else {
    const float flen = (float)(0.5f * (float)H /
                               std::tan(0.5 * ((double)c.fov * 3.14159265358979323846 / 180.0)));
    for (int k = 0; k < 3; k++) look[k] = look[k] * flen + c.eye[k];
    for (int k = 0; k < 3; k++) f.corner[k] = look[k] - (u[k] * (float)W + v[k] * (float)H) * 0.5f;
  }
  for (int k = 0; k < 3; k++) {
    f.u[k] = u[k];
    f.v[k] = v[k];
    f.eye[k] = c.eye[k];
  }
  cross3(f.u, f.v, f.look);  // OnData's look = normalize(cross(u, v))
  norm3(f.look);
  f.ortho = c.ortho != 0;
  f.W = W;
  f.H = H;
  f.vx = c.viewport[0];
  f.vy = c.viewport[1];
  f.vw = c.viewport[2];
  f.vh = c.viewport[3];
  f.step = c.step;
}

// Kept loop pixels along one axis: [first, first + count) in loop steps.
void kept_range(int lo, int hi, int step, int axis, int size, int off, int vsize, int &first,
                int &count) {
  first = 0;
  count = 0;
  int i = 0;
  bool started = false;
  for (int x = lo; x < hi; x += step, i++) {
    const int p = viewport_px(x, axis, size, off, vsize);
    const bool ok = p >= 0 && p < size;
    if (ok && !started) {
      first = i;
      started = true;
    }
    if (ok) count++;
    else if (started) break;  // monotone: nothing further is kept
  }
}

__global__ void camera_rays_kernel(const Frame f, int x0, int y0, srt_ray *__restrict__ rays,
                                   uint32_t *__restrict__ pixel) {
  const size_t n = (size_t)f.nx * f.ny;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
       k += (size_t)gridDim.x * blockDim.x) {
    const int ix = (int)(k % f.nx), iy = (int)(k / f.nx);
    const int x = x0 + (f.xs + ix) * f.step, y = y0 + (f.ys + iy) * f.step;
    const int px = viewport_px(x, 0, f.W, f.vx, f.vw);
    const int py = viewport_px(y, 1, f.H, f.vy, f.vh);
    const float a = ((float)px + 0.0f) + (float)f.step / 2.0f;
    const float b = (((float)py + 0.0f) - (float)f.step / 2.0f) + 1.0f;
    float o[3], d[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const float p = (f.corner[c] + f.u[c] * a) + f.v[c] * b;
      o[c] = f.ortho ? p : f.eye[c];
      d[c] = f.ortho ? f.look[c] : p - f.eye[c];
    }
    norm3(d);
    float4 *r4 = reinterpret_cast<float4 *>(rays + k);
    r4[0] = make_float4(o[0], o[1], o[2], __uint_as_float(kNone));
    r4[1] = make_float4(d[0], d[1], d[2], 0.0f);
    if (pixel) pixel[k] = ((uint32_t)y << 16) | (uint32_t)x;
  }
}

// clamp() of the RGBA8 write: (int)(f * 255.0) as x86-64 converts (values
// out of int range give INT_MIN), then [0, 255].
__device__ __forceinline__ unsigned char to_u8(float f) {
  const double d = (double)f * 255.0;
  int i = (d >= -2147483648.0 && d < 2147483648.0) ? __double2int_rz(d) : INT_MIN;
  i = i < 0 ? 0 : (i > 255 ? 255 : i);
  return (unsigned char)i;
}

__global__ void framebuffer_kernel(const srt_hit *__restrict__ hits,
                                   const uint32_t *__restrict__ pixel,
                                   const float4 *__restrict__ rgba, uint32_t n, int W, int H,
                                   int step, int format, void *__restrict__ color,
                                   float *__restrict__ depth) {
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const float4 h = reinterpret_cast<const float4 *>(hits)[k];
    if (__float_as_uint(h.w) == kNone) continue;
    const int x = (int)(pixel[k] & 0xffffu), y = (int)(pixel[k] >> 16);
    const float4 c = rgba ? rgba[k] : make_float4(1.0f, 1.0f, 1.0f, 1.0f);
    for (int vv = 0; vv < step; vv++) {
      const int row = H - y - 1 + vv;
      if (row > H - 1 || row < 0) continue;
      for (int uu = 0; uu < step; uu++) {
        const int col = x + uu;
        if (col > W - 1) continue;
        const size_t p = (size_t)row * W + col;
        if (color && format == 0)
          reinterpret_cast<uchar4 *>(color)[p] =
              make_uchar4(to_u8(c.x * 1.0f), to_u8(c.y * 1.0f), to_u8(c.z * 1.0f),
                          to_u8(c.w * 1.0f));
        else if (color)
          reinterpret_cast<float4 *>(color)[p] =
              make_float4(c.x * 1.0f, c.y * 1.0f, c.z * 1.0f, c.w * 1.0f);
        if (depth) depth[p] = h.x * 1.0f;
      }
    }
  }
}

srt_status check_camera(const srt_camera *c) {
  if (!c || c->width <= 0 || c->height <= 0 || c->width > 65535 || c->height > 65535 ||
      c->step < 1 || c->viewport[2] < 0 || c->viewport[3] < 0 || c->region[0] < 0 ||
      c->region[1] < 0 || c->region[2] > 65535 || c->region[3] > 65535) {
    set_error("invalid camera: sizes 1..65535, step >= 1, region within 0..65535");
    return SRT_ERR_INVALID;
  }
  return SRT_OK;
}

}  // namespace
}  // namespace srt

using namespace srt;

extern "C" {

SRT_API srt_status srt_camera_rays(srt_ctx *ctx, const srt_camera *cam, srt_ray *rays,
                                   uint32_t *pixel, uint32_t *count) {
  if (!ctx || !cam || !rays || !count) {
    set_error("NULL argument");
    return SRT_ERR_INVALID;
  }
  *count = 0;
  srt_status s = check_camera(cam);
  if (s != SRT_OK) return s;
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_status(e, "set device");
  if (!is_device_ptr(rays) || (pixel && !is_device_ptr(pixel))) {
    set_error("srt_camera_rays: rays and pixel must be device memory");
    return SRT_ERR_INVALID;
  }
  if (reinterpret_cast<uintptr_t>(rays) & 15u) {
    set_error("ray array must be 16-byte aligned");
    return SRT_ERR_INVALID;
  }
  Frame f;
  build_frame(*cam, f);
  kept_range(cam->region[0], cam->region[2], cam->step, 0, cam->width, f.vx, f.vw, f.xs, f.nx);
  kept_range(cam->region[1], cam->region[3], cam->step, 1, cam->height, f.vy, f.vh, f.ys, f.ny);
  const size_t n = (size_t)f.nx * f.ny;
  if (n == 0) return SRT_OK;
  camera_rays_kernel<<<ctx->num_sms * 8, 256, 0, ctx->stream>>>(f, cam->region[0],
                                                                cam->region[1], rays, pixel);
  ctx->launches++;
  if ((s = cuda_status(cudaGetLastError(), "camera rays")) != SRT_OK) return s;
  *count = (uint32_t)n;
  return SRT_OK;
}

SRT_API srt_status srt_framebuffer_write(srt_ctx *ctx, const srt_camera *cam,
                                         const srt_hit *hits, const uint32_t *pixel,
                                         const float *rgba, uint32_t n, int32_t format,
                                         void *color, float *depth) {
  if (!ctx || !cam || (n && (!hits || !pixel)) || (format != 0 && format != 1)) {
    set_error("invalid framebuffer arguments");
    return SRT_ERR_INVALID;
  }
  srt_status s = check_camera(cam);
  if (s != SRT_OK) return s;
  if (n == 0) return SRT_OK;
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_status(e, "set device");
  if (!is_device_ptr(hits) || !is_device_ptr(pixel) || (rgba && !is_device_ptr(rgba)) ||
      (color && !is_device_ptr(color)) || (depth && !is_device_ptr(depth))) {
    set_error("srt_framebuffer_write: all arrays must be device memory");
    return SRT_ERR_INVALID;
  }
  if ((reinterpret_cast<uintptr_t>(hits) | reinterpret_cast<uintptr_t>(rgba) |
       reinterpret_cast<uintptr_t>(color)) & 15u) {
    set_error("hit, colour and framebuffer arrays must be 16-byte aligned");
    return SRT_ERR_INVALID;
  }
  framebuffer_kernel<<<ctx->num_sms * 8, 256, 0, ctx->stream>>>(
      hits, pixel, reinterpret_cast<const float4 *>(rgba), n, cam->width, cam->height,
      cam->step, format, color, depth);
  ctx->launches++;
  return cuda_status(cudaGetLastError(), "framebuffer write");
}

}  // extern "C"
