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
#include <mutex>
#include <vector>

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

// ---------------------------------------------------------------- samples
// The serial renderer's random stream: TinyMT64 (M. Saito and M. Matsumoto,
// "Tiny Mersenne Twister", 2011) with initialize_random's parameters.  Its
// state step is linear over GF(2) on the 128 state bits, so the state n
// draws later is A^n times the state: the host jumps to each row's first
// draw with powers of A and the GPU draws every row in parallel.
constexpr uint32_t kTmtMat1 = 0xfa051f40u, kTmtMat2 = 0xffd0fff4u;
constexpr uint64_t kTmtTmat = 0x58d02ffeffbfffbcull;

__host__ __device__ inline void tmt_next(uint64_t &s0, uint64_t &s1) {
  s0 &= 0x7fffffffffffffffull;
  uint64_t x = s0 ^ s1;
  x ^= x << 12;
  x ^= x >> 32;
  x ^= x << 32;
  x ^= x << 11;
  s0 = s1;
  s1 = x;
  if (x & 1u) {
    s0 ^= (uint64_t)kTmtMat1;
    s1 ^= (uint64_t)kTmtMat2 << 32;
  }
}

// One draw: the tempered output as a double in [0, 1], rounded to float.
__host__ __device__ inline float tmt_real(uint64_t s0, uint64_t s1) {
  uint64_t x = s0 + s1;
  x ^= s0 >> 8;
  if (x & 1u) x ^= kTmtTmat;
  return (float)((double)x * (1.0 / 18446744073709551616.0));
}

void tmt_seed(uint64_t seed, uint64_t &s0, uint64_t &s1) {
  uint64_t st[2] = {seed ^ ((uint64_t)kTmtMat1 << 32), (uint64_t)kTmtMat2 ^ kTmtTmat};
  for (int i = 1; i < 8; i++) {
    const uint64_t p = st[(i - 1) & 1];
    st[i & 1] ^= (uint64_t)i + 6364136223846793005ull * (p ^ (p >> 62));
  }
  if ((st[0] & 0x7fffffffffffffffull) == 0 && st[1] == 0) {
    st[0] = 'T';
    st[1] = 'M';
  }
  s0 = st[0];
  s1 = st[1];
}

// 128 x 128 matrices over GF(2): column j is the image of state bit j
// (bits 0..63: s0, 64..127: s1).
struct Gf2 {
  uint64_t col[128][2];
};

inline void gf2_apply(const Gf2 &m, uint64_t &s0, uint64_t &s1) {
  uint64_t r0 = 0, r1 = 0;
  for (int j = 0; j < 128; j++) {
    const uint64_t bit = j < 64 ? (s0 >> j) & 1u : (s1 >> (j - 64)) & 1u;
    if (bit) {
      r0 ^= m.col[j][0];
      r1 ^= m.col[j][1];
    }
  }
  s0 = r0;
  s1 = r1;
}

inline void gf2_mul(const Gf2 &a, const Gf2 &b, Gf2 &out) {  // out = a b
  for (int j = 0; j < 128; j++) {
    uint64_t s0 = b.col[j][0], s1 = b.col[j][1];
    gf2_apply(a, s0, s1);
    out.col[j][0] = s0;
    out.col[j][1] = s1;
  }
}

// A^(2^b), b < 64, computed once.
const std::vector<Gf2> &tmt_powers() {
  static std::vector<Gf2> p;
  static std::once_flag once;
  std::call_once(once, [] {
    p.resize(64);
    for (int j = 0; j < 128; j++) {
      uint64_t s0 = j < 64 ? 1ull << j : 0, s1 = j < 64 ? 0 : 1ull << (j - 64);
      tmt_next(s0, s1);
      p[0].col[j][0] = s0;
      p[0].col[j][1] = s1;
    }
    for (int b = 1; b < 64; b++) gf2_mul(p[b - 1], p[b - 1], p[b]);
  });
  return p;
}

void tmt_jump(uint64_t &s0, uint64_t &s1, uint64_t n) {
  const std::vector<Gf2> &p = tmt_powers();
  for (int b = 0; b < 64 && n; b++, n >>= 1)
    if (n & 1u) gf2_apply(p[b], s0, s1);
}

// Draws of one frame: row j of the kept pixels starts at rows[j] and makes
// per_row draws.
__global__ void jitter_kernel(const ulonglong2 *__restrict__ rows, int ny, size_t per_row,
                              float *__restrict__ draws) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < ny; j += gridDim.x * blockDim.x) {
    uint64_t s0 = rows[j].x, s1 = rows[j].y;
    float *out = draws + (size_t)j * per_row;
    for (size_t i = 0; i < per_row; i++) {
      tmt_next(s0, s1);
      out[i] = tmt_real(s0, s1);
    }
  }
}

// Camera::generateStereoEnvRay (render/render_camera.cc:65-118) with the
// stereo camera's frame (u, v, look) = m_uvw; double where the reference
// widens (fmod, atan2 and the psi rotation), float sinf / cosf elsewhere.
__device__ inline void stereo_env_ray(const float eye[3], const float uvw[9], float zp,
                                      float es, float image_u, float image_v, int W, int H,
                                      float org[3], float dir[3]) {
  const bool left = image_v < (float)(H / 2);
  const float theta = (float)(M_PI * fmod(2.0 * (double)image_v / (double)H, 1.0));
  const float phi = (float)(2.0 * M_PI * (double)(image_u / (float)W));
  // sinf / cosf as double and rounded: the C library's float functions
  // return the correctly rounded value in all but rare cases
  const float st = (float)sin((double)theta), ct = (float)cos((double)theta);
  const float sp = (float)sin((double)phi), cp = (float)cos((double)phi);
  const float o0 = st * cp, o1 = ct, o2 = st * sp;
  float par[3] = {left ? -o2 : o2, 0.0f, left ? o0 : -o0};
  norm3(par);
#pragma unroll
  for (int k = 0; k < 3; k++) org[k] = eye[k] + par[k] * es;
  float psi = (float)atan2((double)es, (double)zp);
  if (left) psi = -psi;
  const double cps = cos((double)psi), sps = sin((double)psi);
  const float d0 = (float)(o0 * cps - o2 * sps), d1 = o1, d2 = (float)(o0 * sps + o2 * cps);
#pragma unroll
  for (int k = 0; k < 3; k++) dir[k] = (uvw[k] * d0 + uvw[3 + k] * d1) + uvw[6 + k] * d2;
}

// Draws before subsample (vv, uu) of a pixel with S x S samples.
__host__ __device__ inline int draws_before(int S, int vv, int uu) {
  const int row = vv == 0 ? 0 : (S - 1) + (vv - 1) * (2 * S - 1);
  const int in = vv == 0 ? (uu > 0 ? uu - 1 : 0) : (uu == 0 ? 0 : 1 + 2 * (uu - 1));
  return row + in;
}

struct SampleSet {
  int S, stereo;
  float zp, es;
  float uvw[9];  // stereo camera frame
};

__global__ void camera_rays_ex_kernel(const Frame f, const SampleSet ss, int x0, int y0,
                                      const float *__restrict__ draws,
                                      srt_ray *__restrict__ rays, uint32_t *__restrict__ pixel) {
  const int S = ss.S, S2 = S * S, D = 2 * S * (S - 1);
  const size_t n = (size_t)f.nx * f.ny * S2;
  for (size_t r = blockIdx.x * (size_t)blockDim.x + threadIdx.x; r < n;
       r += (size_t)gridDim.x * blockDim.x) {
    const size_t q = r / S2;
    const int sub = (int)(r - q * S2), vv = sub / S, uu = sub - vv * S;
    const int ix = (int)(q % f.nx), iy = (int)(q / f.nx);
    const int x = x0 + (f.xs + ix) * f.step, y = y0 + (f.ys + iy) * f.step;
    const int px = viewport_px(x, 0, f.W, f.vx, f.vw);
    const int py = viewport_px(y, 1, f.H, f.vy, f.vh);
    float ju = 0.0f, jv = 0.0f;
    if (D) {
      const float *dq = draws + q * D + draws_before(S, vv, uu);
      if (uu != 0) ju = dq[0];
      if (vv != 0) jv = dq[uu != 0 ? 1 : 0];
    }
    const float su = ((float)uu + ju) / (float)S, sv = ((float)vv + jv) / (float)S;
    const float a = ((float)px + su) + (float)f.step / 2.0f;
    const float b = (((float)py + sv) - (float)f.step / 2.0f) + 1.0f;
    float o[3], d[3];
    if (ss.stereo) {
      stereo_env_ray(f.eye, ss.uvw, ss.zp, ss.es, a, b, f.W, f.H, o, d);
    } else {
#pragma unroll
      for (int c = 0; c < 3; c++) {
        const float p = (f.corner[c] + f.u[c] * a) + f.v[c] * b;
        o[c] = f.ortho ? p : f.eye[c];
        d[c] = f.ortho ? f.look[c] : p - f.eye[c];
      }
    }
    norm3(d);
    float4 *r4 = reinterpret_cast<float4 *>(rays + r);
    r4[0] = make_float4(o[0], o[1], o[2], __uint_as_float(kNone));
    r4[1] = make_float4(d[0], d[1], d[2], 0.0f);
    if (pixel) pixel[r] = ((uint32_t)y << 16) | (uint32_t)x;
  }
}

// Per loop pixel: its S^2 rays' hits summed in order, times 1 / S^2.
__global__ void framebuffer_ex_kernel(const srt_hit *__restrict__ hits,
                                      const uint32_t *__restrict__ pixel,
                                      const float4 *__restrict__ rgba, uint32_t n, int S, int W,
                                      int H, int step, int format, void *__restrict__ color,
                                      float *__restrict__ depth) {
  const uint32_t per = (uint32_t)(S * S), groups = n / per;
  const float inv_n = 1.0f / (float)(S * S);
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < groups;
       g += gridDim.x * blockDim.x) {
    float4 c = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    float dv = 0.0f;
    bool frag = false;
    for (uint32_t q = g * per; q < (g + 1) * per; q++) {
      const float4 h = reinterpret_cast<const float4 *>(hits)[q];
      if (__float_as_uint(h.w) == kNone) continue;
      const float4 col = rgba ? rgba[q] : make_float4(1.0f, 1.0f, 1.0f, 1.0f);
      c.x += col.x;
      c.y += col.y;
      c.z += col.z;
      c.w += col.w;
      dv += h.x;
      frag = true;
    }
    if (!frag) continue;
    dv *= inv_n;
    const int x = (int)(pixel[g * per] & 0xffffu), y = (int)(pixel[g * per] >> 16);
    for (int vv = 0; vv < step; vv++) {
      const int row = H - y - 1 + vv;
      if (row > H - 1 || row < 0) continue;
      for (int uu = 0; uu < step; uu++) {
        const int col = x + uu;
        if (col > W - 1) continue;
        const size_t p = (size_t)row * W + col;
        if (color && format == 0)
          reinterpret_cast<uchar4 *>(color)[p] =
              make_uchar4(to_u8(c.x * inv_n), to_u8(c.y * inv_n), to_u8(c.z * inv_n),
                          to_u8(c.w * inv_n));
        else if (color)
          reinterpret_cast<float4 *>(color)[p] =
              make_float4(c.x * inv_n, c.y * inv_n, c.z * inv_n, c.w * inv_n);
        if (depth) depth[p] = dv;
      }
    }
  }
}

srt_status check_samples(const srt_camera_samples *s) {
  if (!s || s->subsamples < 1 || s->subsamples > 16) {
    set_error("invalid camera samples: subsamples 1..16");
    return SRT_ERR_INVALID;
  }
  return SRT_OK;
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

SRT_API srt_status srt_camera_rays_ex(srt_ctx *ctx, const srt_camera *cam,
                                      const srt_camera_samples *smp, srt_ray *rays,
                                      uint32_t *pixel, uint32_t *count, uint64_t *draws) {
  if (!ctx || !cam || !rays || !count) {
    set_error("NULL argument");
    return SRT_ERR_INVALID;
  }
  *count = 0;
  if (draws) *draws = 0;
  srt_status s = check_camera(cam);
  if (s == SRT_OK) s = check_samples(smp);
  if (s != SRT_OK) return s;
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_status(e, "set device");
  if (!is_device_ptr(rays) || (pixel && !is_device_ptr(pixel))) {
    set_error("srt_camera_rays_ex: rays and pixel must be device memory");
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
  const int S = smp->subsamples;
  const size_t D = (size_t)2 * S * (S - 1);
  const size_t npix = (size_t)f.nx * f.ny, n = npix * S * S;
  if (n == 0) return SRT_OK;
  if (n > 0xffffffffull) {
    set_error("srt_camera_rays_ex: more than 2^32 - 1 rays");
    return SRT_ERR_INVALID;
  }
  SampleSet ss;
  ss.S = S;
  ss.stereo = smp->stereo_env != 0;
  ss.zp = smp->zero_parallax;
  ss.es = smp->eye_separation;
  {
    // the stereo camera's frame (render/render_camera.h:44-60)
    float look[3], u[3], v[3];
    for (int k = 0; k < 3; k++) look[k] = cam->lookat[k] - cam->eye[k];
    cross3(cam->up, look, u);
    norm3(u);
    cross3(look, u, v);
    norm3(v);
    norm3(look);
    for (int k = 0; k < 3; k++) {
      ss.uvw[k] = u[k];
      ss.uvw[3 + k] = v[k];
      ss.uvw[6 + k] = look[k];
    }
  }
  const float *d_draws = nullptr;
  if (D) {
    // row start states on the host (jumps over GF(2)), the draws on the GPU
    uint64_t s0, s1;
    tmt_seed(smp->jitter_seed, s0, s1);
    tmt_jump(s0, s1, smp->jitter_offset);
    const size_t per_row = (size_t)f.nx * D;
    std::vector<ulonglong2> rows(f.ny);
    for (int j = 0; j < f.ny; j++) {
      rows[j] = make_ulonglong2(s0, s1);
      tmt_jump(s0, s1, per_row);
    }
    if ((e = ctx->s_stage_aux.ensure(f.ny * sizeof(ulonglong2))) != cudaSuccess ||
        (e = ctx->s_stage_scal.ensure(npix * D * sizeof(float))) != cudaSuccess)
      return cuda_status(e, "camera jitter");
    // pageable source: the copy has read it when the call returns
    if ((e = cudaMemcpyAsync(ctx->s_stage_aux.p, rows.data(), f.ny * sizeof(ulonglong2),
                             cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess)
      return cuda_status(e, "camera jitter");
    jitter_kernel<<<(f.ny + 63) / 64, 64, 0, ctx->stream>>>(
        ctx->s_stage_aux.as<ulonglong2>(), f.ny, per_row, ctx->s_stage_scal.as<float>());
    ctx->launches++;
    d_draws = ctx->s_stage_scal.as<float>();
  }
  camera_rays_ex_kernel<<<ctx->num_sms * 8, 256, 0, ctx->stream>>>(
      f, ss, cam->region[0], cam->region[1], d_draws, rays, pixel);
  ctx->launches++;
  if ((s = cuda_status(cudaGetLastError(), "camera rays")) != SRT_OK) return s;
  *count = (uint32_t)n;
  if (draws) *draws = npix * D;
  return SRT_OK;
}

SRT_API srt_status srt_framebuffer_write_ex(srt_ctx *ctx, const srt_camera *cam,
                                            const srt_camera_samples *smp,
                                            const srt_hit *hits, const uint32_t *pixel,
                                            const float *rgba, uint32_t n, int32_t format,
                                            void *color, float *depth) {
  if (!ctx || !cam || (n && (!hits || !pixel)) || (format != 0 && format != 1)) {
    set_error("invalid framebuffer arguments");
    return SRT_ERR_INVALID;
  }
  srt_status s = check_camera(cam);
  if (s == SRT_OK) s = check_samples(smp);
  if (s != SRT_OK) return s;
  const uint32_t per = (uint32_t)(smp->subsamples * smp->subsamples);
  if (n % per) {
    set_error("srt_framebuffer_write_ex: n is not a multiple of subsamples^2");
    return SRT_ERR_INVALID;
  }
  if (n == 0) return SRT_OK;
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_status(e, "set device");
  if (!is_device_ptr(hits) || !is_device_ptr(pixel) || (rgba && !is_device_ptr(rgba)) ||
      (color && !is_device_ptr(color)) || (depth && !is_device_ptr(depth))) {
    set_error("srt_framebuffer_write_ex: all arrays must be device memory");
    return SRT_ERR_INVALID;
  }
  if ((reinterpret_cast<uintptr_t>(hits) | reinterpret_cast<uintptr_t>(rgba) |
       reinterpret_cast<uintptr_t>(color)) & 15u) {
    set_error("hit, colour and framebuffer arrays must be 16-byte aligned");
    return SRT_ERR_INVALID;
  }
  framebuffer_ex_kernel<<<ctx->num_sms * 8, 256, 0, ctx->stream>>>(
      hits, pixel, reinterpret_cast<const float4 *>(rgba), n, smp->subsamples, cam->width,
      cam->height, cam->step, format, color, depth);
  ctx->launches++;
  return cuda_status(cudaGetLastError(), "framebuffer write");
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
