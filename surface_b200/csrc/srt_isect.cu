// srt_isect.cu -- shading records of traced rays (srt_trace_opts.isect).
//
// The reference's Traverse ends in BuildIntersection, which fills the
// Intersection fields the GLSL fragment stage interpolates varyings from
// (gles/gles_common.cc:1007-1141): the hit position, the geometric normal,
// the primitive's vertex ids f0..f3 and, for tetrahedra, InterpolateTetra's
// weights d0..d3; for spheres also the tangent and binormal of the spherical
// parameterisation.  Here that step is one pass after the trace kernels: one
// thread per ray reads its hit, ray and (tetrahedra) entering face, gathers
// the primitive's vertices from the arrays the tree was built from and
// writes an 80-byte record as five 16-byte stores.  Keeping it out of the
// traversal kernels keeps their register footprint unchanged.
//
// Every float and double expression keeps the reference's operation order
// (the file is compiled without contraction), so the records are bit for bit
// the reference's; the spheres' angles are the one exception (sphere_uv).
#include <cuda_runtime.h>

#include "srt_internal.cuh"

namespace srt {
namespace {

__device__ __forceinline__ void sub3(const float a[3], const float b[3], float c[3]) {
  c[0] = a[0] - b[0];
  c[1] = a[1] - b[1];
  c[2] = a[2] - b[2];
}
__device__ __forceinline__ float dot3f(const float a[3], const float b[3]) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}
__device__ __forceinline__ void cross3f(const float a[3], const float b[3], float c[3]) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}
// real3::length (render/render_common.h): sqrt of the float sum of squares
__device__ __forceinline__ float len3f(const float a[3]) {
  return sqrtf(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
}
// real3::normalize (render/render_common.h): scale by 1 / sqrt(|v|^2) in double
__device__ __forceinline__ void normalize3(float n[3]) {
  const double l2 = (double)(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
  double len = 0.0;
  if (fabs(l2) > 1.0e-30) len = 1.0 / sqrt(l2);
#pragma unroll
  for (int k = 0; k < 3; k++) n[k] = (float)((double)n[k] * len);
}

// InterpolateTetra (render/render_accel_tetra.cc:148-241) with its default
// mode 0: for each vertex v, the ray from v through pt is cut with the
// opposite face (Pluecker side tests of the six edges against that ray,
// tolerance 0.001), d_v = 1 - |pt - v| / |cut - v|; the four values are
// weighted by sum_k |pt - V_k| / |pt - V_v| and normalised to sum 1.
__device__ void interpolate_tet(const float pt[3], const float V[4][3], float dout[4]) {
  const float kEPS = 0.001f;
  float E[6][3];
  sub3(V[1], V[0], E[0]);
  sub3(V[2], V[1], E[1]);
  sub3(V[0], V[2], E[2]);
  sub3(V[3], V[0], E[3]);
  sub3(V[3], V[1], E[4]);
  sub3(V[3], V[2], E[5]);
#pragma unroll 1
  for (int v = 0; v < 4; v++) {
    const float *ro = V[v];
    float rd[3], pc[3];
    sub3(pt, ro, rd);
    cross3f(rd, ro, pc);
    const float d = len3f(rd);  // (pt - rayorg).length(), the same difference
    float ws[6];
    uint32_t ge = 0, le = 0;  // bit i: ws[i] >= -kEPS / ws[i] <= kEPS
#pragma unroll
    for (int i = 0; i < 6; i++) {
      float cv[3];
      cross3f(E[i], V[i % 3], cv);
      ws[i] = dot3f(rd, cv) + dot3f(E[i], pc);
      ge |= (ws[i] >= -kEPS ? 1u : 0u) << i;
      le |= (ws[i] <= kEPS ? 1u : 0u) << i;
    }
    float cp[3] = {1e16f, 1e16f, 1e16f};
    // the face opposite v is the only one whose vertex list lacks v
    if ((ge & 1u) && (ge & 2u) && (ge & 4u) && v == 3) {
      const float s = ws[0] + ws[1] + ws[2];
#pragma unroll
      for (int k = 0; k < 3; k++) cp[k] = (V[2][k] * ws[0] + V[0][k] * ws[1] + V[1][k] * ws[2]) / s;
    } else if ((le & 2u) && (ge & 16u) && (le & 32u) && v == 0) {
      const float s = ws[5] + ws[1] - ws[4];
#pragma unroll
      for (int k = 0; k < 3; k++) cp[k] = (V[3][k] * ws[1] + V[1][k] * ws[5] - V[2][k] * ws[4]) / s;
    } else if ((le & 4u) && (le & 8u) && (ge & 32u) && v == 1) {
      const float s = ws[2] + ws[3] - ws[5];
#pragma unroll
      for (int k = 0; k < 3; k++) cp[k] = (V[3][k] * ws[2] + V[2][k] * ws[3] - V[0][k] * ws[5]) / s;
    } else if ((le & 1u) && (ge & 8u) && (le & 16u) && v == 2) {
      const float s = ws[0] + ws[4] - ws[3];
#pragma unroll
      for (int k = 0; k < 3; k++) cp[k] = (V[3][k] * ws[0] + V[0][k] * ws[4] - V[1][k] * ws[3]) / s;
    }
    float cr[3];
    sub3(cp, ro, cr);
    float q = d / len3f(cr);
    if (q < 0.0f) {
      q = 0.0f;
    } else if (!(q < 1.0f) && !(q > 0.0f)) {
      q = 1.0f;  // NaN
    }
    dout[v] = 1.0f - q;
  }
  float ds = 0.0f;
  float lens[4];
#pragma unroll
  for (int k = 0; k < 4; k++) {
    float r[3];
    sub3(pt, V[k], r);
    lens[k] = len3f(r);
    ds += lens[k];
  }
  float w = 0.0f;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    dout[k] *= ds / lens[k];
    w += dout[k];
  }
#pragma unroll
  for (int k = 0; k < 4; k++) dout[k] = dout[k] / w;
}

__device__ __forceinline__ void load_vertex(const float *__restrict__ verts, uint32_t id,
                                            float p[3]) {
  p[0] = __ldg(&verts[3 * (size_t)id]);
  p[1] = __ldg(&verts[3 * (size_t)id + 1]);
  p[2] = __ldg(&verts[3 * (size_t)id + 2]);
}

template <int KIND>
__global__ void __launch_bounds__(128)
isect_kernel(const srt_ray *__restrict__ rays, size_t n, const float4 *__restrict__ hits,
             const uint32_t *__restrict__ subface, const float *__restrict__ verts,
             const uint32_t *__restrict__ faces, float4 *__restrict__ out) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float4 h = hits[i];
  const uint32_t prim = __float_as_uint(h.w);
  float4 *o = out + 5 * i;
  if (prim == kNone) {
    const float4 z = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
#pragma unroll
    for (int k = 0; k < 5; k++) o[k] = z;
    return;
  }
  const float4 *r4 = reinterpret_cast<const float4 *>(rays + i);
  const float4 ra = r4[0], rb = r4[1];
  const float t = h.x;
  // isect.position = ray.origin() + isect.t * ray.direction()
  const float pos[3] = {ra.x + t * rb.x, ra.y + t * rb.y, ra.z + t * rb.z};
  float nrm[3] = {0.0f, 0.0f, 0.0f}, tan[3] = {0.0f, 0.0f, 0.0f}, bin[3] = {0.0f, 0.0f, 0.0f};
  uint32_t f[4] = {0u, 0u, 0u, 0u};
  float d[4] = {0.0f, 0.0f, 0.0f, 0.0f};
  if (KIND == SRT_TRIANGLES) {
    // render/render_accel_triangle.cc:2439-2507
    float p[3][3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
      f[k] = __ldg(&faces[3 * (size_t)prim + k]);
      load_vertex(verts, f[k], p[k]);
    }
    float e1[3], e2[3];
    sub3(p[1], p[0], e1);
    sub3(p[2], p[0], e2);
    cross3f(e1, e2, nrm);
    normalize3(nrm);
  } else if (KIND == SRT_TETRAHEDRA) {
    // render/render_accel_tetra.cc:2124-2196; face_table of the entering face
    float p[4][3];
#pragma unroll
    for (int k = 0; k < 4; k++) {
      f[k] = __ldg(&faces[4 * (size_t)prim + k]);
      load_vertex(verts, f[k], p[k]);
    }
    const uint32_t sf = subface[i] & 3u;
    const int ft0[4] = {0, 1, 2, 0}, ft1[4] = {1, 2, 0, 1}, ft2[4] = {3, 3, 3, 2};
    float e1[3], e2[3];
    sub3(p[ft1[sf]], p[ft0[sf]], e1);
    sub3(p[ft2[sf]], p[ft0[sf]], e2);
    cross3f(e1, e2, nrm);
    normalize3(nrm);
    interpolate_tet(pos, p, d);
  } else {
    // render/render_accel_particle.cc:2966-3049
    f[0] = f[1] = f[2] = prim;
    float c[3];
    load_vertex(verts, prim, c);
    sub3(pos, c, nrm);
    const float len = sqrtf(dot3f(nrm, nrm));
    if (len > FLT_EPSILON * 16) {
      const float il = __frcp_rn(len);  // (real)(1.0 / len)
#pragma unroll
      for (int k = 0; k < 3; k++) nrm[k] *= il;
    }
    const float xz2 = nrm[0] * nrm[0] + nrm[2] * nrm[2];
    if (xz2 > 0.0f) {
      const float xz = sqrtf(xz2);
      const float inv = __frcp_rn(xz);
      tan[0] = (float)((-2.0 * kPi) * (double)nrm[0]);
      tan[1] = (float)((2.0 * kPi) * (double)nrm[2]);
      tan[2] = 0.0f;
      bin[0] = (float)(((-kPi * (double)nrm[2]) * (double)inv) * (double)nrm[1]);
      bin[1] = (float)(((-kPi * (double)nrm[0]) * (double)inv) * (double)nrm[1]);
      bin[2] = (float)(kPi * (double)xz);
    } else {
      tan[2] = 1.0f;
      bin[0] = nrm[1] > 0.0f ? 1.0f : -1.0f;
    }
  }
  o[0] = make_float4(pos[0], pos[1], pos[2], __uint_as_float(f[0]));
  o[1] = make_float4(nrm[0], nrm[1], nrm[2], __uint_as_float(f[1]));
  o[2] = make_float4(tan[0], tan[1], tan[2], __uint_as_float(f[2]));
  o[3] = make_float4(bin[0], bin[1], bin[2], __uint_as_float(f[3]));
  o[4] = make_float4(d[0], d[1], d[2], d[3]);
}

}  // namespace

srt_status launch_isect(srt_accel *a, const srt_ray *rays, size_t n, const srt_hit *hits,
                        const uint32_t *subface, srt_isect *isect) {
  if (n == 0) return SRT_OK;
  if ((reinterpret_cast<uintptr_t>(isect) & 15u) != 0) {
    set_error("isect array must be 16-byte aligned");
    return SRT_ERR_INVALID;
  }
  if (a->kind == SRT_TETRAHEDRA && !subface) {
    set_error("tetrahedron shading records need the entering faces");
    return SRT_ERR_INVALID;
  }
  srt_ctx *ctx = a->ctx;
  const int block = 128;
  const unsigned grid = (unsigned)((n + block - 1) / block);
  const float4 *h4 = reinterpret_cast<const float4 *>(hits);
  float4 *o4 = reinterpret_cast<float4 *>(isect);
  switch (a->kind) {
    case SRT_TRIANGLES:
      isect_kernel<SRT_TRIANGLES><<<grid, block, 0, ctx->stream>>>(
          rays, n, h4, subface, a->src_verts, a->src_faces, o4);
      break;
    case SRT_TETRAHEDRA:
      isect_kernel<SRT_TETRAHEDRA><<<grid, block, 0, ctx->stream>>>(
          rays, n, h4, subface, a->src_verts, a->src_faces, o4);
      break;
    case SRT_SPHERES:
      isect_kernel<SRT_SPHERES><<<grid, block, 0, ctx->stream>>>(
          rays, n, h4, subface, a->src_verts, a->src_faces, o4);
      break;
  }
  ctx->launches++;
  return cuda_status(cudaGetLastError(), "isect");
}

}  // namespace srt
