// srt_trace.cu -- closest-hit traversal, one ray per thread.
//
// Each kernel reproduces the reference's Traverse() step for step, so hits
// (including which of several equal-t primitives wins) match bit for bit:
//   triangles  TriangleAccel::Traverse  render/render_accel_triangle.cc:2511-2669
//              IntersectRayAABB :1815-1861, TriangleIsect :1887-1938,
//              TestLeafNode :1994-2437, BuildIntersection :2439-2507
//   tetrahedra TetraAccel::Traverse     render/render_accel_tetra.cc:2200-2289
//              IntersectRayAABB :1934-1978, TestLeafNode :1980-2122,
//              RayTetraPluecker :243-567 (FP64), ComputeParametricDist :123-139
//   spheres    ParticleAccel::Traverse  render/render_accel_particle.cc:3053-3218
//              SphereIsect :2423-2512, BuildIntersection :2968-3049
// The stack discipline (far child pushed first, near child popped next,
// near = dirSign[axis]) and the per-node hitT culling are the reference's.
// Leaves are folded into their parent's child slot for triangles/spheres;
// a hit leaf is pushed as a (first primitive, count) entry, which visits
// leaves in exactly the reference's order.
#include "srt_internal.cuh"

namespace srt {
namespace {

struct RayF {
  float o[3], d[3], inv[3];
  int sgn[3];
};

__device__ __forceinline__ RayF load_ray(const srt_ray *__restrict__ rays, size_t i,
                                         uint32_t &prev_prim, float &prev_t) {
  const float4 *r4 = reinterpret_cast<const float4 *>(rays + i);
  float4 a = __ldg(&r4[0]);
  float4 b = __ldg(&r4[1]);
  RayF r;
  r.o[0] = a.x; r.o[1] = a.y; r.o[2] = a.z;
  r.d[0] = b.x; r.d[1] = b.y; r.d[2] = b.z;
  prev_prim = __float_as_uint(a.w);
  prev_t = b.w;
#pragma unroll
  for (int k = 0; k < 3; k++) {
    r.sgn[k] = r.d[k] < 0.0f ? 1 : 0;
    // (float)(1.0 / (double)d): the correctly rounded reciprocal
    r.inv[k] = __frcp_rn(r.d[k]);
  }
  return r;
}

// IntersectRayAABB; CLAMP: tmax = min(tmax, maxT) (triangle/particle) else
// the tetra variant's tmin <= maxT.
template <bool CLAMP>
__device__ __forceinline__ bool ray_aabb(float maxT, float lx, float ly, float lz,
                                         float hx, float hy, float hz, const RayF &r) {
  const float min_x = r.sgn[0] ? hx : lx;
  const float min_y = r.sgn[1] ? hy : ly;
  const float min_z = r.sgn[2] ? hz : lz;
  const float max_x = r.sgn[0] ? lx : hx;
  const float max_y = r.sgn[1] ? ly : hy;
  const float max_z = r.sgn[2] ? lz : hz;
  const float tmin_x = (min_x - r.o[0]) * r.inv[0];
  const float tmax_x = (max_x - r.o[0]) * r.inv[0];
  const float tmin_y = (min_y - r.o[1]) * r.inv[1];
  const float tmax_y = (max_y - r.o[1]) * r.inv[1];
  float tmin = (tmin_x > tmin_y) ? tmin_x : tmin_y;
  float tmax = (tmax_x < tmax_y) ? tmax_x : tmax_y;
  const float tmin_z = (min_z - r.o[2]) * r.inv[2];
  const float tmax_z = (max_z - r.o[2]) * r.inv[2];
  tmin = (tmin > tmin_z) ? tmin : tmin_z;
  tmax = (tmax < tmax_z) ? tmax : tmax_z;
  if (CLAMP) {
    tmax = (maxT < tmax) ? maxT : tmax;
    return (tmax > 0.0f) && (tmin <= tmax);
  }
  return (tmax > 0.0f) && (tmin <= tmax) && (tmin <= maxT);
}

__device__ __forceinline__ float dot3(const float a[3], const float b[3]) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}
__device__ __forceinline__ void cross3(const float a[3], const float b[3], float c[3]) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}

// TriangleIsect, double-sided.
__device__ __forceinline__ bool tri_isect(float &tio, float &uo, float &vo,
                                          const float p0[3], const float p1[3],
                                          const float p2[3], const RayF &r, float keps) {
  float e1[3], e2[3], p[3], s[3], q[3];
#pragma unroll
  for (int k = 0; k < 3; k++) {
    e1[k] = p1[k] - p0[k];
    e2[k] = p2[k] - p0[k];
  }
  cross3(r.d, e2, p);
  const float det = dot3(e1, p);
  if (fabsf(det) < keps) return false;
  const float inv_det = __frcp_rn(det);  // == (float)(1.0 / (double)det)
#pragma unroll
  for (int k = 0; k < 3; k++) s[k] = r.o[k] - p0[k];
  cross3(s, e1, q);
  const float u = dot3(s, p) * inv_det;
  const float v = dot3(q, r.d) * inv_det;
  const float t = dot3(e2, q) * inv_det;
  if (u < 0.0f || u > 1.0f) return false;
  if (v < 0.0f || u + v > 1.0f) return false;
  if (t < 0.0f || t > tio) return false;
  tio = t;
  uo = u;
  vo = v;
  return true;
}

// --------------------------------------------------------------- FP64 Pluecker
struct D3 {
  double x, y, z;
};
__device__ __forceinline__ D3 dsub(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ D3 dadd(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ D3 dscale(double f, D3 v) { return {v.x * f, v.y * f, v.z * f}; }
__device__ __forceinline__ D3 dcross(D3 a, D3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ double ddot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ int dsign(double x) {
  return x > DBL_EPSILON ? 1 : (x < -DBL_EPSILON ? -1 : 0);
}
struct Plk {
  D3 d, c;
};
__device__ __forceinline__ Plk plk(D3 v0, D3 v1) { return {dsub(v1, v0), dcross(v1, v0)}; }
__device__ __forceinline__ double pdot(const Plk &a, const Plk &b) {
  return ddot(a.d, b.c) + ddot(b.d, a.c);
}
__device__ __forceinline__ D3 bary(double a, double b, D3 A, D3 B, D3 C) {
  return dadd(dadd(dscale(1 - a - b, A), dscale(a, B)), dscale(b, C));
}
__device__ __forceinline__ double param_enter(D3 o, D3 d, D3 pe) {
  if (d.x != 0.0) {
    double iv = 1.0 / d.x;
    return (pe.x - o.x) * iv;
  } else if (d.y != 0.0) {
    double iv = 1.0 / d.y;
    return (pe.y - o.y) * iv;
  }
  double iv = 1.0 / d.z;
  return (pe.z - o.z) * iv;
}

// Entering face, its barycentrics (ue1, ue2), the leaving face's first
// barycentric ul1 and tEnter.  Same branch structure as RayTetraPluecker;
// only the entering point is needed for tEnter (ComputeParametricDist).
__device__ bool ray_tet(D3 orig, D3 dir, const D3 V[4], int &ef, double &ue1,
                        double &ue2, double &ul1, double &te) {
  double uAB, uAC, uDB = 0, uDC = 0, uBC = 0, uAD = 0;
  int sAB, sAC, sDB = -2, sDC = -2, sBC = -2, sAD = -2;
  double eu1 = 0, eu2 = 0, lu1 = 0;
  D3 ep = {0, 0, 0};
  int enterF = -1;
  const D3 dest = dadd(orig, dir);
  const Plk ray = plk(orig, dest);
  int next = 0;
#define ENTER(F, A1, A2, P0, P1, P2) \
  do { enterF = F; eu1 = A1; eu2 = A2; ep = bary(eu1, eu2, P0, P1, P2); } while (0)
#define LEAVE(F, A1, A2) \
  do { lu1 = A1; (void)(A2); } while (0)
#define DONE() \
  do { te = param_enter(orig, dir, ep); ef = enterF; ue1 = eu1; ue2 = eu2; ul1 = lu1; return true; } while (0)

  uAB = pdot(ray, plk(V[0], V[1])); sAB = dsign(uAB);
  uAC = pdot(ray, plk(V[0], V[2])); sAC = dsign(uAC);
  if ((sAC == -sAB) || (sAC == 0) || (sAB == 0)) {
    uBC = pdot(ray, plk(V[1], V[2])); sBC = dsign(uBC);
    int sABC = sAB;
    if (sABC == 0) { sABC = -sAC; if (sABC == 0) sABC = sBC; }
    if ((sABC != 0) && ((sBC == sABC) || (sBC == 0))) {
      double inv = 1.0 / (uAB + uBC - uAC);
      if (sABC == 1) { ENTER(3, -uAC * inv, uAB * inv, V[0], V[1], V[2]); next = -1; }
      else { LEAVE(3, -uAC * inv, uAB * inv); next = 1; }
      uAD = pdot(ray, plk(V[0], V[3])); sAD = dsign(uAD);
      if ((sAD == next) || (sAD == 0)) {
        uDB = pdot(ray, plk(V[3], V[1])); sDB = dsign(uDB);
        if ((sDB == next) || ((sDB == 0) && ((sAD != 0) || (sAB != 0)))) {
          double iv = 1.0 / (uAD + uDB - uAB);
          if (next == 1) ENTER(2, uDB * iv, -uAB * iv, V[1], V[0], V[3]);
          else LEAVE(2, uDB * iv, -uAB * iv);
          DONE();
        }
      }
      uDC = pdot(ray, plk(V[3], V[2])); sDC = dsign(uDC);
      if ((sDC == -next) || ((sDC == 0) && ((sAD != 0) || (sAC != 0)))) {
        double iv = 1.0 / (uAC - uDC - uAD);
        if (next == 1) ENTER(1, uAC * iv, -uDC * iv, V[2], V[3], V[0]);
        else LEAVE(1, uAC * iv, -uDC * iv);
        DONE();
      } else {
        if (sDB == -2) uDB = pdot(ray, plk(V[3], V[1]));
        double iv = 1.0 / (uDC - uBC - uDB);
        if (next == 1) ENTER(0, -uDB * iv, uDC * iv, V[3], V[2], V[1]);
        else LEAVE(0, -uDB * iv, uDC * iv);
        DONE();
      }
    }
  }
  uAD = pdot(ray, plk(V[0], V[3])); sAD = dsign(uAD);
  if ((sAD == -sAB) || (sAB == 0) || (sAD == 0)) {
    uDB = pdot(ray, plk(V[3], V[1])); sDB = dsign(uDB);
    int sBAD = -sAB;
    if (sBAD == 0) { sBAD = sAD; if (sBAD == 0) sBAD = sDB; }
    if ((sBAD != 0) && ((sDB == sBAD) || (sDB == 0))) {
      double inv = 1.0 / (uAD + uDB - uAB);
      if (sBAD == 1) { ENTER(2, uDB * inv, -uAB * inv, V[1], V[0], V[3]); next = -1; }
      else { LEAVE(2, uDB * inv, -uAB * inv); next = 1; }
      uDC = pdot(ray, plk(V[3], V[2])); sDC = dsign(uDC);
      if ((sDC == -next) || ((sDC == 0) && ((sAD != 0) || (sAC != 0)))) {
        double iv = 1.0 / (uAC - uDC - uAD);
        if (next == 1) ENTER(1, uAC * iv, -uDC * iv, V[2], V[3], V[0]);
        else LEAVE(1, uAC * iv, -uDC * iv);
        DONE();
      } else {
        if (sBC == -2) uBC = pdot(ray, plk(V[1], V[2]));
        double iv = 1.0 / (uDC - uBC - uDB);
        if (next == 1) ENTER(0, -uDB * iv, uDC * iv, V[3], V[2], V[1]);
        else LEAVE(0, -uDB * iv, uDC * iv);
        DONE();
      }
    }
  }
  if ((-sAD == sAC) || (sAC == 0) || (sAD == 0)) {
    uDC = pdot(ray, plk(V[3], V[2])); sDC = dsign(uDC);
    int sCDA = sAC;
    if (sCDA == 0) { sCDA = -sAD; if (sCDA == 0) sCDA = -sDC; }
    if ((sCDA != 0) && ((-sDC == sCDA) || (sDC == 0))) {
      double ivCDA = 1.0 / (uAC - uDC - uAD);
      if (sBC == -2) uBC = pdot(ray, plk(V[1], V[2]));
      if (sDB == -2) uDB = pdot(ray, plk(V[3], V[1]));
      double ivDCB = 1.0 / (uDC - uBC - uDB);
      if (sCDA == 1) {
        ENTER(1, uAC * ivCDA, -uDC * ivCDA, V[2], V[3], V[0]);
        LEAVE(0, -uDB * ivDCB, uDC * ivDCB);
      } else {
        LEAVE(1, uAC * ivCDA, -uDC * ivCDA);
        ENTER(0, -uDB * ivDCB, uDC * ivDCB, V[3], V[2], V[1]);
      }
      DONE();
    }
  }
#undef ENTER
#undef LEAVE
#undef DONE
  return false;
}

// --------------------------------------------------------------- sphere
__device__ __forceinline__ bool sphere_isect(float &tio, const float c[3], float radius,
                                             const RayF &r, float prevT,
                                             const float prevN[3], bool self) {
  const float oc[3] = {r.o[0] - c[0], r.o[1] - c[1], r.o[2] - c[2]};
  const float a = dot3(r.d, r.d);
  const float b = 2.0f * dot3(r.d, oc);
  const float cc = dot3(oc, oc) - radius * radius;
  const float disc = (float)((double)(b * b) - (4.0 * (double)a) * (double)cc);
  float t0, t1;
  if (disc < 0.0f) return false;
  if (disc == 0.0f) {
    t0 = t1 = -0.5f * (b / a);
  } else {
    const float ds = sqrtf(disc);
    const float q = (b < 0.0f) ? (-b - ds) * 0.5f : (-b + ds) * 0.5f;
    t0 = q / a;
    t1 = cc / q;
  }
  if (t0 > t1) {
    float tmp = t0;
    t0 = t1;
    t1 = tmp;
  }
  if (t1 < 0.0f) return false;
  if (self) {
    const float t = t1;
    float nrm[3];
#pragma unroll
    for (int k = 0; k < 3; k++) nrm[k] = (r.o[k] + t * r.d[k]) - c[k];
    if ((t < tio) && (t < prevT) && (dot3(nrm, prevN) <= 0.0f)) {
      tio = t;
      return true;
    }
    return false;
  }
  const float t = (t0 < 0.0f) ? t1 : t0;
  if (t < tio) {
    tio = t;
    return true;
  }
  return false;
}

// real3::normalize (render/render_common.h:64-77): length in double.
__device__ __forceinline__ void normalize_ref(float n[3]) {
  const double l2 = (double)(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
  double len = 0.0;
  if (fabs(l2) > 1.0e-30) len = 1.0 / sqrt(l2);
#pragma unroll
  for (int k = 0; k < 3; k++) n[k] = (float)((double)n[k] * len);
}

// --------------------------------------------------------------- kernels
template <int KIND>  // SRT_TRIANGLES or SRT_SPHERES
__global__ void __launch_bounds__(128)
trace_node2_kernel(const Node2 *__restrict__ nodes, const float4 *__restrict__ prims,
                   const uint32_t *__restrict__ sidx, const srt_ray *__restrict__ rays,
                   size_t n, srt_hit *__restrict__ hits,
                   const SceneInfo *__restrict__ scene,
                   const float *__restrict__ prev_normals, float *__restrict__ normal_out,
                   unsigned long long *__restrict__ stats, uint32_t max_iter,
                   uint32_t *__restrict__ err) {
  uint32_t n_branch = 0, n_leaf = 0, n_prim = 0;
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t prev_prim;
  float prev_t;
  const RayF r = load_ray(rays, i, prev_prim, prev_t);
  const float keps = scene->keps;
  float pn[3] = {0.0f, 0.0f, 0.0f};
  if (KIND == SRT_SPHERES && prev_normals && prev_prim != kNone) {
    pn[0] = prev_normals[3 * i];
    pn[1] = prev_normals[3 * i + 1];
    pn[2] = prev_normals[3 * i + 2];
  }
  float best_t = FLT_MAX, best_u = 0.0f, best_v = 0.0f;
  uint32_t best_prim = kNone, best_j = kNone;
  uint2 stk[kStack];
  int sp = 0;
  stk[0] = make_uint2(0u, 0u);
  uint32_t it = 0;
  while (sp >= 0) {
    if (++it > max_iter) {
      atomicOr(err, kErrIter);
      break;
    }
    const uint2 e = stk[sp--];
    if (e.y == 0) {
      n_branch++;
      const float4 *np = reinterpret_cast<const float4 *>(nodes + e.x);
      const float4 a = __ldg(np), b = __ldg(np + 1), c = __ldg(np + 2);
      const uint4 d = __ldg(reinterpret_cast<const uint4 *>(np + 3));
      const float hitT = best_t;
      bool h[2];
      h[0] = ray_aabb<true>(hitT, a.x, a.y, a.z, a.w, b.x, b.y, r);
      h[1] = ray_aabb<true>(hitT, b.z, b.w, c.x, c.y, c.z, c.w, r);
      if (h[0] || h[1]) {
        const int axis = (int)(d.z >> 30);
        const int nearc = r.sgn[axis], farc = 1 - nearc;
        const uint2 ce[2] = {make_uint2(d.x, d.z & kCountMask),
                             make_uint2(d.y, d.w & kCountMask)};
        if (sp + 2 >= kStack) {
          atomicOr(err, kErrStack);
          break;
        }
        if (h[farc]) stk[++sp] = ce[farc];
        if (h[nearc]) stk[++sp] = ce[nearc];
      }
    } else {
      n_leaf++;
      n_prim += e.y;
      float t = best_t;
      for (uint32_t j = e.x; j < e.x + e.y; j++) {
        if (KIND == SRT_TRIANGLES) {
          const float4 q0 = __ldg(&prims[3 * (size_t)j]);
          const uint32_t f = __float_as_uint(q0.w);
          if (f == prev_prim) continue;
          const float4 q1 = __ldg(&prims[3 * (size_t)j + 1]);
          const float4 q2 = __ldg(&prims[3 * (size_t)j + 2]);
          const float p0[3] = {q0.x, q0.y, q0.z};
          const float p1[3] = {q1.x, q1.y, q1.z};
          const float p2[3] = {q2.x, q2.y, q2.z};
          float u, v;
          if (tri_isect(t, u, v, p0, p1, p2, r, keps)) {
            best_t = t;
            best_u = u;
            best_v = v;
            best_prim = f;
            best_j = j;
          }
        } else {
          const float4 s = __ldg(&prims[j]);
          const uint32_t f = __ldg(&sidx[j]);
          const float c[3] = {s.x, s.y, s.z};
          if (sphere_isect(t, c, s.w, r, prev_t, pn, prev_prim == f)) {
            best_t = t;
            best_prim = f;
            best_j = j;
          }
        }
      }
    }
  }
  if (stats) {
    atomicAdd(&stats[0], (unsigned long long)n_branch);
    atomicAdd(&stats[1], (unsigned long long)n_leaf);
    atomicAdd(&stats[2], (unsigned long long)n_prim);
  }
  srt_hit h;
  if (best_t < FLT_MAX) {
    h.t = best_t;
    h.u = best_u;
    h.v = best_v;
    h.prim = best_prim;
  } else {
    h.t = FLT_MAX;
    h.u = 0.0f;
    h.v = 0.0f;
    h.prim = kNone;
  }
  reinterpret_cast<float4 *>(hits)[i] =
      make_float4(h.t, h.u, h.v, __uint_as_float(h.prim));
  if (normal_out) {
    float nn[3] = {0.0f, 0.0f, 0.0f};
    if (best_j != kNone) {
      if (KIND == SRT_TRIANGLES) {
        const float4 q0 = prims[3 * (size_t)best_j];
        const float4 q1 = prims[3 * (size_t)best_j + 1];
        const float4 q2 = prims[3 * (size_t)best_j + 2];
        const float e1[3] = {q1.x - q0.x, q1.y - q0.y, q1.z - q0.z};
        const float e2[3] = {q2.x - q0.x, q2.y - q0.y, q2.z - q0.z};
        cross3(e1, e2, nn);
        normalize_ref(nn);
      } else {
        const float4 s = prims[best_j];
        const float c[3] = {s.x, s.y, s.z};
        // position = org + t * dir; vnormalize(position - centre)
#pragma unroll
        for (int k = 0; k < 3; k++) nn[k] = (r.o[k] + best_t * r.d[k]) - c[k];
        const float len = sqrtf(dot3(nn, nn));
        if (len > FLT_EPSILON * 16) {
          const float il = __frcp_rn(len);
#pragma unroll
          for (int k = 0; k < 3; k++) nn[k] *= il;
        }
      }
    }
    normal_out[3 * i] = nn[0];
    normal_out[3 * i + 1] = nn[1];
    normal_out[3 * i + 2] = nn[2];
  }
}

__global__ void __launch_bounds__(128)
trace_tet_kernel(const NodeT *__restrict__ nodes, const float4 *__restrict__ prims,
                 const uint32_t *__restrict__ sidx, const srt_ray *__restrict__ rays,
                 size_t n, srt_hit *__restrict__ hits, uint32_t *__restrict__ subface,
                 const uint32_t *__restrict__ faces, const float *__restrict__ vscalar,
                 float *__restrict__ scalar_out, unsigned long long *__restrict__ stats,
                 uint32_t max_iter, uint32_t *__restrict__ err) {
  uint32_t n_branch = 0, n_leaf = 0, n_prim = 0;
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t prev_prim;
  float prev_t;
  const RayF r = load_ray(rays, i, prev_prim, prev_t);
  const D3 o = {r.o[0], r.o[1], r.o[2]};
  const D3 dd = {r.d[0], r.d[1], r.d[2]};
  float best_t = FLT_MAX, best_u = 0.0f, best_v = 0.0f;
  uint32_t best_prim = kNone, best_sub = 0;
  double best_e1 = 0.0, best_e2 = 0.0;
  uint32_t stk[kStack];
  int sp = 0;
  stk[0] = 0u;
  uint32_t it = 0;
  while (sp >= 0) {
    if (++it > max_iter) {
      atomicOr(err, kErrIter);
      break;
    }
    const uint32_t ni = stk[sp--];
    const float4 *np = reinterpret_cast<const float4 *>(nodes + ni);
    const float4 a = __ldg(np), b = __ldg(np + 1);
    const uint32_t meta = __float_as_uint(a.w), ref = __float_as_uint(b.w);
    const bool hit = ray_aabb<false>(best_t, a.x, a.y, a.z, b.x, b.y, b.z, r);
    n_branch++;  // every popped node is box-tested (the reference's numNodeTraversals
                 // counts the hit branches only)
    if (!(meta & kLeafBit)) {
      if (hit) {
        const int nearc = r.sgn[meta & 3u], farc = 1 - nearc;
        if (sp + 2 >= kStack) {
          atomicOr(err, kErrStack);
          break;
        }
        stk[++sp] = ref + (uint32_t)farc;
        stk[++sp] = ref + (uint32_t)nearc;
      }
    } else if (hit) {
      const uint32_t cnt = meta & kCountMask;
      n_leaf++;
      n_prim += cnt;
      float t = best_t;
      for (uint32_t j = ref; j < ref + cnt; j++) {
        const uint32_t f = __ldg(&sidx[j]);
        if (f == prev_prim) continue;
        const float4 q0 = __ldg(&prims[3 * (size_t)j]);
        const float4 q1 = __ldg(&prims[3 * (size_t)j + 1]);
        const float4 q2 = __ldg(&prims[3 * (size_t)j + 2]);
        const D3 V[4] = {{q0.x, q0.y, q0.z}, {q0.w, q1.x, q1.y},
                         {q1.z, q1.w, q2.x}, {q2.y, q2.z, q2.w}};
        int ef;
        double ue1, ue2, ul1, te;
        if (ray_tet(o, dd, V, ef, ue1, ue2, ul1, te)) {
          if ((te >= 0.0) && (te < (double)t)) {
            best_t = (float)te;
            best_u = (float)ue1;
            best_v = (float)ul1;  // the reference's isect.v receives uLeave1
            best_prim = f;
            best_sub = (uint32_t)ef;
            best_e1 = ue1;
            best_e2 = ue2;
            t = (float)te;
          }
        }
      }
    }
  }
  if (stats) {
    atomicAdd(&stats[0], (unsigned long long)n_branch);
    atomicAdd(&stats[1], (unsigned long long)n_leaf);
    atomicAdd(&stats[2], (unsigned long long)n_prim);
  }
  const bool any = best_t < FLT_MAX;
  reinterpret_cast<float4 *>(hits)[i] =
      make_float4(any ? best_t : FLT_MAX, any ? best_u : 0.0f, any ? best_v : 0.0f,
                  __uint_as_float(any ? best_prim : kNone));
  if (subface) subface[i] = any ? best_sub : 0u;
  if (scalar_out) {
    float s = 0.0f;
    if (any && faces && vscalar) {
      // entering face vertex order (A, B, C) per face id, as the Pluecker
      // test's barycentric points are formed
      const int fA[4] = {3, 2, 1, 0}, fB[4] = {2, 3, 0, 1}, fC[4] = {1, 0, 3, 2};
      const uint32_t *tv = faces + 4 * (size_t)best_prim;
      const double sa = vscalar[tv[fA[best_sub]]], sb = vscalar[tv[fB[best_sub]]],
                   sc = vscalar[tv[fC[best_sub]]];
      s = (float)((1.0 - best_e1 - best_e2) * sa + best_e1 * sb + best_e2 * sc);
    }
    scalar_out[i] = s;
  }
}

}  // namespace

srt_status launch_trace(srt_accel *a, const srt_ray *rays, size_t n, srt_hit *hits,
                        const float *prev_normals, uint32_t *subface,
                        const float *vscalar, float *scalar_out, float *normal_out,
                        unsigned long long *stats) {
  if (n == 0) return SRT_OK;
  srt_ctx *ctx = a->ctx;
  const int block = 128;
  const unsigned grid = (unsigned)((n + block - 1) / block);
  // each node and leaf is visited at most once per ray
  const uint32_t max_iter = (uint32_t)std::min<size_t>(4 * a->n + 64, 0xfffffff0u);
  const SceneInfo *scene = a->scene.as<SceneInfo>();
  switch (a->kind) {
    case SRT_TRIANGLES:
      trace_node2_kernel<SRT_TRIANGLES><<<grid, block, 0, ctx->stream>>>(
          a->nodes.as<Node2>(), a->prims.as<float4>(), a->indices.as<uint32_t>(), rays, n,
          hits, scene, nullptr, normal_out, stats, max_iter, ctx->d_err);
      break;
    case SRT_SPHERES:
      trace_node2_kernel<SRT_SPHERES><<<grid, block, 0, ctx->stream>>>(
          a->nodes.as<Node2>(), a->prims.as<float4>(), a->indices.as<uint32_t>(), rays, n,
          hits, scene, prev_normals, normal_out, stats, max_iter, ctx->d_err);
      break;
    case SRT_TETRAHEDRA:
      trace_tet_kernel<<<grid, block, 0, ctx->stream>>>(
          a->nodes.as<NodeT>(), a->prims.as<float4>(), a->indices.as<uint32_t>(), rays, n,
          hits, subface, a->src_faces, vscalar, scalar_out, stats, max_iter, ctx->d_err);
      break;
  }
  ctx->launches++;
  return cuda_status(cudaGetLastError(), "trace");
}

}  // namespace srt
