// srt_trace.cu -- closest-hit traversal, one ray per thread.
//
// The hits are exactly the reference's Traverse() results, tie-breaking
// included:
//   triangles  TriangleAccel::Traverse  render/render_accel_triangle.cc:2511-2669
//              IntersectRayAABB :1815-1861, TriangleIsect :1887-1938,
//              TestLeafNode :1994-2437, BuildIntersection :2439-2507
//   tetrahedra TetraAccel::Traverse     render/render_accel_tetra.cc:2200-2289
//              IntersectRayAABB :1934-1978, TestLeafNode :1980-2122,
//              RayTetraPluecker :243-567 (FP64), ComputeParametricDist :123-139
//   spheres    ParticleAccel::Traverse  render/render_accel_particle.cc:3053-3218
//              SphereIsect :2423-2512, BuildIntersection :2968-3049
//
// The reference walks depth first, near child = dirSign[axis] with its
// axis taken from (clz(code) - 2) % 3, and prunes boxes entered after its
// current hit.  Its answer is the sequential scan, in that order, of every
// primitive the ray hits, provided no primitive reports a distance before
// its own leaf box's entry (then no pruning ever hides an acceptable
// primitive).  The default walk therefore goes front to back (pass 1),
// finds m, the smallest hit distance, and counts the primitives at m
// (tetrahedra: within 8 float steps, since the reference compares a double
// distance with its float-rounded current one).  One such primitive is the
// answer; several -- an exact tie -- are ordered by the reference-order walk
// restricted to boxes entered before m.  A primitive hit before its leaf
// box's entry sends the ray through the reference's own walk.  The
// single-pass kernels (SRT_TRACE_SINGLE_PASS) run that walk for every ray.
//
// Leaves are folded into their parent's child slot for triangles/spheres;
// a hit leaf is pushed as a (first primitive, count) entry, which visits
// leaves in exactly the reference's order.
#include <mutex>
#include <type_traits>

#include "srt_internal.cuh"
#include "srt_walks.cuh"

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
// The ray's side of the Pluecker tests, formed once per ray: its Pluecker
// coordinates (through orig and orig + dir) and, for ComputeParametricDist,
// the first axis with a nonzero direction, the origin's coordinate on it and
// the direction's reciprocal there.
struct TetRay {
  Plk ray;
  double oa, iva;
  float sel[3];  // one-hot selector of that axis
};

__device__ __forceinline__ TetRay tet_ray(D3 orig, D3 dir) {
  TetRay t;
  t.ray = plk(orig, dadd(orig, dir));
  const int ax = dir.x != 0.0 ? 0 : (dir.y != 0.0 ? 1 : 2);
  const double da = ax == 0 ? dir.x : (ax == 1 ? dir.y : dir.z);
  t.oa = ax == 0 ? orig.x : (ax == 1 ? orig.y : orig.z);
  t.iva = 1.0 / da;
  t.sel[0] = ax == 0 ? 1.0f : 0.0f;
  t.sel[1] = ax == 1 ? 1.0f : 0.0f;
  t.sel[2] = ax == 2 ? 1.0f : 0.0f;
  return t;
}

// A tetrahedron's vertices as stored (float), widened at use.
// The corners of a tetrahedron of double-precision positions (the same
// interface; the one-hot axis product of doubles is exact as well).
struct TetVD {
  double v[12];
  __device__ __forceinline__ D3 operator[](int k) const { return {v[3 * k], v[3 * k + 1], v[3 * k + 2]}; }
  __device__ __forceinline__ double axis(int k, const float (&sel)[3]) const {
    return (v[3 * k] * (double)sel[0] + v[3 * k + 1] * (double)sel[1]) + v[3 * k + 2] * (double)sel[2];
  }
};

struct TetV {
  float v[12];
  __device__ __forceinline__ D3 operator[](int k) const {
    return {(double)v[3 * k], (double)v[3 * k + 1], (double)v[3 * k + 2]};
  }
  // coordinate of vertex k on the axis selected one-hot by sel (exact: the
  // other two terms are zeros)
  __device__ __forceinline__ double axis(int k, const float (&sel)[3]) const {
    return (double)((v[3 * k] * sel[0] + v[3 * k + 1] * sel[1]) + v[3 * k + 2] * sel[2]);
  }
};

// Entering face, its barycentrics (ue1, ue2), the leaving face's first
// barycentric ul1 and tEnter, as RayTetraPluecker decides them
// (render/render_accel_tetra.cc:243-567), written without divergent
// arithmetic: all six edge products are formed up front (the reference forms
// those its branches reach; each is the same value whenever formed), the
// branch structure runs on their signs alone to pick the entering and
// leaving faces, and then each face's barycentrics come from its own
// expression -- face f: inv = 1 / ((P + Q) - R), (a1, a2) = (X * inv, Y * inv):
//   f = 3: P, Q, R = uAB, uBC, uAC   X, Y = -uAC,  uAB   points (A, B, C)
//   f = 2:           uAD, uDB, uAB         uDB, -uAB          (B, A, D)
//   f = 1:           uAC, -uDC, uAD        uAC, -uDC          (C, D, A)
//   f = 0:           uDC, -uBC, uDB       -uDB,  uDC          (D, C, B)
// Only the entering point's coordinate on the ray's first nonzero axis is
// formed, (pe - o) * (1 / d) there as ComputeParametricDist does, the point
// being the reference's ((1 - a - b) * P0 + a * P1) + b * P2.
// ul1 (the leaving face's barycentric, only a kept hit reports it) is formed
// only when te < take_below.
template <class TV>
__device__ __forceinline__ bool ray_tet(const TetRay &R, const TV &V, double take_below,
                                        int &ef, double &ue1, double &ue2, double &ul1,
                                        double &te) {
  const Plk &ray = R.ray;
  const double uAB = pdot(ray, plk(V[0], V[1])), uAC = pdot(ray, plk(V[0], V[2]));
  const double uAD = pdot(ray, plk(V[0], V[3])), uBC = pdot(ray, plk(V[1], V[2]));
  const double uDB = pdot(ray, plk(V[3], V[1])), uDC = pdot(ray, plk(V[3], V[2]));
  const int sAB = dsign(uAB), sAC = dsign(uAC), sAD = dsign(uAD), sBC = dsign(uBC),
            sDB = dsign(uDB), sDC = dsign(uDC);
  int enter = -1, leave = -1;
  if ((sAC == -sAB) || (sAC == 0) || (sAB == 0)) {
    int sABC = sAB;
    if (sABC == 0) { sABC = -sAC; if (sABC == 0) sABC = sBC; }
    if ((sABC != 0) && ((sBC == sABC) || (sBC == 0))) {
      const int next = sABC == 1 ? -1 : 1;
      int f2;
      if (((sAD == next) || (sAD == 0)) &&
          ((sDB == next) || ((sDB == 0) && ((sAD != 0) || (sAB != 0)))))
        f2 = 2;
      else if ((sDC == -next) || ((sDC == 0) && ((sAD != 0) || (sAC != 0))))
        f2 = 1;
      else
        f2 = 0;
      enter = next == 1 ? f2 : 3;
      leave = next == 1 ? 3 : f2;
    }
  }
  if (enter < 0 && ((sAD == -sAB) || (sAB == 0) || (sAD == 0))) {
    int sBAD = -sAB;
    if (sBAD == 0) { sBAD = sAD; if (sBAD == 0) sBAD = sDB; }
    if ((sBAD != 0) && ((sDB == sBAD) || (sDB == 0))) {
      const int next = sBAD == 1 ? -1 : 1;
      const int f2 = ((sDC == -next) || ((sDC == 0) && ((sAD != 0) || (sAC != 0)))) ? 1 : 0;
      enter = next == 1 ? f2 : 2;
      leave = next == 1 ? 2 : f2;
    }
  }
  if (enter < 0 && ((-sAD == sAC) || (sAC == 0) || (sAD == 0))) {
    int sCDA = sAC;
    if (sCDA == 0) { sCDA = -sAD; if (sCDA == 0) sCDA = -sDC; }
    if ((sCDA != 0) && ((-sDC == sCDA) || (sDC == 0))) {
      enter = sCDA == 1 ? 1 : 0;
      leave = sCDA == 1 ? 0 : 1;
    }
  }
  if (enter < 0) return false;
  // face terms, selected by face id
  auto P = [&](int f) { return f == 3 ? uAB : f == 2 ? uAD : f == 1 ? uAC : uDC; };
  auto Q = [&](int f) { return f == 3 ? uBC : f == 2 ? uDB : f == 1 ? -uDC : -uBC; };
  auto Rr = [&](int f) { return f == 3 ? uAC : f == 2 ? uAB : f == 1 ? uAD : uDB; };
  auto X = [&](int f) { return f == 3 ? -uAC : f == 2 ? uDB : f == 1 ? uAC : -uDB; };
  auto Y = [&](int f) { return f == 3 ? uAB : f == 2 ? -uAB : f == 1 ? -uDC : uDC; };
  const double inv_e = 1.0 / ((P(enter) + Q(enter)) - Rr(enter));
  const double a = X(enter) * inv_e, b = Y(enter) * inv_e;
  // entering point's vertices (3 - f, f ^ 2, f ^ 1), coordinates on the axis
  const double c0 = V.axis(0, R.sel), c1 = V.axis(1, R.sel), c2 = V.axis(2, R.sel),
               c3 = V.axis(3, R.sel);
  auto C = [&](int k) { return k == 0 ? c0 : k == 1 ? c1 : k == 2 ? c2 : c3; };
  const double p0 = C(3 - enter), p1 = C(enter ^ 2), p2 = C(enter ^ 1);
  const double epa = (p0 * (1 - a - b) + p1 * a) + p2 * b;
  te = (epa - R.oa) * R.iva;
  ef = enter;
  ue1 = a;
  ue2 = b;
  ul1 = 0.0;
  if (te < take_below) ul1 = X(leave) * (1.0 / ((P(leave) + Q(leave)) - Rr(leave)));
  return true;
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


// IntersectRayAABB that also reports the box entry distance.
template <bool CLAMP>
__device__ __forceinline__ bool ray_aabb_t(float maxT, float lx, float ly, float lz,
                                           float hx, float hy, float hz, const RayF &r,
                                           float &tmin_out) {
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
  tmin_out = tmin;
  if (CLAMP) {
    tmax = (maxT < tmax) ? maxT : tmax;
    return (tmax > 0.0f) && (tmin <= tmax);
  }
  return (tmax > 0.0f) && (tmin <= tmax) && (tmin <= maxT);
}

// --------------------------------------------------------------- walks
// Tree walks shared by the kernels.  Every walk is "while-while": a lane
// stops at its next leaf and the leaf's primitives are tested when all
// lanes of the warp hold one, so the primitive tests run on full warps.

// Relative pruning margins above the smallest hit distance m: boxes entered
// before m * (1 + rel) are walked.  Float triangle and sphere distances can
// err by ~1e-4 relative (ill-conditioned quadratic, grazing hits), so they
// get 2^-8; the FP64 tetrahedron distance is exact to ~1e-15 and the leaf
// padding is 16 ulp(1), so 2^-16 suffices.
constexpr float kRelTri = 3.90625e-3f;          // 2^-8
constexpr float kRelTet = 1.52587890625e-5f;    // 2^-16

__device__ __forceinline__ float bound_rel(float m, float rel) {
  return (m < FLT_MAX) ? m + fabsf(m) * rel + 1e-30f : FLT_MAX;
}

// A hit distance below the entry distance of its own leaf box (the same
// float the reference's box test computes; NaN counts as below).  Only a
// primitive still among the candidates at the smallest distance m can then
// be hidden by the reference's pruning: any box around a primitive with
// t >= entry is entered at or before t, so a box can only be pruned for a
// running distance below that primitive's own.  Such rays take the
// reference's walk.
__device__ __forceinline__ bool below_entry(double t, float entry) {
  return !(t >= (double)entry);
}

struct Work {
  uint32_t branch = 0, leaf = 0, prim = 0, it = 0;
  bool fail = false;
};

struct Best {
  float t = FLT_MAX, u = 0.0f, v = 0.0f;
  uint32_t prim = kNone, j = kNone;
  uint32_t sub = 0;
  double e1 = 0.0, e2 = 0.0;
};

// Per-ray context of the two-child walks.
struct Ctx2 {
  RayF r;
  uint32_t prev_prim;
  float prev_t;
  float pn[3];
  float keps;
};

// One primitive of a two-child kind as loaded from the primitive cache
// (a triangle's three corners with its id, or a sphere and its id), so that
// a leaf walk can load the next primitive while it tests this one.
template <int KIND>
struct Prim2 {
  float4 q0, q1, q2;
  uint32_t f;
  __device__ __forceinline__ void load(const float4 *__restrict__ prims,
                                       const uint32_t *__restrict__ sidx, uint32_t j) {
    if (KIND == SRT_TRIANGLES) {
      q0 = __ldg(&prims[3 * (size_t)j]);
      q1 = __ldg(&prims[3 * (size_t)j + 1]);
      q2 = __ldg(&prims[3 * (size_t)j + 2]);
      f = __float_as_uint(q0.w);
    } else {
      q0 = __ldg(&prims[j]);
      f = __ldg(&sidx[j]);
    }
  }
  // Hit distance below tio (t, u, v), false on a miss.
  __device__ __forceinline__ bool test(const Ctx2 &c, float tio, float &t, float &u,
                                       float &v) const {
    if (KIND == SRT_TRIANGLES) {
      if (f == c.prev_prim) return false;
      const float p0[3] = {q0.x, q0.y, q0.z}, p1[3] = {q1.x, q1.y, q1.z},
                  p2[3] = {q2.x, q2.y, q2.z};
      t = tio;
      return tri_isect(t, u, v, p0, p1, p2, c.r, c.keps);
    } else {
      const float c3[3] = {q0.x, q0.y, q0.z};
      t = tio;
      u = v = 0.0f;
      return sphere_isect(t, c3, q0.w, c.r, c.prev_t, c.pn, c.prev_prim == f);
    }
  }
};

// Hit distance of sorted primitive j (two-child kinds), FLT_MAX on a miss.
template <int KIND>
__device__ __forceinline__ bool cand2(const float4 *__restrict__ prims,
                                      const uint32_t *__restrict__ sidx, uint32_t j,
                                      const Ctx2 &c, float tio, float &t, float &u, float &v,
                                      uint32_t &f) {
  Prim2<KIND> P;
  P.load(prims, sidx, j);
  f = P.f;
  return P.test(c, tio, t, u, v);
}

// The reference's Traverse, step for step (render/render_accel_triangle.cc:2511,
// render/render_accel_particle.cc:3053), with the running distance starting
// at t0 (FLT_MAX: the reference's own walk; b.prim stays kNone when nothing
// is accepted below t0).
template <int KIND>
__device__ void ref_walk2(const Node2 *__restrict__ nodes, const float4 *__restrict__ prims,
                          const uint32_t *__restrict__ sidx, const Ctx2 &c, Best &b,
                          Work &w, uint32_t max_iter, uint32_t root = 0,
                          float t0 = FLT_MAX) {
  b = Best();
  b.t = t0;
  uint2 stk[kStack];
  int sp = 0;
  stk[0] = make_uint2(root, 0u);
  while (true) {
    uint2 leaf = make_uint2(0u, 0u);
    while (sp >= 0) {
      if (++w.it > max_iter) { w.fail = true; sp = -1; break; }
      const uint2 e = stk[sp--];
      if (e.y != 0) { leaf = e; break; }
      w.branch++;
      const float4 *np = reinterpret_cast<const float4 *>(nodes + e.x);
      const float4 a = __ldg(np), bb = __ldg(np + 1), cc = __ldg(np + 2);
      const uint4 d = __ldg(reinterpret_cast<const uint4 *>(np + 3));
      bool h[2];
      h[0] = ray_aabb<true>(b.t, a.x, a.y, a.z, a.w, bb.x, bb.y, c.r);
      h[1] = ray_aabb<true>(b.t, bb.z, bb.w, cc.x, cc.y, cc.z, cc.w, c.r);
      if (h[0] || h[1]) {
        const int nearc = c.r.sgn[d.z >> 30], farc = 1 - nearc;
        const uint2 ce[2] = {make_uint2(d.x, d.z & kCountMask),
                             make_uint2(d.y, d.w & kCountMask)};
        if (sp + 2 >= kStack) { w.fail = true; sp = -1; break; }
        if (h[farc]) stk[++sp] = ce[farc];
        if (h[nearc]) stk[++sp] = ce[nearc];
      }
    }
    if (leaf.y == 0) break;
    w.leaf++;
    w.prim += leaf.y;
    float t = b.t;
    for (uint32_t j = leaf.x; j < leaf.x + leaf.y; j++) {
      float u, v;
      uint32_t f;
      if (cand2<KIND>(prims, sidx, j, c, t, t, u, v, f)) {
        b.t = t; b.u = u; b.v = v; b.prim = f; b.j = j;
      }
    }
  }
  if (b.prim == kNone) b.t = FLT_MAX;
}

// The fallback for a ray whose candidate at m lies below its leaf box's
// entry: the reference's walk started from pass 1's pruning bound T.  It
// returns the reference's primitive: that primitive and every primitive
// that can prune its boxes lie below T by more than the float error of a
// distance, so a running distance at or above T (which the full walk may
// hold on the way) prunes none of them.  Nothing accepted below T: the full
// walk decides.
template <int KIND>
__device__ __forceinline__ void ref_walk2_from(const Node2 *__restrict__ nodes,
                                               const float4 *__restrict__ prims,
                                               const uint32_t *__restrict__ sidx,
                                               const Ctx2 &c, Best &b, Work &w,
                                               uint32_t max_iter, float m, uint32_t root = 0) {
  ref_walk2<KIND>(nodes, prims, sidx, c, b, w, max_iter, root, bound_rel(m, kRelTri));
  if (b.prim != kNone || w.fail) return;
  w.it = 0;
  ref_walk2<KIND>(nodes, prims, sidx, c, b, w, max_iter, root);
}

// Reference order through boxes entered before `bnd`, accepting from `t0`
// on (the candidates at m).
template <int KIND>
__device__ void window_walk2(const Node2 *__restrict__ nodes,
                             const float4 *__restrict__ prims,
                             const uint32_t *__restrict__ sidx, const Ctx2 &c, float bnd,
                             float t0, Best &b, Work &w, uint32_t max_iter,
                             uint32_t root = 0) {
  b = Best();
  float t = t0;
  uint2 stk[kStack];
  int sp = 0;
  stk[0] = make_uint2(root, 0u);
  while (true) {
    uint2 leaf = make_uint2(0u, 0u);
    while (sp >= 0) {
      if (++w.it > max_iter) { w.fail = true; sp = -1; break; }
      const uint2 e = stk[sp--];
      if (e.y != 0) { leaf = e; break; }
      w.branch++;
      const float4 *np = reinterpret_cast<const float4 *>(nodes + e.x);
      const float4 a = __ldg(np), bb = __ldg(np + 1), cc = __ldg(np + 2);
      const uint4 d = __ldg(reinterpret_cast<const uint4 *>(np + 3));
      bool h[2];
      h[0] = ray_aabb<true>(bnd, a.x, a.y, a.z, a.w, bb.x, bb.y, c.r);
      h[1] = ray_aabb<true>(bnd, bb.z, bb.w, cc.x, cc.y, cc.z, cc.w, c.r);
      if (h[0] || h[1]) {
        const int nearc = c.r.sgn[d.z >> 30], farc = 1 - nearc;
        const uint2 ce[2] = {make_uint2(d.x, d.z & kCountMask),
                             make_uint2(d.y, d.w & kCountMask)};
        if (sp + 2 >= kStack) { w.fail = true; sp = -1; break; }
        if (h[farc]) stk[++sp] = ce[farc];
        if (h[nearc]) stk[++sp] = ce[nearc];
      }
    }
    if (leaf.y == 0) break;
    w.leaf++;
    w.prim += leaf.y;
    for (uint32_t j = leaf.x; j < leaf.x + leaf.y; j++) {
      float u, v;
      uint32_t f;
      if (cand2<KIND>(prims, sidx, j, c, t, t, u, v, f)) {
        b.t = t; b.u = u; b.v = v; b.prim = f; b.j = j;
      }
    }
  }
}

// --------------------------------------------------------------- kernels
// Pass 1 (front to back) runs in the main kernels and settles the common
// case: no hit, or exactly one primitive at the smallest distance m.  Rays
// with an exact tie at m, or with a primitive reported before its own leaf
// box's entry, are appended to a deferred list; a second kernel resolves
// them with the reference-order walk restricted to boxes entered before m
// (ties) or with the reference's full walk.  Keeping those walks out of the
// main kernels keeps their register and stack footprint small.


// BuildIntersection's (u, v) of a sphere hit (render/render_accel_particle.cc:
// 2968-3047): position = org + t * dir, n = vnormalize(position - centre),
// then the spherical coordinates of n.  Also returns n.
__device__ __forceinline__ void sphere_hit_uv(const RayF &r, const float4 *__restrict__ prims,
                                              Best &b, float nn[3]) {
  const float4 s = prims[b.j];
  const float c3[3] = {s.x, s.y, s.z};
#pragma unroll
  for (int k = 0; k < 3; k++) nn[k] = (r.o[k] + b.t * r.d[k]) - c3[k];
  const float len = sqrtf(dot3(nn, nn));
  if (len > FLT_EPSILON * 16) {
    const float il = __frcp_rn(len);
#pragma unroll
    for (int k = 0; k < 3; k++) nn[k] *= il;
  }
  sphere_uv(nn, b.u, b.v);
}

template <int KIND>
__device__ __forceinline__ void store_node2(size_t i, const Best &b, const Ctx2 &c,
                                            const float4 *__restrict__ prims,
                                            srt_hit *__restrict__ hits,
                                            float *__restrict__ normal_out) {
  const bool any = b.t < FLT_MAX && b.prim != kNone;
  float nn[3] = {0.0f, 0.0f, 0.0f};
  float hu = any ? b.u : 0.0f, hv = any ? b.v : 0.0f;
  if (KIND == SRT_SPHERES && any) {
    // the spherical (u, v) replace the hit's u, v, as in the reference
    Best bs = b;
    sphere_hit_uv(c.r, prims, bs, nn);
    hu = bs.u;
    hv = bs.v;
  }
  reinterpret_cast<float4 *>(hits)[i] =
      make_float4(any ? b.t : FLT_MAX, hu, hv, __uint_as_float(any ? b.prim : kNone));
  if (!normal_out) return;
  if (any) {
    if (KIND == SRT_TRIANGLES) {
      const float4 q0 = prims[3 * (size_t)b.j];
      const float4 q1 = prims[3 * (size_t)b.j + 1];
      const float4 q2 = prims[3 * (size_t)b.j + 2];
      const float e1[3] = {q1.x - q0.x, q1.y - q0.y, q1.z - q0.z};
      const float e2[3] = {q2.x - q0.x, q2.y - q0.y, q2.z - q0.z};
      cross3(e1, e2, nn);
      normalize_ref(nn);
    }
  }
  normal_out[3 * i] = nn[0];
  normal_out[3 * i + 1] = nn[1];
  normal_out[3 * i + 2] = nn[2];
}

// Work counters of the rays the active lanes finished, merged per warp
// before the atomics (per-ray atomics on four addresses serialise in L2).
__device__ __forceinline__ void add_stats(unsigned long long *stats, const Work &w,
                                          uint32_t full) {
  if (!stats) return;
  const unsigned m = __activemask();
  const int leader = __ffs(m) - 1;
  const uint32_t c[4] = {w.branch, w.leaf, w.prim, full ? 1u : 0u};
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const uint32_t s = __reduce_add_sync(m, c[k]);
    if ((int)(threadIdx.x & 31u) == leader && s) atomicAdd(&stats[k], (unsigned long long)s);
  }
}

template <int KIND>
__device__ __forceinline__ Ctx2 make_ctx2(const srt_ray *__restrict__ rays, size_t i,
                                          const SceneInfo *__restrict__ scene,
                                          const float *__restrict__ prev_normals) {
  Ctx2 c;
  c.r = load_ray(rays, i, c.prev_prim, c.prev_t);
  c.keps = scene->keps;
  c.pn[0] = c.pn[1] = c.pn[2] = 0.0f;
  if (KIND == SRT_SPHERES && prev_normals && c.prev_prim != kNone) {
    c.pn[0] = prev_normals[3 * i];
    c.pn[1] = prev_normals[3 * i + 1];
    c.pn[2] = prev_normals[3 * i + 2];
  }
  return c;
}

// Stacks of the front-to-back walks, entries (child entry, box entry
// distance).  LocalStack: a per-thread array.  SharedStack: the first
// kShDepth entries of each thread in shared memory, entry k of thread t at
// [k][t] so that the lanes of a warp fall on 32 different banks whatever
// their depths, deeper entries in a per-thread array (a front-to-back walk
// holds at most one entry per tree level; the trees of the scenes here are
// 19 to 21 levels deep, so the array is seldom touched).
constexpr int kShDepth = 16;

template <int D>
struct LocalStackN {
  static constexpr int kDepth = D;
  uint2 e[D];
  float t[D];
  __device__ __forceinline__ void put(int k, uint2 v, float d) {
    e[k] = v;
    t[k] = d;
  }
  __device__ __forceinline__ uint2 get(int k, float &d) const {
    d = t[k];
    return e[k];
  }
};

using LocalStack = LocalStackN<kStack>;

template <int NT>
struct SharedStack {
  static constexpr int kDepth = kStack;
  uint2 (*se)[NT];
  float (*st)[NT];
  uint2 e[kStack - kShDepth];
  float t[kStack - kShDepth];
  __device__ __forceinline__ SharedStack(uint2 (*se_)[NT], float (*st_)[NT])
      : se(se_), st(st_) {}
  __device__ __forceinline__ void put(int k, uint2 v, float d) {
    if (k < kShDepth) {
      se[k][threadIdx.x] = v;
      st[k][threadIdx.x] = d;
    } else {
      e[k - kShDepth] = v;
      t[k - kShDepth] = d;
    }
  }
  __device__ __forceinline__ uint2 get(int k, float &d) const {
    if (k < kShDepth) {
      d = st[k][threadIdx.x];
      return se[k][threadIdx.x];
    }
    d = t[k - kShDepth];
    return e[k - kShDepth];
  }
};

// Shared-memory columns of a block of NT threads' stacks.
#define SRT_SHARED_STACK(NAME, NT)                         \
  __shared__ uint2 NAME##_e[kShDepth][NT];                 \
  __shared__ float NAME##_t[kShDepth][NT];                 \
  SharedStack<NT> NAME(NAME##_e, NAME##_t)

// Pass 1 of the default walk for the two-child kinds: front to back from
// `root`; returns m (smallest hit distance), how many primitives hit at m,
// the one found first (in b), and whether one of those at m was reported
// before its own leaf box's entry.
template <int KIND, class Stk = LocalStack>
__device__ __forceinline__ void pass1_node2(const Node2 *__restrict__ nodes,
                                            const float4 *__restrict__ prims,
                                            const uint32_t *__restrict__ sidx,
                                            const Ctx2 &c, uint32_t root, Best &b, Work &w,
                                            uint32_t max_iter, float &m_out,
                                            uint32_t &at_m_out, bool &viol_out,
                                            Stk &&stk = Stk()) {
  float m = FLT_MAX, m2 = FLT_MAX;  // smallest and second smallest distance
  float e_best = 0.0f;              // leaf box entry of the candidate at m
  uint32_t at_m = 0;
  bool viol = false;
  int sp = 0;
  stk.put(0, make_uint2(root, 0u), -FLT_MAX);
  while (true) {
    uint2 leaf = make_uint2(0u, 0u);
    float lt = 0.0f;
    while (sp >= 0) {
      if (++w.it > max_iter) { w.fail = true; sp = -1; break; }
      float et;
      const uint2 e = stk.get(sp, et);
      sp--;
      const float bnd = bound_rel(m, kRelTri);
      if (et > bnd) continue;
      if (e.y != 0) { leaf = e; lt = et; break; }
      w.branch++;
      const float4 *np = reinterpret_cast<const float4 *>(nodes + e.x);
      const float4 a = __ldg(np), bb = __ldg(np + 1), cc = __ldg(np + 2);
      const uint4 d = __ldg(reinterpret_cast<const uint4 *>(np + 3));
      float t0, t1;
      const bool h0 = ray_aabb_t<true>(bnd, a.x, a.y, a.z, a.w, bb.x, bb.y, c.r, t0);
      const bool h1 = ray_aabb_t<true>(bnd, bb.z, bb.w, cc.x, cc.y, cc.z, cc.w, c.r, t1);
      const uint2 e0 = make_uint2(d.x, d.z & kCountMask),
                  e1 = make_uint2(d.y, d.w & kCountMask);
      if (sp + 2 >= std::remove_reference_t<Stk>::kDepth) { w.fail = true; sp = -1; break; }
      if (h0 && h1) {
        const bool first1 = t1 < t0;
        stk.put(++sp, first1 ? e0 : e1, first1 ? t0 : t1);
        stk.put(++sp, first1 ? e1 : e0, first1 ? t1 : t0);
      } else if (h0) {
        stk.put(++sp, e0, t0);
      } else if (h1) {
        stk.put(++sp, e1, t1);
      }
    }
    if (leaf.y == 0) break;
    w.leaf++;
    w.prim += leaf.y;
    // primitive j + 1 is loaded while j is tested
    Prim2<KIND> nx;
    nx.load(prims, sidx, leaf.x);
    for (uint32_t j = leaf.x; j < leaf.x + leaf.y; j++) {
      const Prim2<KIND> P = nx;
      if (j + 1 < leaf.x + leaf.y) nx.load(prims, sidx, j + 1);
      float t, u, v;
      if (!P.test(c, FLT_MAX, t, u, v)) continue;
      if (t < m) {
        m2 = m;
        m = t;
        at_m = 1;
        viol = below_entry(t, lt);
        e_best = lt;
        b.t = t; b.u = u; b.v = v; b.prim = P.f; b.j = j;
      } else {
        if (t < m2) m2 = t;
        if (t == m) {
          at_m++;
          viol = viol || below_entry(t, lt);
        }
      }
    }
  }
  // a single candidate below its box's entry e is hidden only by another
  // primitive nearer than e (all tested: e lies below the pruning bound)
  if (viol && at_m == 1) viol = !(m2 >= e_best) || !(e_best < bound_rel(m, kRelTri));
  m_out = m;
  at_m_out = at_m;
  viol_out = viol;
}

// Rays of a first-pass kernel: with `next` (a zeroed counter), persistent
// warps take 32 consecutive rays at a time until all n are done, so every SM
// stays busy to the end whatever the rays cost; without it, one thread per
// ray over the grid.
template <typename Body>
__device__ __forceinline__ void for_each_ray(size_t n, uint32_t *__restrict__ next,
                                             const Body &body) {
  if (!next) {
    const size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (k < n) body(k);
    return;
  }
  const int lane = threadIdx.x & 31;
  while (true) {
    uint32_t b0 = 0;
    if (lane == 0) b0 = atomicAdd(next, 32u);
    b0 = __shfl_sync(0xffffffffu, b0, 0);
    if ((size_t)b0 >= n) break;
    const size_t k = (size_t)b0 + (size_t)lane;
    if (k < n) body(k);
  }
}

// Two-child kinds (triangles, spheres).  SINGLE: the reference's walk for
// every ray.
template <int KIND, bool SINGLE>
__global__ void __launch_bounds__(128)
trace_node2_kernel(const Node2 *__restrict__ nodes, const float4 *__restrict__ prims,
                   const uint32_t *__restrict__ sidx, const srt_ray *__restrict__ rays,
                   size_t n, srt_hit *__restrict__ hits,
                   const SceneInfo *__restrict__ scene,
                   const float *__restrict__ prev_normals, float *__restrict__ normal_out,
                   unsigned long long *__restrict__ stats, Deferred *__restrict__ dlist,
                   uint32_t *__restrict__ dcount, uint32_t max_iter,
                   uint32_t *__restrict__ err, const uint32_t *__restrict__ order,
                   uint32_t *__restrict__ next = nullptr) {
  for_each_ray(n, next, [&](size_t k) {
    const size_t i = order ? (size_t)__ldg(&order[k]) : k;  // ray of this thread
    const Ctx2 c = make_ctx2<KIND>(rays, i, scene, prev_normals);
    Work w;
    Best b;
    if (SINGLE) {
      ref_walk2<KIND>(nodes, prims, sidx, c, b, w, max_iter);
    } else {
      float m;
      uint32_t at_m;
      bool viol;
      pass1_node2<KIND>(nodes, prims, sidx, c, 0u, b, w, max_iter, m, at_m, viol);
      if (!w.fail && (viol || at_m > 1)) {
        const uint32_t q = atomicAdd(dcount, 1u);
        dlist[q] = Deferred{(uint32_t)i, viol ? 1u : 0u, (double)m};
        add_stats(stats, w, 0);
        return;
      }
    }
    if (w.fail) atomicOr(err, kErrIter);
    add_stats(stats, w, 0);
    store_node2<KIND>(i, b, c, prims, hits, normal_out);
  });
}

template <int KIND>
__global__ void __launch_bounds__(128)
resolve_node2_kernel(const Node2 *__restrict__ nodes, const float4 *__restrict__ prims,
                     const uint32_t *__restrict__ sidx, const srt_ray *__restrict__ rays,
                     srt_hit *__restrict__ hits, const SceneInfo *__restrict__ scene,
                     const float *__restrict__ prev_normals,
                     float *__restrict__ normal_out, unsigned long long *__restrict__ stats,
                     const Deferred *__restrict__ dlist, const uint32_t *__restrict__ dcount,
                     uint32_t max_iter, uint32_t *__restrict__ err) {
  const uint32_t cnt = *dcount;
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < cnt;
       k += gridDim.x * blockDim.x) {
    const Deferred dfr = dlist[k];
    const Ctx2 c = make_ctx2<KIND>(rays, dfr.ray, scene, prev_normals);
    Work w;
    Best b;
    if (dfr.full) {
      ref_walk2_from<KIND>(nodes, prims, sidx, c, b, w, max_iter, (float)dfr.m);
    } else {
      // triangles keep the last candidate at m (t <= current), spheres the
      // first (t < current)
      const float m = (float)dfr.m;
      const float t0 = (KIND == SRT_TRIANGLES) ? m : nextafterf(m, FLT_MAX);
      window_walk2<KIND>(nodes, prims, sidx, c, bound_rel(m, kRelTri), t0, b, w, max_iter);
    }
    if (w.fail) atomicOr(err, kErrIter);
    add_stats(stats, w, dfr.full);
    store_node2<KIND>(dfr.ray, b, c, prims, hits, normal_out);
  }
}

// ---- tetrahedra (own-box nodes, FP64 entry distance)
struct CtxT {
  RayF r;
  TetRay tr;
  uint32_t prev_prim;
};

// (ul1 is formed only for te < take_below: the candidates a caller keeps)
// P: float4 (a float cache, three per tetrahedron) or double2 (a cache of
// double-precision positions, six per tetrahedron).
template <typename P>
__device__ __forceinline__ bool candT(const P *__restrict__ prims,
                                      const uint32_t *__restrict__ sidx, uint32_t j,
                                      const CtxT &c, double take_below, uint32_t &f, int &ef,
                                      double &e1, double &e2, double &ul1, double &te) {
  f = __ldg(&sidx[j]);
  if (f == c.prev_prim) return false;
  if constexpr (std::is_same<P, double2>::value) {
    TetVD V;
#pragma unroll
    for (int q = 0; q < 6; q++) {
      const double2 d = __ldg(&prims[6 * (size_t)j + q]);
      V.v[2 * q] = d.x;
      V.v[2 * q + 1] = d.y;
    }
    return ray_tet(c.tr, V, take_below, ef, e1, e2, ul1, te) && te >= 0.0;
  } else {
    const float4 q0 = __ldg(&prims[3 * (size_t)j]);
    const float4 q1 = __ldg(&prims[3 * (size_t)j + 1]);
    const float4 q2 = __ldg(&prims[3 * (size_t)j + 2]);
    const TetV V = {{q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w, q2.x, q2.y, q2.z, q2.w}};
    return ray_tet(c.tr, V, take_below, ef, e1, e2, ul1, te) && te >= 0.0;
  }
}

__device__ __forceinline__ void take_tet(Best &b, double te, double e1, double e2,
                                         double ul1, uint32_t f, int ef) {
  b.t = (float)te;
  b.u = (float)e1;
  b.v = (float)ul1;  // the reference's isect.v receives uLeave1
  b.prim = f;
  b.sub = (uint32_t)ef;
  b.e1 = e1;
  b.e2 = e2;
}

// The reference's walk (render/render_accel_tetra.cc:2200) with the
// running distance starting at t0 or, with WINDOW, the reference order
// through boxes entered before `bnd` keeping only candidates at most `whi`
// away.
template <bool WINDOW, typename P = float4>
__device__ void walkT(const NodeT *__restrict__ nodes, const P *__restrict__ prims,
                      const uint32_t *__restrict__ sidx, const CtxT &c, float bnd,
                      double whi, Best &b, Work &w, uint32_t max_iter, float t0 = FLT_MAX) {
  b = Best();
  float t = t0;
  uint32_t stk[kStack];
  int sp = 0;
  stk[0] = 0u;
  while (true) {
    uint32_t lref = 0, lcnt = 0;
    while (sp >= 0) {
      if (++w.it > max_iter) { w.fail = true; sp = -1; break; }
      const uint32_t ni = stk[sp--];
      const float4 *np = reinterpret_cast<const float4 *>(nodes + ni);
      const float4 a = __ldg(np), bb = __ldg(np + 1);
      const uint32_t meta = __float_as_uint(a.w), ref = __float_as_uint(bb.w);
      w.branch++;
      if (!ray_aabb<false>(WINDOW ? bnd : t, a.x, a.y, a.z, bb.x, bb.y, bb.z, c.r)) continue;
      if (meta & kLeafBit) { lref = ref; lcnt = meta & kCountMask; break; }
      const int nearc = c.r.sgn[meta & 3u], farc = 1 - nearc;
      if (sp + 2 >= kStack) { w.fail = true; sp = -1; break; }
      stk[++sp] = ref + (uint32_t)farc;
      stk[++sp] = ref + (uint32_t)nearc;
    }
    if (lcnt == 0) break;
    w.leaf++;
    w.prim += lcnt;
    for (uint32_t j = lref; j < lref + lcnt; j++) {
      uint32_t f;
      int ef;
      double e1, e2, ul1, te;
      if (!candT(prims, sidx, j, c, (double)t, f, ef, e1, e2, ul1, te)) continue;
      if (WINDOW && !(te <= whi)) continue;
      if (te < (double)t) {
        take_tet(b, te, e1, e2, ul1, f, ef);
        t = (float)te;
      }
    }
  }
}

__device__ __forceinline__ double window_hi(double m) {
  float wf = __double2float_rn(m);
#pragma unroll
  for (int k = 0; k < 8; k++) wf = nextafterf(wf, FLT_MAX);
  return (double)wf;
}

// The tetrahedron fallback: the reference's walk from pass 1's pruning
// bound, the full walk if nothing is accepted below it (see ref_walk2_from).
template <typename P>
__device__ __forceinline__ void walkT_from(const NodeT *__restrict__ nodes,
                                           const P *__restrict__ prims,
                                           const uint32_t *__restrict__ sidx, const CtxT &c,
                                           Best &b, Work &w, uint32_t max_iter, double m) {
  walkT<false, P>(nodes, prims, sidx, c, 0.0f, 0.0, b, w, max_iter, bound_rel((float)m, kRelTet));
  if (b.prim != kNone || w.fail) return;
  w.it = 0;
  walkT<false, P>(nodes, prims, sidx, c, 0.0f, 0.0, b, w, max_iter);
}

__device__ __forceinline__ void store_tet(size_t i, const Best &b,
                                          srt_hit *__restrict__ hits,
                                          uint32_t *__restrict__ subface,
                                          const uint32_t *__restrict__ faces,
                                          const float *__restrict__ vscalar,
                                          float *__restrict__ scalar_out) {
  const bool any = b.t < FLT_MAX && b.prim != kNone;
  reinterpret_cast<float4 *>(hits)[i] =
      make_float4(any ? b.t : FLT_MAX, any ? b.u : 0.0f, any ? b.v : 0.0f,
                  __uint_as_float(any ? b.prim : kNone));
  if (subface) subface[i] = any ? b.sub : 0u;
  if (scalar_out) {
    float s = 0.0f;
    if (any && faces && vscalar) {
      // entering face vertex order (A, B, C) per face id, as the Pluecker
      // test forms its barycentric point
      // (A, B, C) = (3 - f, f ^ 2, f ^ 1): faces 0..3 -> (3,2,1), (2,3,0), (1,0,3), (0,1,2)
      const uint32_t *tv = faces + 4 * (size_t)b.prim;
      const double sa = vscalar[tv[3 - b.sub]], sb = vscalar[tv[b.sub ^ 2u]],
                   sc = vscalar[tv[b.sub ^ 1u]];
      s = (float)((1.0 - b.e1 - b.e2) * sa + b.e1 * sb + b.e2 * sc);
    }
    scalar_out[i] = s;
  }
}

__device__ __forceinline__ CtxT make_ctxT(const srt_ray *__restrict__ rays, size_t i) {
  CtxT c;
  float prev_t;
  c.r = load_ray(rays, i, c.prev_prim, prev_t);
  c.tr = tet_ray({c.r.o[0], c.r.o[1], c.r.o[2]}, {c.r.d[0], c.r.d[1], c.r.d[2]});
  return c;
}

// Per-ray state of a tetrahedron first pass: the smallest and second
// smallest hit distances m, m2 and the window of up to four entry distances
// within 8 float steps of m (kept to recount when m drops), each rounded up
// to float -- exact for the comparisons against the float window bound.
// defer: the ray needs the reference-order walk, over the whole tree (full:
// a candidate in that window reported before its own leaf box's entry) or
// through the window at m (several candidates near m).  The outcome does not
// depend on the order the leaves are visited in: every tetrahedron whose leaf
// box is entered below the final pruning bound is tested in any order.
struct TetPass1 {
  double m = DBL_MAX, m2 = DBL_MAX;
  float e_best = 0.0f;  // leaf box entry of the candidate at m
  float wl[4] = {0.0f, 0.0f, 0.0f, 0.0f};
  uint32_t wset = 0;   // bit k: window slot k holds an entry
  uint32_t wviol = 0;  // bit k: slot k's entry lies below its own leaf box's entry
  bool overflow = false, viol_lost = false;

  __device__ __forceinline__ float bound() const {
    return (m < DBL_MAX) ? bound_rel((float)m, kRelTet) : FLT_MAX;
  }

  // Tests the `cnt` tetrahedra of a leaf at sorted slot `ref`, entered at lt.
  template <typename P>
  __device__ __forceinline__ void leaf(const P *__restrict__ prims,
                                       const uint32_t *__restrict__ sidx, const CtxT &c,
                                       uint32_t ref, uint32_t cnt, float lt, Best &b) {
    for (uint32_t j = ref; j < ref + cnt; j++) {
      uint32_t f;
      int ef;
      double e1, e2, ul1, te;
      if (!candT(prims, sidx, j, c, m, f, ef, e1, e2, ul1, te)) continue;
      const bool below = below_entry(te, lt);
      if (te < m) {
        m2 = m;
        m = te;
        e_best = lt;
        take_tet(b, te, e1, e2, ul1, f, ef);
        const float whi = (float)window_hi(m);
#pragma unroll
        for (int k = 0; k < 4; k++)
          if (!(wl[k] <= whi)) wset &= ~(1u << k);
        wviol &= wset;
      } else if (te < m2) {
        m2 = te;
      }
      if (te <= window_hi(m)) {
        if (wset != 0xfu) {
          const int k = __ffs(~wset) - 1;  // first free slot
          const float r = __double2float_ru(te);
#pragma unroll
          for (int q = 0; q < 4; q++)
            if (q == k) wl[q] = r;
          wset |= 1u << k;
          wviol |= (below ? 1u : 0u) << k;
        } else {
          overflow = true;
          viol_lost = viol_lost || below;
        }
      }
    }
  }

  __device__ __forceinline__ void finish(double &m_out, bool &defer_out,
                                         bool &full_out) const {
    const int nwin = __popc(wset);
    bool viol = viol_lost || wviol != 0;
    // a single candidate below its box's entry e is hidden only by another
    // primitive nearer than e (all tested: e lies below the pruning bound)
    if (viol && nwin == 1 && !overflow)
      viol = !(m2 >= (double)e_best) || !(e_best < bound_rel((float)m, kRelTet));
    m_out = m;
    defer_out = viol || nwin > 1 || overflow;
    full_out = viol;
  }
};

// A child's stack entry, read with its box at the parent: (ref, leaf count),
// count 0 for a branch (whose children sit at ref, ref + 1).
__device__ __forceinline__ uint2 tet_entry(float4 lo, float4 hi) {
  const uint32_t meta = __float_as_uint(lo.w);
  return make_uint2(__float_as_uint(hi.w), (meta & kLeafBit) ? meta & kCountMask : 0u);
}

// Pass 1 of the default tetrahedron walk for one ray: front to back, stack
// entries from tet_entry so that a popped branch loads only its children's
// boxes.
template <class Stk = LocalStack, typename PT = float4>
__device__ __forceinline__ void pass1_tet(const NodeT *__restrict__ nodes,
                                          const PT *__restrict__ prims,
                                          const uint32_t *__restrict__ sidx, const CtxT &c,
                                          Best &b, Work &w, uint32_t max_iter, double &m_out,
                                          bool &defer_out, bool &full_out, Stk &&stk = Stk()) {
  TetPass1 P;
  int sp = -1;
  {
    const float4 *np = reinterpret_cast<const float4 *>(nodes);
    const float4 a = __ldg(np), bb = __ldg(np + 1);
    float t0;
    if (ray_aabb_t<false>(FLT_MAX, a.x, a.y, a.z, bb.x, bb.y, bb.z, c.r, t0)) {
      stk.put(0, tet_entry(a, bb), t0);
      sp = 0;
    }
  }
  while (true) {
    uint2 leaf = make_uint2(0u, 0u);
    float lt = 0.0f;
    while (sp >= 0) {
      if (++w.it > max_iter) { w.fail = true; sp = -1; break; }
      float et;
      const uint2 e = stk.get(sp, et);
      sp--;
      const float bnd = P.bound();
      if (et > bnd) continue;
      if (e.y != 0) { leaf = e; lt = et; break; }
      w.branch++;
      // the two children are adjacent: test their own boxes here
      const float4 *cp = reinterpret_cast<const float4 *>(nodes + e.x);
      const float4 a0 = __ldg(cp), b0 = __ldg(cp + 1), a1 = __ldg(cp + 2), b1 = __ldg(cp + 3);
      float t0, t1;
      const bool h0 = ray_aabb_t<false>(bnd, a0.x, a0.y, a0.z, b0.x, b0.y, b0.z, c.r, t0);
      const bool h1 = ray_aabb_t<false>(bnd, a1.x, a1.y, a1.z, b1.x, b1.y, b1.z, c.r, t1);
      const uint2 e0 = tet_entry(a0, b0), e1 = tet_entry(a1, b1);
      if (sp + 2 >= std::remove_reference_t<Stk>::kDepth) { w.fail = true; sp = -1; break; }
      if (h0 && h1) {
        const bool first1 = t1 < t0;
        stk.put(++sp, first1 ? e0 : e1, first1 ? t0 : t1);
        stk.put(++sp, first1 ? e1 : e0, first1 ? t1 : t0);
      } else if (h0) {
        stk.put(++sp, e0, t0);
      } else if (h1) {
        stk.put(++sp, e1, t1);
      }
    }
    if (leaf.y == 0) break;
    w.leaf++;
    w.prim += leaf.y;
    P.leaf(prims, sidx, c, leaf.x, leaf.y, lt, b);
  }
  P.finish(m_out, defer_out, full_out);
}

template <bool SINGLE, typename P = float4>
__global__ void __launch_bounds__(128)
trace_tet_kernel(const NodeT *__restrict__ nodes, const P *__restrict__ prims,
                 const uint32_t *__restrict__ sidx, const srt_ray *__restrict__ rays,
                 size_t n, srt_hit *__restrict__ hits, uint32_t *__restrict__ subface,
                 const uint32_t *__restrict__ faces, const float *__restrict__ vscalar,
                 float *__restrict__ scalar_out, unsigned long long *__restrict__ stats,
                 Deferred *__restrict__ dlist, uint32_t *__restrict__ dcount,
                 uint32_t max_iter, uint32_t *__restrict__ err,
                 const uint32_t *__restrict__ order, uint32_t *__restrict__ next = nullptr) {
  SRT_SHARED_STACK(sstk, 128);
  for_each_ray(n, next, [&](size_t k) {
    const size_t i = order ? (size_t)__ldg(&order[k]) : k;  // ray of this thread
    const CtxT c = make_ctxT(rays, i);
    Work w;
    Best b;
    if (SINGLE) {
      walkT<false>(nodes, prims, sidx, c, 0.0f, 0.0, b, w, max_iter);
    } else {
      double m;
      bool defer, full;
      pass1_tet(nodes, prims, sidx, c, b, w, max_iter, m, defer, full, sstk);
      if (!w.fail && defer) {
        const uint32_t q = atomicAdd(dcount, 1u);
        dlist[q] = Deferred{(uint32_t)i, full ? 1u : 0u, m};
        add_stats(stats, w, 0);
        return;
      }
    }
    if (w.fail) atomicOr(err, kErrIter);
    add_stats(stats, w, 0);
    store_tet(i, b, hits, subface, faces, vscalar, scalar_out);
  });
}

template <typename P = float4>
__global__ void __launch_bounds__(128)
resolve_tet_kernel(const NodeT *__restrict__ nodes, const P *__restrict__ prims,
                   const uint32_t *__restrict__ sidx, const srt_ray *__restrict__ rays,
                   srt_hit *__restrict__ hits, uint32_t *__restrict__ subface,
                   const uint32_t *__restrict__ faces, const float *__restrict__ vscalar,
                   float *__restrict__ scalar_out, unsigned long long *__restrict__ stats,
                   const Deferred *__restrict__ dlist, const uint32_t *__restrict__ dcount,
                   uint32_t max_iter, uint32_t *__restrict__ err) {
  const uint32_t cnt = *dcount;
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < cnt;
       k += gridDim.x * blockDim.x) {
    const Deferred dfr = dlist[k];
    const CtxT c = make_ctxT(rays, dfr.ray);
    Work w;
    Best b;
    if (dfr.full) {
      walkT_from(nodes, prims, sidx, c, b, w, max_iter, dfr.m);
    } else {
      const double whi = window_hi(dfr.m);
      walkT<true>(nodes, prims, sidx, c, bound_rel((float)whi, kRelTet), whi, b, w,
                  max_iter);
    }
    if (w.fail) atomicOr(err, kErrIter);
    add_stats(stats, w, dfr.full);
    store_tet(dfr.ray, b, hits, subface, faces, vscalar, scalar_out);
  }
}

// --------------------------------------------------------------- batches
// All rays of many triangle scenes in one persistent launch: each warp
// takes the next 32 * R rays from a global counter (scenes of very
// different cost balance across the GPU), finds the ray's scene from the
// ray offsets and walks that scene's tree from its root, with a stack of
// DEPTH entries (a walk that would need more stops with the limit error).
// order (or NULL): the rays in a coherent order, grouped by scene.
template <int DEPTH>
__global__ void __launch_bounds__(256)
trace_batch_kernel(const Node2 *__restrict__ nodes, const float4 *__restrict__ prims,
                   const srt_ray *__restrict__ rays, srt_hit *__restrict__ hits,
                   const SceneInfo *__restrict__ scenes, const uint32_t *__restrict__ roots,
                   const uint32_t *__restrict__ roff, int nseg, uint32_t total,
                   uint32_t *__restrict__ work, int R, unsigned long long *__restrict__ stats,
                   Deferred *__restrict__ dlist, uint32_t *__restrict__ dcount,
                   uint32_t max_iter, uint32_t *__restrict__ err,
                   const uint32_t *__restrict__ order) {
  // each warp takes 32 * R rays at a time (no block-wide barrier: a warp
  // whose rays finish early takes more work at once)
  const uint32_t lane = threadIdx.x & 31u;
  while (true) {
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(work, 32u * (uint32_t)R);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= total) break;
    for (int r = 0; r < R; r++) {
      const uint32_t k = base + (uint32_t)r * 32u + lane;
      if (k >= total) break;
      const uint32_t i = order ? __ldg(&order[k]) : k;
      const int sg = seg_of(roff, nseg, i);
      Ctx2 c;
      c.r = load_ray(rays, i, c.prev_prim, c.prev_t);
      c.keps = scenes[sg].keps;
      c.pn[0] = c.pn[1] = c.pn[2] = 0.0f;
      Work w;
      Best b;
      float m;
      uint32_t at_m;
      bool viol;
      pass1_node2<SRT_TRIANGLES>(nodes, prims, nullptr, c, __ldg(&roots[sg]), b, w, max_iter,
                                 m, at_m, viol, LocalStackN<DEPTH>());
      if (!w.fail && (viol || at_m > 1)) {
        const uint32_t q = atomicAdd(dcount, 1u);
        dlist[q] = Deferred{i, viol ? 1u : 0u, (double)m};
      } else {
        if (w.fail) atomicOr(err, kErrIter);
        store_node2<SRT_TRIANGLES>(i, b, c, prims, hits, nullptr);
      }
      add_stats(stats, w, 0);
    }
  }
}

__global__ void __launch_bounds__(128)
resolve_batch_kernel(const Node2 *__restrict__ nodes, const float4 *__restrict__ prims,
                     const srt_ray *__restrict__ rays, srt_hit *__restrict__ hits,
                     const SceneInfo *__restrict__ scenes, const uint32_t *__restrict__ roots,
                     const uint32_t *__restrict__ roff, int nseg,
                     unsigned long long *__restrict__ stats,
                     const Deferred *__restrict__ dlist, const uint32_t *__restrict__ dcount,
                     uint32_t max_iter, uint32_t *__restrict__ err) {
  const uint32_t cnt = *dcount;
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < cnt;
       k += gridDim.x * blockDim.x) {
    const Deferred dfr = dlist[k];
    const int sg = seg_of(roff, nseg, dfr.ray);
    Ctx2 c;
    c.r = load_ray(rays, dfr.ray, c.prev_prim, c.prev_t);
    c.keps = scenes[sg].keps;
    c.pn[0] = c.pn[1] = c.pn[2] = 0.0f;
    const uint32_t root = __ldg(&roots[sg]);
    Work w;
    Best b;
    if (dfr.full) {
      ref_walk2_from<SRT_TRIANGLES>(nodes, prims, nullptr, c, b, w, max_iter, (float)dfr.m,
                                    root);
    } else {
      const float m = (float)dfr.m;
      window_walk2<SRT_TRIANGLES>(nodes, prims, nullptr, c, bound_rel(m, kRelTri), m, b, w,
                                  max_iter, root);
    }
    if (w.fail) atomicOr(err, kErrIter);
    add_stats(stats, w, dfr.full);
    store_node2<SRT_TRIANGLES>(dfr.ray, b, c, prims, hits, nullptr);
  }
}

}  // namespace

// Blocks of `block` threads of kernel fn that one SM holds at once (the same
// on every device of this architecture; looked up once per kernel).
int resident_blocks(const void *fn, int block) {
  static std::mutex mu;
  static std::vector<std::pair<const void *, int>> known;
  std::lock_guard<std::mutex> lock(mu);
  for (auto &k : known)
    if (k.first == fn) return k.second;
  int nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, block, 0) != cudaSuccess || nb < 1) {
    cudaGetLastError();
    nb = 1;
  }
  known.emplace_back(fn, nb);
  return nb;
}

srt_status launch_trace(srt_accel *a, const srt_ray *rays, size_t n, srt_hit *hits,
                        const float *prev_normals, uint32_t *subface,
                        const float *vscalar, float *scalar_out, float *normal_out,
                        unsigned long long *stats, uint32_t flags, uint32_t max_iter_cap) {
  if (n == 0) return SRT_OK;
  if (n > 0xffffffffull) {
    set_error("at most 2^32-1 rays per call");
    return SRT_ERR_INVALID;
  }
  srt_ctx *ctx = a->ctx;
  const int block = 128;
  const unsigned grid = (unsigned)((n + block - 1) / block);
  const unsigned rgrid = (unsigned)ctx->num_sms * 8;
  // every node and leaf is visited at most once per walk; a caller's cap
  // may only lower that
  uint32_t max_iter = (uint32_t)std::min<size_t>(8 * a->n + 64, 0xfffffff0u);
  if (max_iter_cap) max_iter = std::min(max_iter, max_iter_cap);
  const SceneInfo *scene = a->scene.as<SceneInfo>();
  const bool single = (flags & SRT_TRACE_SINGLE_PASS) != 0;
  cudaStream_t st = ctx->stream;
  // scratch header: [0] deferred-ray count, [1] persistent warps' ray counter
  Deferred *dlist = nullptr;
  uint32_t *dcount = nullptr, *next = nullptr;
  {
    cudaError_t e = ctx->s_defer.ensure((single ? 0 : n * sizeof(Deferred)) + 256);
    if (e != cudaSuccess) return cuda_status(e, "deferred list");
    dcount = ctx->s_defer.as<uint32_t>();
    dlist = reinterpret_cast<Deferred *>(ctx->s_defer.as<char>() + 256);
    if ((e = cudaMemsetAsync(dcount, 0, 8, st)) != cudaSuccess)
      return cuda_status(e, "deferred count");
    if (single) dcount = nullptr, dlist = nullptr;
    if (!(flags & SRT_TRACE_GRID)) next = ctx->s_defer.as<uint32_t>() + 1;
  }
  const float *pn = a->kind == SRT_SPHERES ? prev_normals : nullptr;
  // first-pass grid: the whole ray set, or (persistent warps) as many blocks
  // as the SMs hold at once, never more than the rays need
  auto fgrid = [&](const void *fn) -> unsigned {
    if (!next) return grid;
    const unsigned p = (unsigned)(ctx->num_sms * resident_blocks(fn, block));
    return std::max(1u, std::min(grid, p));
  };
  const uint32_t *order = nullptr;
  if (flags & SRT_TRACE_SORT_RAYS) {
    srt_status s = ray_order(ctx, rays, n, &order);
    if (s != SRT_OK) return s;
  }
  switch (a->kind) {
    case SRT_TRIANGLES:
    case SRT_SPHERES: {
      const Node2 *nd = a->nodes.as<Node2>();
      const float4 *pr = a->prims.as<float4>();
      const uint32_t *ix = a->indices.as<uint32_t>();
      const bool tri = a->kind == SRT_TRIANGLES;
      const auto kern = tri ? (single ? trace_node2_kernel<SRT_TRIANGLES, true>
                                      : trace_node2_kernel<SRT_TRIANGLES, false>)
                            : (single ? trace_node2_kernel<SRT_SPHERES, true>
                                      : trace_node2_kernel<SRT_SPHERES, false>);
      kern<<<fgrid((const void *)kern), block, 0, st>>>(
          nd, pr, ix, rays, n, hits, scene, pn, normal_out, stats, dlist, dcount, max_iter,
          ctx->d_err, order, next);
      if (!single) {
        const auto res = tri ? resolve_node2_kernel<SRT_TRIANGLES>
                             : resolve_node2_kernel<SRT_SPHERES>;
        res<<<rgrid, block, 0, st>>>(nd, pr, ix, rays, hits, scene, pn, normal_out, stats,
                                     dlist, dcount, max_iter, ctx->d_err);
        ctx->launches++;
      }
      break;
    }
    case SRT_TETRAHEDRA: {
      const NodeT *nd = a->nodes.as<NodeT>();
      const uint32_t *ix = a->indices.as<uint32_t>();
      // the primitive cache holds floats, or the doubles of double-precision
      // positions
      auto run = [&](auto *pr) {
        using P = std::remove_cv_t<std::remove_pointer_t<decltype(pr)>>;
        const auto kern = single ? trace_tet_kernel<true, P> : trace_tet_kernel<false, P>;
        kern<<<fgrid((const void *)kern), block, 0, st>>>(nd, pr, ix, rays, n, hits, subface,
                                                          a->src_faces, vscalar, scalar_out,
                                                          stats, dlist, dcount, max_iter,
                                                          ctx->d_err, order, next);
        if (!single) {
          resolve_tet_kernel<P><<<rgrid, block, 0, st>>>(nd, pr, ix, rays, hits, subface,
                                                         a->src_faces, vscalar, scalar_out,
                                                         stats, dlist, dcount, max_iter,
                                                         ctx->d_err);
          ctx->launches++;
        }
      };
      if (a->dbl)
        run(a->prims.as<const double2>());
      else
        run(a->prims.as<const float4>());
      break;
    }
  }
  ctx->launches++;
  return cuda_status(cudaGetLastError(), "trace");
}

srt_status launch_trace_batch(srt_ctx *ctx, BatchTree &bt, const srt_ray *rays,
                              srt_hit *hits, int block, int R,
                              unsigned long long *stats, int depth,
                              const uint32_t *order) {
  const uint32_t total = (uint32_t)bt.nrays;
  if (total == 0) return SRT_OK;
  cudaStream_t st = ctx->stream;
  cudaError_t e = ctx->s_defer.ensure((size_t)total * sizeof(Deferred) + 256);
  if (e != cudaSuccess) return cuda_status(e, "deferred list");
  uint32_t *dcount = ctx->s_defer.as<uint32_t>();  // [0] deferred count, [1] work counter
  Deferred *dlist = reinterpret_cast<Deferred *>(ctx->s_defer.as<char>() + 256);
  if ((e = cudaMemsetAsync(dcount, 0, 8, st)) != cudaSuccess)
    return cuda_status(e, "batch counters");
  const auto kern = depth <= 24 ? trace_batch_kernel<24>
                    : depth <= 32 ? trace_batch_kernel<32> : trace_batch_kernel<48>;
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, block, 0);
  if (per_sm < 1) per_sm = 1;
  const uint32_t max_iter = (uint32_t)std::min<size_t>(8 * bt.nprims + 64, 0xfffffff0u);
  kern<<<ctx->num_sms * per_sm, block, 0, st>>>(
      bt.nodes.as<Node2>(), bt.prims.as<float4>(), rays, hits, bt.scenes.as<SceneInfo>(),
      bt.roots.as<uint32_t>(), bt.roff.as<uint32_t>(), bt.nseg, total, dcount + 1, R, stats,
      dlist, dcount, max_iter, ctx->d_err, order);
  resolve_batch_kernel<<<ctx->num_sms * 8, 128, 0, st>>>(
      bt.nodes.as<Node2>(), bt.prims.as<float4>(), rays, hits, bt.scenes.as<SceneInfo>(),
      bt.roots.as<uint32_t>(), bt.roff.as<uint32_t>(), bt.nseg, stats, dlist, dcount,
      max_iter, ctx->d_err);
  ctx->launches += 2;
  return cuda_status(cudaGetLastError(), "batch trace");
}

}  // namespace srt

// ================================================================ scenes
// RenderGraph::Trace (gles/gles_render_graph.cc:143-314) for a whole ray
// array.  Per ray: the top-level BVHTree walk collects the elements whose
// world box the ray enters (render/render_bvh_tree.cc:504-585, double slab
// test with SetupRay's guarded reciprocals), sorted by entry distance (a
// stable insertion sort: std::sort's order for up to 16 candidates); each
// element in that order unless its entry lies beyond the nearest world hit
// so far: the ray is taken into the element's local space with the inverse
// transforms (Matrixd::MultV, double), traversed, and the hit point taken
// back to world space; the world distance (float length) decides, strictly
// smaller wins.  The previous hit's primitive, distance and normal apply
// only inside the element the ray left.
//
// On the GPU this runs in rounds.  scene_top_kernel walks the top-level
// tree of every ray and stores its sorted candidates; round r takes every
// live ray's r-th candidate, one kernel per element kind (so a warp runs one
// kind's walk), walks the element with the same exact walks as the single
// accel trace, applies the world-distance rule to the ray's running best and
// queues the ray's next candidate unless that one's entry lies beyond the
// nearest hit (then so do all later ones: they are sorted).  An element's
// hit depends on the ray and that element alone, so the rounds return the
// sequential loop's result exactly.  Rays with more candidates than the
// rounds hold run the loop in one thread (scene_loop_kernel).
namespace srt {
namespace {

constexpr int kTopCand = 64;
constexpr int kTopStack = 64;

__device__ __forceinline__ bool top_aabb(const TopNode &t, const double o[3],
                                         const double inv[3], const int sgn[3], double &tmin,
                                         double &tmax) {
  const double mnx = sgn[0] ? t.bmax[0] : t.bmin[0], mny = sgn[1] ? t.bmax[1] : t.bmin[1],
               mnz = sgn[2] ? t.bmax[2] : t.bmin[2];
  const double mxx = sgn[0] ? t.bmin[0] : t.bmax[0], mxy = sgn[1] ? t.bmin[1] : t.bmax[1],
               mxz = sgn[2] ? t.bmin[2] : t.bmax[2];
  const double tminx = (mnx - o[0]) * inv[0], tmaxx = (mxx - o[0]) * inv[0];
  const double tminy = (mny - o[1]) * inv[1], tmaxy = (mxy - o[1]) * inv[1];
  double a = (tminx > tminy) ? tminx : tminy;
  double b = (tmaxx < tmaxy) ? tmaxx : tmaxy;
  const double tminz = (mnz - o[2]) * inv[2], tmaxz = (mxz - o[2]) * inv[2];
  a = (a > tminz) ? a : tminz;
  b = (b < tmaxz) ? b : tmaxz;
  if ((b > 0.0) && (a <= b)) {
    tmin = a;
    tmax = b;
    return true;
  }
  return false;
}

// Matrixd::MultV: dst[k] = m[0][k] v0 + m[1][k] v1 + m[2][k] v2 + m[3][k].
__device__ __forceinline__ void multv(const double m[16], const double v[3], double o[3]) {
#pragma unroll
  for (int k = 0; k < 3; k++) o[k] = ((m[k] * v[0] + m[4 + k] * v[1]) + m[8 + k] * v[2]) + m[12 + k];
}

// The top-level walk of one ray: candidates (entry distance, element) in
// walk order, then stably sorted by entry distance.  Returns their number.
__device__ __forceinline__ int top_candidates(const TopNode *__restrict__ top,
                                              const double ro[3], const double rd[3],
                                              double ct[kTopCand], uint32_t cid[kTopCand],
                                              uint32_t max_iter, uint32_t &ntop,
                                              uint32_t *__restrict__ err) {
  int sgn[3];
  double inv[3];
#pragma unroll
  for (int k = 0; k < 3; k++) {
    sgn[k] = rd[k] < 0.0 ? 1 : 0;
    inv[k] = fabs(rd[k]) > 2.0e-15 ? 1.0 / rd[k] : (rd[k] < 0.0 ? -(double)FLT_MAX : (double)FLT_MAX);
  }
  int nc = 0;
  int stk[kTopStack];
  int sp = 0, node = 0;
  for (uint32_t guard = 0; guard < max_iter; guard++) {
    const TopNode &t = top[node];
    ntop++;
    if (t.leaf) {
      double a, b;
      if (top_aabb(t, ro, inv, sgn, a, b)) {
        if (nc < kTopCand) {
          ct[nc] = a;
          cid[nc] = t.id;
          nc++;
        } else {
          atomicOr(err, kErrStack);
        }
      }
      if (sp < 1) break;
      node = stk[--sp];
    } else {
      double a0, b0, a1, b1;
      const bool h0 = t.child[0] > 0 && top_aabb(top[t.child[0]], ro, inv, sgn, a0, b0);
      const bool h1 = t.child[1] > 0 && top_aabb(top[t.child[1]], ro, inv, sgn, a1, b1);
      if (!h0 && !h1) {
        if (sp < 1) break;
        node = stk[--sp];
      } else if (h0 && !h1) {
        node = t.child[0];
      } else if (h1 && !h0) {
        node = t.child[1];
      } else {
        const int order = sgn[t.axis];
        if (sp >= kTopStack) {
          atomicOr(err, kErrStack);
          break;
        }
        stk[sp++] = t.child[1 - order];
        node = t.child[order];
      }
    }
  }
  for (int a = 1; a < nc; a++) {  // stable insertion sort by entry distance
    const double kt = ct[a];
    const uint32_t kid = cid[a];
    int b = a - 1;
    while (b >= 0 && kt < ct[b]) {
      ct[b + 1] = ct[b];
      cid[b + 1] = cid[b];
      b--;
    }
    ct[b + 1] = kt;
    cid[b + 1] = kid;
  }
  return nc;
}

// The ray in the element's local space: double origin and direction by the
// inverse transforms, stored as float as the reference's Ray does.
__device__ __forceinline__ RayF local_ray(const SceneElem &e, const double ro[3],
                                          const double rd[3], double lo[3], double ld[3]) {
  multv(e.invT, ro, lo);
  multv(e.invT33, rd, ld);
  RayF lr;
#pragma unroll
  for (int k = 0; k < 3; k++) {
    lr.o[k] = (float)lo[k];
    lr.d[k] = (float)ld[k];
    lr.sgn[k] = lr.d[k] < 0.0f ? 1 : 0;
    lr.inv[k] = __frcp_rn(lr.d[k]);
  }
  return lr;
}

// World distance of a local hit: the float hit point lo + t ld, taken to
// world space by T, minus the world origin, float length.
__device__ __forceinline__ float world_dist(const SceneElem &e, const double lo[3],
                                            const double ld[3], float t, const float org[3]) {
  double lp[3];
#pragma unroll
  for (int k = 0; k < 3; k++) lp[k] = (double)(float)(lo[k] + (double)t * ld[k]);
  double wp[3];
  multv(e.T, lp, wp);
  float po[3];
#pragma unroll
  for (int k = 0; k < 3; k++) po[k] = (float)wp[k] - org[k];
  return sqrtf(po[0] * po[0] + po[1] * po[1] + po[2] * po[2]);
}

// Per-kind walk context of a ray inside one element.
template <int KIND>
struct KindCtx {
  using T = Ctx2;
};
template <>
struct KindCtx<SRT_TETRAHEDRA> {
  using T = CtxT;
};

// Ray i in element e_id's local space (self-hit data only when e_id is the
// ray's previous element); the local ray's double origin and direction in
// lo / ld.
template <int KIND>
__device__ __forceinline__ typename KindCtx<KIND>::T
elem_ctx(const SceneWork &W, uint32_t i, uint32_t e_id, const SceneElem &e, const RayF &r0,
         uint32_t prev_prim, float prev_t, double lo[3], double ld[3]) {
  const double ro[3] = {r0.o[0], r0.o[1], r0.o[2]}, rd[3] = {r0.d[0], r0.d[1], r0.d[2]};
  const RayF lr = local_ray(e, ro, rd, lo, ld);
  const bool same = W.prev_element && __ldg(&W.prev_element[i]) == e_id;
  if constexpr (KIND == SRT_TETRAHEDRA) {
    CtxT c;
    c.r = lr;
    c.tr = tet_ray({lr.o[0], lr.o[1], lr.o[2]}, {lr.d[0], lr.d[1], lr.d[2]});
    c.prev_prim = same ? prev_prim : kNone;
    return c;
  } else {
    Ctx2 c;
    c.r = lr;
    c.prev_prim = same ? prev_prim : kNone;
    c.prev_t = same ? prev_t : 0.0f;
    c.keps = e.scene->keps;
#pragma unroll
    for (int k = 0; k < 3; k++)
      c.pn[k] = (same && W.prev_normals) ? __ldg(&W.prev_normals[3 * (size_t)i + k]) : 0.0f;
    return c;
  }
}

// The front-to-back pass in one element.  Returns whether its result is
// final; otherwise m and full tell the replay (as for the resolve kernels).
template <int KIND>
__device__ __forceinline__ bool elem_pass1(const SceneElem &e, const typename KindCtx<KIND>::T &c,
                                           Best &b, Work &w, uint32_t max_iter, double &m,
                                           bool &full) {
  if constexpr (KIND == SRT_TETRAHEDRA) {
    bool defer;
    const NodeT *nodes = static_cast<const NodeT *>(e.nodes);
    if (e.aux & kTetAuxDouble)
      pass1_tet(nodes, reinterpret_cast<const double2 *>(e.prims), e.sidx, c, b, w, max_iter, m,
                defer, full);
    else
      pass1_tet(nodes, e.prims, e.sidx, c, b, w, max_iter, m, defer, full);
    return w.fail || !defer;
  } else {
    float mf;
    uint32_t at_m;
    bool viol;
    pass1_node2<KIND>(static_cast<const Node2 *>(e.nodes), e.prims, e.sidx, c, 0u, b, w,
                      max_iter, mf, at_m, viol);
    m = mf;
    full = viol;
    return w.fail || !(viol || at_m > 1);
  }
}

// The replay of an inconclusive pass: the reference's walk from the pass's
// bound (full) or the reference order through the window at m.
template <int KIND>
__device__ __forceinline__ void elem_replay(const SceneElem &e,
                                            const typename KindCtx<KIND>::T &c, Best &b,
                                            Work &w, uint32_t max_iter, double m, bool full) {
  w.it = 0;
  if constexpr (KIND == SRT_TETRAHEDRA) {
    const NodeT *nodes = static_cast<const NodeT *>(e.nodes);
    auto replay = [&](auto *prims) {
      if (full) {
        walkT_from(nodes, prims, e.sidx, c, b, w, max_iter, m);
      } else {
        const double whi = window_hi(m);
        walkT<true>(nodes, prims, e.sidx, c, bound_rel((float)whi, kRelTet), whi, b, w,
                    max_iter);
      }
    };
    if (e.aux & kTetAuxDouble)
      replay(reinterpret_cast<const double2 *>(e.prims));
    else
      replay(e.prims);
  } else {
    const Node2 *nodes = static_cast<const Node2 *>(e.nodes);
    const float mf = (float)m;
    if (full) {
      ref_walk2_from<KIND>(nodes, e.prims, e.sidx, c, b, w, max_iter, mf);
    } else {
      const float t0 = (KIND == SRT_TRIANGLES) ? mf : nextafterf(mf, FLT_MAX);
      window_walk2<KIND>(nodes, e.prims, e.sidx, c, bound_rel(mf, kRelTri), t0, b, w,
                         max_iter);
    }
  }
}

__device__ __forceinline__ void add_counts(unsigned long long *__restrict__ stats, int first,
                                           const uint32_t *c, int nc) {
  const unsigned m = __activemask();
  const int leader = __ffs(m) - 1;
  for (int k = 0; k < nc; k++) {
    const uint32_t s = __reduce_add_sync(m, c[k]);
    if ((int)(threadIdx.x & 31u) == leader) atomicAdd(&stats[first + k], (unsigned long long)s);
  }
}

__device__ __forceinline__ float inf_f() { return __int_as_float(0x7f800000); }

// Sorted item -> (ray, candidate slot).  Phase 0 items are ray ids (slot
// 0); phase 1 items index the dense [ray][slot - 1] key array.
__device__ __forceinline__ void item_ray_slot(int phase, uint32_t item, uint32_t &ray,
                                              uint32_t &slot) {
  ray = phase ? item / (kRoundCand - 1) : item;
  slot = phase ? item % (kRoundCand - 1) + 1 : 0u;
}

__global__ void __launch_bounds__(128)
scene_top_kernel(const TopNode *__restrict__ top, SceneWork W) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= W.n) return;
  const float4 *r4 = reinterpret_cast<const float4 *>(W.rays + i);
  const float4 a = __ldg(&r4[0]), b = __ldg(&r4[1]);
  const double ro[3] = {a.x, a.y, a.z}, rd[3] = {b.x, b.y, b.z};
  double ct[kTopCand];
  uint32_t cid[kTopCand];
  uint32_t ntop = 0;
  const int nc = top_candidates(top, ro, rd, ct, cid, W.max_iter, ntop, W.err);
  reinterpret_cast<float4 *>(W.hits)[i] = make_float4(FLT_MAX, 0.0f, 0.0f, __uint_as_float(kNone));
  if (W.element) W.element[i] = kNone;
  W.tnear[i] = inf_f();
  uint32_t key = W.nelem;  // no first candidate for the rounds
  bool loop_only = nc > kRoundCand;
  if (W.rank_start[3] < W.nelem)  // line and solid elements: the per-ray loop walks them
    for (int c = 0; c < nc && !loop_only; c++)
      loop_only = __ldg(&W.elem_rank[cid[c]]) >= W.rank_start[3];
  if (loop_only) {
    W.ncand[i] = 0;
    W.ovf[atomicAdd(&W.counters[2], 1u)] = (uint32_t)i;
  } else {
    W.ncand[i] = (uint8_t)nc;
    for (int c = 0; c < nc; c++) {
      W.cand_t[i * kRoundCand + c] = ct[c];
      W.cand_e[i * kRoundCand + c] = cid[c];
    }
    if (nc > 0) key = __ldg(&W.elem_rank[cid[0]]);
  }
  W.keys0[i] = key;
  if (W.stats) add_counts(W.stats, 0, &ntop, 1);
}

// Each kind's range of a sorted key array (element ranks, kinds in rank
// order, nelem for none): lower bounds of the kinds' first ranks.
__global__ void scene_range_kernel(SceneWork W, int phase) {
  const int t = threadIdx.x;
  if (t >= 4) return;
  const uint32_t *keys = phase ? W.keys1 : W.keys0;
  const size_t n = phase ? W.n * (kRoundCand - 1) : W.n;
  const uint32_t want = W.rank_start[t];
  size_t lo = 0, hi = n;
  while (lo < hi) {
    const size_t mid = lo + (hi - lo) / 2;
    if (keys[mid] < want) lo = mid + 1;
    else hi = mid;
  }
  W.bounds[4 * phase + t] = (uint32_t)lo;
}

// A sphere element's hit takes the spherical (u, v) that the element
// accel's Traverse returns, from the local ray and local distance.
template <typename Ctx>
__device__ __forceinline__ void elem_sphere_uv(const Ctx &c, const SceneElem &e, Best &b) {
  if (!(b.t < FLT_MAX) || b.prim == kNone) return;
  float nn[3];
  sphere_hit_uv(c.r, e.prims, b, nn);
}

// An element walk's result: phase 0 (each ray's first candidate) makes it
// the ray's running best; phase 1 (later candidates that the early cull
// keeps after phase 0) stores it per (ray, slot) for the selection.
__device__ __forceinline__ void finish_item(const SceneWork &W, int phase, uint32_t ray,
                                            size_t cs, uint32_t e_id, const SceneElem &e,
                                            const double lo[3], const double ld[3],
                                            const float org[3], const Best &b) {
  const bool hit = b.t < FLT_MAX && b.prim != kNone;
  const float tw = hit ? world_dist(e, lo, ld, b.t, org) : inf_f();
  if (phase == 0) {
    if (hit && tw < inf_f()) {
      W.tnear[ray] = tw;
      reinterpret_cast<float4 *>(W.hits)[ray] = make_float4(tw, b.u, b.v, __uint_as_float(b.prim));
      if (W.element) W.element[ray] = e_id;
    }
  } else {
    W.res[cs] = make_float4(tw, b.u, b.v, __uint_as_float(hit ? b.prim : kNone));
  }
}

// The element walks of one kind over its range of the sorted items, 32
// items per warp fetch: the front-to-back pass; items it leaves
// inconclusive go to the kind's deferred list (slots lo.. of dlist) for
// scene_resolve_kernel, so the pass runs with the registers and branch
// structure of the single-accel trace.
template <int KIND>
__global__ void __launch_bounds__(128)
scene_walk_kernel(SceneWork W, int phase) {
  const uint32_t *vals = phase ? W.vals1 : W.vals0;
  const uint32_t lo = *(volatile uint32_t *)&W.bounds[4 * phase + KIND];
  const uint32_t hi = *(volatile uint32_t *)&W.bounds[4 * phase + KIND + 1];
  uint32_t *fetch = &W.counters[4 + 3 * phase + KIND];
  uint32_t *dcount = &W.counters[10 + 3 * phase + KIND];
  const int lane = (int)(threadIdx.x & 31u);
  uint32_t c[4] = {0, 0, 0, 0};  // element walks, branch nodes, leaves, primitives
  while (true) {
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(fetch, 32u);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= hi - lo) break;
    const uint32_t k = lo + base + (uint32_t)lane;
    if (k < hi) {
      const uint32_t item = vals[k];
      uint32_t ray, slot;
      item_ray_slot(phase, item, ray, slot);
      const size_t cs = (size_t)ray * kRoundCand + slot;
      const uint32_t e_id = W.cand_e[cs];
      const SceneElem &e = W.elems[e_id];
      uint32_t prev_prim;
      float prev_t;
      const RayF r0 = load_ray(W.rays, ray, prev_prim, prev_t);
      double lo3[3], ld3[3];
      const auto ctx = elem_ctx<KIND>(W, ray, e_id, e, r0, prev_prim, prev_t, lo3, ld3);
      Best b;
      Work w;
      double m;
      bool full;
      const bool done = elem_pass1<KIND>(e, ctx, b, w, W.max_iter, m, full);
      c[0]++;
      c[1] += w.branch;
      c[2] += w.leaf;
      c[3] += w.prim;
      if (w.fail) atomicOr(W.err, kErrIter);
      if (done) {
        if constexpr (KIND == SRT_SPHERES) elem_sphere_uv(ctx, e, b);
        finish_item(W, phase, ray, cs, e_id, e, lo3, ld3, r0.o, b);
      } else {
        W.dlist[lo + atomicAdd(dcount, 1u)] = Deferred{item, full ? 1u : 0u, m};
      }
    }
  }
  if (W.stats) add_counts(W.stats, 1, c, 4);
}

// The deferred items of one kind: the replay, then the same result.
template <int KIND>
__global__ void __launch_bounds__(128)
scene_resolve_kernel(SceneWork W, int phase) {
  const uint32_t lo = *(volatile uint32_t *)&W.bounds[4 * phase + KIND];
  const uint32_t cnt = *(volatile uint32_t *)&W.counters[10 + 3 * phase + KIND];
  uint32_t c[4] = {0, 0, 0, 0};
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < cnt;
       k += gridDim.x * blockDim.x) {
    const Deferred d = W.dlist[lo + k];
    uint32_t ray, slot;
    item_ray_slot(phase, d.ray, ray, slot);
    const size_t cs = (size_t)ray * kRoundCand + slot;
    const uint32_t e_id = W.cand_e[cs];
    const SceneElem &e = W.elems[e_id];
    uint32_t prev_prim;
    float prev_t;
    const RayF r0 = load_ray(W.rays, ray, prev_prim, prev_t);
    double lo3[3], ld3[3];
    const auto ctx = elem_ctx<KIND>(W, ray, e_id, e, r0, prev_prim, prev_t, lo3, ld3);
    Best b;
    Work w;
    elem_replay<KIND>(e, ctx, b, w, W.max_iter, d.m, d.full != 0);
    c[1] += w.branch;
    c[2] += w.leaf;
    c[3] += w.prim;
    if (w.fail) atomicOr(W.err, kErrIter);
    if constexpr (KIND == SRT_SPHERES) elem_sphere_uv(ctx, e, b);
    finish_item(W, phase, ray, cs, e_id, e, lo3, ld3, r0.o, b);
  }
  if (W.stats) add_counts(W.stats, 1, c, 4);
}

// Closest hit of ray i in element e_id: pass and, if needed, replay (the
// loop kernel's per-candidate walk).  Local ray in lo / ld.
template <int KIND>
__device__ __forceinline__ bool elem_hit(const SceneWork &W, uint32_t i, uint32_t e_id,
                                         const SceneElem &e, const RayF &r0, uint32_t prev_prim,
                                         float prev_t, double lo[3], double ld[3], Best &b,
                                         Work &w) {
  const auto ctx = elem_ctx<KIND>(W, i, e_id, e, r0, prev_prim, prev_t, lo, ld);
  double m;
  bool full;
  if (!elem_pass1<KIND>(e, ctx, b, w, W.max_iter, m, full)) elem_replay<KIND>(e, ctx, b, w, W.max_iter, m, full);
  if (w.fail) atomicOr(W.err, kErrIter);
  if constexpr (KIND == SRT_SPHERES) elem_sphere_uv(ctx, e, b);
  return b.t < FLT_MAX && b.prim != kNone;
}

// Phase 1 keys, dense per ray: the element rank of every later candidate
// whose entry does not lie beyond the nearest hit of phase 0 (the
// candidates are sorted, so the first culled one ends them), none (nelem)
// for the rest.  The sequential loop walks a subset of these: its nearest
// distance only shrinks.
__global__ void __launch_bounds__(128)
scene_gather_kernel(SceneWork W) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= W.n) return;
  const uint32_t nc = W.ncand[i];
  const double tn = (double)W.tnear[i];
  bool live = true;
#pragma unroll
  for (uint32_t c = 1; c < (uint32_t)kRoundCand; c++) {
    const size_t cs = i * kRoundCand + c;
    uint32_t key = W.nelem;
    if (live && c < nc) {
      if (tn < W.cand_t[cs]) live = false;
      else key = __ldg(&W.elem_rank[W.cand_e[cs]]);
    }
    W.keys1[i * (kRoundCand - 1) + (c - 1)] = key;
  }
}

// The sequential rule over candidates 1.. of each ray, from the phase-0
// best: skip a candidate entered beyond the nearest hit, take a strictly
// nearer hit.
__global__ void __launch_bounds__(128)
scene_select_kernel(SceneWork W) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= W.n) return;
  const uint32_t nc = W.ncand[i];
  if (nc < 2) return;
  float tn = W.tnear[i];
  int best = -1;
  float4 bh = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  for (uint32_t c = 1; c < nc; c++) {
    const size_t cs = i * kRoundCand + c;
    if ((double)tn < W.cand_t[cs]) break;
    const float4 r = W.res[cs];
    if (__float_as_uint(r.w) != kNone && r.x < tn) {
      tn = r.x;
      bh = r;
      best = (int)c;
    }
  }
  if (best >= 0) {
    reinterpret_cast<float4 *>(W.hits)[i] = bh;
    if (W.element) W.element[i] = W.cand_e[i * kRoundCand + best];
  }
}

// Closest hit of a local ray in a line element (LineAccel::Traverse; the
// reference's line walk has no self-hit rule).  LSTACK: the walk's stack.
template <int LSTACK>
__device__ __forceinline__ bool elem_hit_lines(const SceneElem &e, const RayF &lr, Best &b,
                                               uint32_t c[4]) {
  using namespace srt_line_walk;
  const RayL R = make_ray(lr.o, lr.d);
  unsigned long long nb = 0, nl = 0, nt = 0;
  const LineHit H = line_walk<LSTACK, true>(static_cast<const LNode *>(e.nodes),
                                            reinterpret_cast<const LineRec *>(e.prims),
                                            e.aux != 0, R, nb, nl, nt);
  c[1] += (uint32_t)nb;
  c[2] += (uint32_t)nl;
  c[3] += (uint32_t)nt;
  if (H.rec < 0) return false;
  b.t = H.t;
  b.u = H.u;
  b.v = H.v;
  b.prim = __ldg(&reinterpret_cast<const LineRec *>(e.prims)[H.rec].prim);
  return true;
}

// Closest hit of a local ray in a solid element (SolidAccel::Traverse, the
// previous solid skipped inside the element the ray left): u = v = 0.
// STACK: the walk's stack.
template <int STACK>
__device__ __forceinline__ bool elem_hit_solids(const SceneElem &e, const RayF &lr,
                                                uint32_t prev, Best &b, uint32_t *err) {
  using namespace srt_solid_walk;
  const SNode *nodes = static_cast<const SNode *>(e.nodes);
  const void *recs = e.prims;
  float t, bp[3], bn[3];
  uint32_t prim;
  bool ok;
  const int nv = e.aux & 255;
  if (e.aux & kSolidAuxDouble) {
    if (nv == 5)
      ok = solid_walk<5, STACK, double>(nodes, recs, lr.o, lr.d, prev, t, prim, bp, bn);
    else if (nv == 6)
      ok = solid_walk<6, STACK, double>(nodes, recs, lr.o, lr.d, prev, t, prim, bp, bn);
    else
      ok = solid_walk<8, STACK, double>(nodes, recs, lr.o, lr.d, prev, t, prim, bp, bn);
  } else if (nv == 5) {
    ok = solid_walk<5, STACK>(nodes, recs, lr.o, lr.d, prev, t, prim, bp, bn);
  } else if (nv == 6) {
    ok = solid_walk<6, STACK>(nodes, recs, lr.o, lr.d, prev, t, prim, bp, bn);
  } else {
    ok = solid_walk<8, STACK>(nodes, recs, lr.o, lr.d, prev, t, prim, bp, bn);
  }
  if (!ok) atomicOr(err, kErrStack);
  if (!(t < FLT_MAX)) return false;
  b.t = t;
  b.u = b.v = 0.0f;
  b.prim = prim;
  return true;
}

// The whole loop in one thread, for the rays with more candidates than
// the per-ray slots hold and the rays that meet a line or solid element.
// LSTACK: the line and solid walks' stack (the deepest such tree + 2 at
// least).
template <int LSTACK>
__global__ void __launch_bounds__(128)
scene_loop_kernel(const TopNode *__restrict__ top, SceneWork W) {
  const uint32_t cnt = *(volatile uint32_t *)&W.counters[2];
  uint32_t c[4] = {0, 0, 0, 0};
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < cnt;
       k += gridDim.x * blockDim.x) {
    const uint32_t i = W.ovf[k];
    uint32_t prev_prim;
    float prev_t;
    const RayF r0 = load_ray(W.rays, i, prev_prim, prev_t);
    const double ro[3] = {r0.o[0], r0.o[1], r0.o[2]}, rd[3] = {r0.d[0], r0.d[1], r0.d[2]};
    double ct[kTopCand];
    uint32_t cid[kTopCand];
    uint32_t ntop = 0;
    const int nc = top_candidates(top, ro, rd, ct, cid, W.max_iter, ntop, W.err);
    double tnear = DBL_MAX;
    float bt = FLT_MAX, bu = 0.0f, bv = 0.0f;
    uint32_t bp = kNone, be = kNone;
    for (int q = 0; q < nc; q++) {
      if (tnear < ct[q]) continue;
      const SceneElem &e = W.elems[cid[q]];
      double lo[3], ld[3];
      Best b;
      Work w;
      bool hit;
      if (e.kind >= kSceneLines) {
        const double ro3[3] = {r0.o[0], r0.o[1], r0.o[2]}, rd3[3] = {r0.d[0], r0.d[1], r0.d[2]};
        const RayF lr = local_ray(e, ro3, rd3, lo, ld);
        const bool same = W.prev_element && __ldg(&W.prev_element[i]) == cid[q];
        hit = e.kind == kSceneLines
                  ? elem_hit_lines<LSTACK>(e, lr, b, c)
                  : elem_hit_solids<LSTACK>(e, lr, same ? prev_prim : kNone, b, W.err);
      } else if (e.kind == SRT_TETRAHEDRA)
        hit = elem_hit<SRT_TETRAHEDRA>(W, i, cid[q], e, r0, prev_prim, prev_t, lo, ld, b, w);
      else if (e.kind == SRT_TRIANGLES)
        hit = elem_hit<SRT_TRIANGLES>(W, i, cid[q], e, r0, prev_prim, prev_t, lo, ld, b, w);
      else
        hit = elem_hit<SRT_SPHERES>(W, i, cid[q], e, r0, prev_prim, prev_t, lo, ld, b, w);
      c[0]++;
      c[1] += w.branch;
      c[2] += w.leaf;
      c[3] += w.prim;
      if (!hit) continue;
      const float tw = world_dist(e, lo, ld, b.t, r0.o);
      if ((double)tw < tnear) {
        tnear = tw;
        bt = tw;
        bu = b.u;
        bv = b.v;
        bp = b.prim;
        be = cid[q];
      }
    }
    reinterpret_cast<float4 *>(W.hits)[i] = make_float4(bt, bu, bv, __uint_as_float(bp));
    if (W.element) W.element[i] = be;
  }
  if (W.stats) add_counts(W.stats, 1, c, 4);
}

// Resident blocks per SM of the persistent kernels (the same on every device
// of one architecture): walks of the three kinds, loop (short and long line
// stack).
int g_per_sm[5] = {1, 1, 1, 1, 1};
std::once_flag g_per_sm_once;

void scene_occupancy() {
  const void *fn[5] = {(const void *)scene_walk_kernel<SRT_TRIANGLES>,
                       (const void *)scene_walk_kernel<SRT_TETRAHEDRA>,
                       (const void *)scene_walk_kernel<SRT_SPHERES>,
                       (const void *)scene_loop_kernel<64>,
                       (const void *)scene_loop_kernel<520>};
  for (int k = 0; k < 5; k++) {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn[k], 128, 0);
    g_per_sm[k] = per_sm > 0 ? per_sm : 1;
  }
}

}  // namespace

template <int KIND>
static void launch_kind(srt_ctx *ctx, const SceneWork &W, int phase, cudaStream_t st) {
  scene_walk_kernel<KIND><<<(unsigned)(ctx->num_sms * g_per_sm[KIND]), 128, 0, st>>>(W, phase);
  scene_resolve_kernel<KIND><<<(unsigned)(ctx->num_sms * 4), 128, 0, st>>>(W, phase);
  ctx->launches += 2;
}

srt_status launch_scene_trace(srt_ctx *ctx, const TopNode *top, SceneWork W, uint32_t kinds,
                              bool deep_lines, const SceneStreams &ss) {
  if (W.n == 0) return SRT_OK;
  cudaStream_t st = ctx->stream;
  cudaError_t e = cudaMemsetAsync(W.counters, 0, kSceneCounters * sizeof(uint32_t), st);
  if (e != cudaSuccess) return cuda_status(e, "scene counters");
  std::call_once(g_per_sm_once, scene_occupancy);
  const unsigned rgrid = (unsigned)((W.n + 127) / 128);
  int kb = 1;  // key bits: ranks 0..nelem-1 and none = nelem
  while ((1u << kb) <= W.nelem) kb++;
  scene_top_kernel<<<rgrid, 128, 0, st>>>(top, W);
  ctx->launches++;
  // the rays with more candidates than slots run their loop alongside
  cudaEventRecord(ss.fork[0], st);
  cudaStreamWaitEvent(ss.side[3], ss.fork[0], 0);
  if (deep_lines)
    scene_loop_kernel<520><<<(unsigned)(ctx->num_sms * g_per_sm[4]), 128, 0, ss.side[3]>>>(top, W);
  else
    scene_loop_kernel<64><<<(unsigned)(ctx->num_sms * g_per_sm[3]), 128, 0, ss.side[3]>>>(top, W);
  ctx->launches++;
  cudaEventRecord(ss.join[3], ss.side[3]);
  for (int phase = 0; phase < 2; phase++) {
    if (phase == 1) {
      scene_gather_kernel<<<rgrid, 128, 0, st>>>(W);
      ctx->launches++;
    }
    // items in (element rank, ray) order: a stable sort of the dense keys
    srt_status s = phase ? sort_pairs(ctx, W.keys1, W.vals1, W.n * (kRoundCand - 1), true, kb)
                         : sort_pairs(ctx, W.keys0, W.vals0, W.n, true, kb);
    if (s != SRT_OK) return s;
    scene_range_kernel<<<1, 32, 0, st>>>(W, phase);
    ctx->launches++;
    // each kind's walks and replays on its own stream
    cudaEventRecord(ss.fork[1 + phase], st);
    for (int k = 0; k < 3; k++) {
      if (!(kinds & (1u << k))) continue;
      cudaStreamWaitEvent(ss.side[k], ss.fork[1 + phase], 0);
      if (k == SRT_TRIANGLES)
        launch_kind<SRT_TRIANGLES>(ctx, W, phase, ss.side[k]);
      else if (k == SRT_SPHERES)
        launch_kind<SRT_SPHERES>(ctx, W, phase, ss.side[k]);
      else
        launch_kind<SRT_TETRAHEDRA>(ctx, W, phase, ss.side[k]);
      cudaEventRecord(ss.join[k], ss.side[k]);
      cudaStreamWaitEvent(st, ss.join[k], 0);
    }
  }
  scene_select_kernel<<<rgrid, 128, 0, st>>>(W);
  ctx->launches++;
  cudaStreamWaitEvent(st, ss.join[3], 0);
  return cuda_status(cudaGetLastError(), "scene trace");
}

}  // namespace srt

// ======================================================= no-allocation trace
// srt_trace_closest_noalloc runs the same two kernels as srt_trace_closest
// (first pass + deferred-ray resolve) but keeps its deferred-ray list in the
// fixed device array below instead of the context's growable scratch, so a
// call allocates no device or host memory.
//
// Layout of g_noalloc_scratch: bytes [0, 256) are the header, whose first
// uint32 is the deferred-ray count.  That count must be zero when the first
// kernel starts; every call clears it itself (cudaMemsetAsync on the
// context's stream) before its first launch.  Records of 16 bytes follow at
// byte 256, one per deferred ray, at most kNoAllocMaxRays of them (4 MiB).
// The rest of the array needs no initial value.
//
// The array is one per device and shared by every context and stream on that
// device: two calls whose kernels overlap in time (different streams, or
// different host threads without ordering) race on it and may return wrong
// hits.  Order such calls on one stream or synchronise between them.
namespace srt {
namespace {

constexpr size_t kNoAllocMaxRays = 262144;
constexpr size_t kNoAllocHeader = 256;
constexpr int kNoAllocMaxDevices = 64;

__device__ __align__(256) unsigned char
    g_noalloc_scratch[kNoAllocHeader + kNoAllocMaxRays * sizeof(Deferred)];

std::mutex g_noalloc_mu;
void *g_noalloc_base[kNoAllocMaxDevices];

// Device address of g_noalloc_scratch on the current device, looked up once
// per device (the lookup is the set-up: it may load this module's device
// code on that device).
srt_status noalloc_scratch(int device, unsigned char **out) {
  if (device < 0 || device >= kNoAllocMaxDevices) {
    set_error("device ordinal out of range for the no-allocation scratch");
    return SRT_ERR_INVALID;
  }
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_base[device]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) return cuda_status(e, "no-allocation scratch set-up");
    g_noalloc_base[device] = p;
  }
  *out = static_cast<unsigned char *>(g_noalloc_base[device]);
  return SRT_OK;
}

}  // namespace
}  // namespace srt

extern "C" SRT_API srt_status srt_trace_closest_noalloc(srt_accel *a, const srt_ray *rays,
                                                        size_t n, srt_hit *hits) {
  using namespace srt;
  if (!a || (!rays && n) || (!hits && n)) {
    set_error("NULL argument");
    return SRT_ERR_INVALID;
  }
  if (!a->built) {
    set_error("accel not built");
    return SRT_ERR_INVALID;
  }
  if (n > kNoAllocMaxRays) {
    set_error("srt_trace_closest_noalloc: at most 262144 rays per call; split the ray array");
    return SRT_ERR_LIMIT;
  }
  if (n == 0) return SRT_OK;
  srt_ctx *ctx = a->ctx;
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_status(e, "set device");
  if (!is_device_ptr(rays) || !is_device_ptr(hits)) {
    set_error("srt_trace_closest_noalloc: rays and hits must be device memory");
    return SRT_ERR_INVALID;
  }
  if ((reinterpret_cast<uintptr_t>(rays) | reinterpret_cast<uintptr_t>(hits)) & 15u) {
    set_error("ray and hit arrays must be 16-byte aligned");
    return SRT_ERR_INVALID;
  }
  unsigned char *base = nullptr;
  srt_status s = noalloc_scratch(ctx->device, &base);
  if (s != SRT_OK) return s;
  uint32_t *dcount = reinterpret_cast<uint32_t *>(base);
  Deferred *dlist = reinterpret_cast<Deferred *>(base + kNoAllocHeader);
  cudaStream_t st = ctx->stream;
  if ((e = cudaMemsetAsync(dcount, 0, 4, st)) != cudaSuccess)
    return cuda_status(e, "deferred count");
  const int block = 128;
  const unsigned grid = (unsigned)((n + block - 1) / block);
  const unsigned rgrid = (unsigned)ctx->num_sms * 8;
  const uint32_t max_iter = (uint32_t)std::min<size_t>(8 * a->n + 64, 0xfffffff0u);
  const SceneInfo *scene = a->scene.as<SceneInfo>();
  const float4 *pr = a->prims.as<float4>();
  const uint32_t *ix = a->indices.as<uint32_t>();
  switch (a->kind) {
    case SRT_TRIANGLES: {
      const Node2 *nd = a->nodes.as<Node2>();
      trace_node2_kernel<SRT_TRIANGLES, false><<<grid, block, 0, st>>>(
          nd, pr, ix, rays, n, hits, scene, nullptr, nullptr, nullptr, dlist, dcount, max_iter,
          ctx->d_err, nullptr);
      resolve_node2_kernel<SRT_TRIANGLES><<<rgrid, block, 0, st>>>(
          nd, pr, ix, rays, hits, scene, nullptr, nullptr, nullptr, dlist, dcount, max_iter,
          ctx->d_err);
      break;
    }
    case SRT_SPHERES: {
      const Node2 *nd = a->nodes.as<Node2>();
      trace_node2_kernel<SRT_SPHERES, false><<<grid, block, 0, st>>>(
          nd, pr, ix, rays, n, hits, scene, nullptr, nullptr, nullptr, dlist, dcount, max_iter,
          ctx->d_err, nullptr);
      resolve_node2_kernel<SRT_SPHERES><<<rgrid, block, 0, st>>>(
          nd, pr, ix, rays, hits, scene, nullptr, nullptr, nullptr, dlist, dcount, max_iter,
          ctx->d_err);
      break;
    }
    case SRT_TETRAHEDRA: {
      if (a->dbl) {
        set_error("srt_trace_closest_noalloc: double-precision tetrahedra take srt_trace_closest");
        return SRT_ERR_UNSUPPORTED;
      }
      const NodeT *nd = a->nodes.as<NodeT>();
      trace_tet_kernel<false><<<grid, block, 0, st>>>(nd, pr, ix, rays, n, hits, nullptr,
                                                      a->src_faces, nullptr, nullptr, nullptr,
                                                      dlist, dcount, max_iter, ctx->d_err, nullptr);
      resolve_tet_kernel<<<rgrid, block, 0, st>>>(nd, pr, ix, rays, hits, nullptr, a->src_faces,
                                                  nullptr, nullptr, nullptr, dlist, dcount,
                                                  max_iter, ctx->d_err);
      break;
    }
  }
  ctx->launches += 2;
  return cuda_status(cudaGetLastError(), "trace (no allocation)");
}
