// srt_walks.cuh -- device records and per-ray tests of the line and solid
// accels, shared by their own trace kernels (srt_line.cu, srt_solid.cu) and
// the scene trace's per-ray loop (srt_trace.cu), which walks line and solid
// elements of a render graph.
#pragma once

#include <cfloat>
#include <cstdint>

// ------------------------------------------------------------------ lines
namespace srt_line_walk {

// Device node: w1 bit 31 set for a leaf (w0 = first record, the low bits = count),
// else w0 = left child, w1 = right child | axis << 29.
struct alignas(16) LNode {
  float bmin[3];
  uint32_t w0;
  float bmax[3];
  uint32_t w1;
};
static_assert(sizeof(LNode) == 32, "two 16-byte loads");

// One line in leaf order: the terms of CylinderIsect that do not depend on
// the ray.  dn0 = normalize(p0 - p1); p0D = -dot(p0, dn0); p1D = -dot(p1, -dn0).
struct alignas(16) LineRec {
  float p0[3], rr;
  float p1[3], dd;
  float dn0[3], p0D;
  float p1D;
  uint32_t prim;
  float pad[2];
};
static_assert(sizeof(LineRec) == 64, "four 16-byte loads");

constexpr uint32_t kLineLeaf = 0x80000000u;
constexpr float kCapEps = 1.0e-6f;  // the file-level kEPS of render_accel_line.cc

__device__ __forceinline__ float dot3(const float a[3], const float b[3]) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

// vnormalize (:439-454): (float)sqrt((double)x) is the float sqrt and
// (float)(1.0 / (double)len) the float reciprocal, both correctly rounded.
__device__ __forceinline__ void normalize3(const float a[3], float out[3]) {
  const float len = __fsqrt_rn(dot3(a, a));
  out[0] = a[0];
  out[1] = a[1];
  out[2] = a[2];
  if (len > FLT_EPSILON * 16.0f) {
    const float inv = __frcp_rn(len);
    out[0] *= inv;
    out[1] *= inv;
    out[2] *= inv;
  }
}

__device__ __forceinline__ LineRec load_line(const LineRec *p) {
  const float4 *q = reinterpret_cast<const float4 *>(p);
  const float4 a = __ldg(q), b = __ldg(q + 1), c = __ldg(q + 2), d = __ldg(q + 3);
  LineRec r;
  r.p0[0] = a.x;
  r.p0[1] = a.y;
  r.p0[2] = a.z;
  r.rr = a.w;
  r.p1[0] = b.x;
  r.p1[1] = b.y;
  r.p1[2] = b.z;
  r.dd = b.w;
  r.dn0[0] = c.x;
  r.dn0[1] = c.y;
  r.dn0[2] = c.z;
  r.p0D = c.w;
  r.p1D = d.x;
  r.prim = __float_as_uint(d.y);
  return r;
}

struct RayL {
  float org[3], dir[3], rd[3], inv[3], nn;
  int sign[3];
};

// CylinderIsect (:488-577) for one line record; *pt is the closest hit so
// far (updated on a hit, as the reference does through its pointer).
__device__ __forceinline__ bool cyl_isect(const LineRec &L, const RayL &R, bool cap, float *pt,
                                          float *pu, float *pv, bool &hit_cap) {
  const float tmax = *pt;
  float d[3], m[3];
  for (int k = 0; k < 3; k++) {
    d[k] = L.p1[k] - L.p0[k];
    m[k] = R.org[k] - L.p0[k];
  }
  const float md = dot3(m, d), nd = dot3(R.dir, d), dd = L.dd, rr = L.rr;
  hit_cap = false;
  float capT = FLT_MAX;
  if (cap && fabsf(dot3(R.dir, L.dn0)) > kCapEps) {
    const float dn1[3] = {-L.dn0[0], -L.dn0[1], -L.dn0[2]};
    const float p0T = -(dot3(R.org, L.dn0) + L.p0D) / dot3(R.rd, L.dn0);
    const float p1T = -(dot3(R.org, dn1) + L.p1D) / dot3(R.rd, dn1);
    float a0[3], a1[3];
    for (int k = 0; k < 3; k++) {
      a0[k] = (R.org[k] + R.rd[k] * p0T) - L.p0[k];
      a1[k] = (R.org[k] + R.rd[k] * p1T) - L.p1[k];
    }
    const float s0 = dot3(a0, a0), s1 = dot3(a1, a1);
    if (p0T > 0.0f && p0T < tmax && s0 < rr * rr) {
      hit_cap = true;
      capT = p0T;
      *pt = capT;
      *pu = __fsqrt_rn(s0);
      *pv = 0.0f;
    }
    if (p1T > 0.0f && p1T < tmax && p1T < capT && s1 < rr * rr) {
      hit_cap = true;
      capT = p1T;
      *pt = capT;
      *pu = __fsqrt_rn(s1);
      *pv = 1.0f;
    }
  }
  if (md <= 0.0f && nd <= 0.0f) return hit_cap;
  if (md >= dd && nd >= 0.0f) return hit_cap;
  const float mn = dot3(m, R.dir);
  const float A = dd * R.nn - nd * nd;
  const float kk = dot3(m, m) - rr * rr;
  const float C = dd * kk - md * md;
  const float B = dd * mn - nd * md;
  // solve2e (:456-486), the smaller root
  float t;
  if (fabsf(A) <= FLT_EPSILON) {
    t = -C / B;
  } else {
    const float D = B * B - A * C;
    if (D < 0.0f) return hit_cap;
    if (D == 0.0f) {
      t = -B / A;
    } else {
      float x1 = (float)(((double)fabsf(B) + sqrt((double)D)) / (double)A);
      if (B >= 0.0f) x1 = -x1;
      const float x2 = C / (A * x1);
      t = x1 > x2 ? x2 : x1;
    }
  }
  if (0.0f <= t && t <= tmax && t <= capT) {
    float s = md + t * nd;
    s /= dd;
    if (0.0f <= s && s <= 1.0f) {
      hit_cap = false;
      *pt = t;
      *pu = 0.0f;
      *pv = s;
      return true;
    }
  }
  return hit_cap;
}

// IntersectRayAABB (:377-420) with the reference's selection order.
__device__ __forceinline__ bool box_hit(const LNode &nd, const RayL &R, float maxT) {
  float lo[3], hi[3];
  for (int k = 0; k < 3; k++) {
    lo[k] = R.sign[k] ? nd.bmax[k] : nd.bmin[k];
    hi[k] = R.sign[k] ? nd.bmin[k] : nd.bmax[k];
  }
  const float tx0 = (lo[0] - R.org[0]) * R.inv[0], tx1 = (hi[0] - R.org[0]) * R.inv[0];
  const float ty0 = (lo[1] - R.org[1]) * R.inv[1], ty1 = (hi[1] - R.org[1]) * R.inv[1];
  float tmin = (tx0 > ty0) ? tx0 : ty0;
  float tmax = (tx1 < ty1) ? tx1 : ty1;
  const float tz0 = (lo[2] - R.org[2]) * R.inv[2], tz1 = (hi[2] - R.org[2]) * R.inv[2];
  tmin = (tmin > tz0) ? tmin : tz0;
  tmax = (tmax < tz1) ? tmax : tz1;
  return (tmax > 0.0f) && (tmin <= tmax) && (tmin <= maxT);
}

__device__ __forceinline__ LNode load_node(const LNode *p) {
  const float4 *q = reinterpret_cast<const float4 *>(p);
  const float4 a = __ldg(q), b = __ldg(q + 1);
  LNode n;
  n.bmin[0] = a.x;
  n.bmin[1] = a.y;
  n.bmin[2] = a.z;
  n.w0 = __float_as_uint(a.w);
  n.bmax[0] = b.x;
  n.bmax[1] = b.y;
  n.bmax[2] = b.z;
  n.w1 = __float_as_uint(b.w);
  return n;
}


// The ray's terms of the walk: sign, reciprocal, unit direction, |dir|^2.
__device__ __forceinline__ RayL make_ray(const float org[3], const float dir[3]) {
  RayL R;
  for (int k = 0; k < 3; k++) {
    R.org[k] = org[k];
    R.dir[k] = dir[k];
    R.sign[k] = dir[k] < 0.0f ? 1 : 0;
    R.inv[k] = __frcp_rn(dir[k]);  // (float)(1.0 / dir), correctly rounded
  }
  normalize3(R.dir, R.rd);
  R.nn = dot3(R.dir, R.dir);
  return R;
}

// The nearest line hit of a ray and the walk's counts.
struct LineHit {
  float t = FLT_MAX, u = 0.0f, v = 0.0f;
  bool cap = false;
  int rec = -1;  // record (leaf order) of the hit, -1: none
};

// LineAccel::Traverse (:733-765) for one ray, one thread: near child
// first, boxes culled by the nearest hit so far, every line of an entered
// leaf tested.  STACK: entries of the node stack (tree depth + 2 at least).
// nb / nl / nt count branch nodes, leaves and line tests when STATS.
template <int STACK, bool STATS>
__device__ __forceinline__ LineHit line_walk(const LNode *__restrict__ nodes,
                                             const LineRec *__restrict__ recs, bool cap,
                                             const RayL &R, unsigned long long &nb,
                                             unsigned long long &nl, unsigned long long &nt) {
  LineHit H;
  float hitT = FLT_MAX;
  int stack[STACK];
  int sp = 0;
  stack[0] = 0;
  while (sp >= 0) {
    const LNode nd = load_node(nodes + stack[sp]);
    sp--;
    if (!(nd.w1 & kLineLeaf)) {
      if (STATS) nb++;
      if (box_hit(nd, R, hitT)) {
        const int axis = (int)(nd.w1 >> 29);
        const int right = (int)(nd.w1 & 0x1fffffffu), left = (int)nd.w0;
        const int nearc = R.sign[axis];
        stack[++sp] = nearc ? left : right;  // far
        stack[++sp] = nearc ? right : left;  // near
      }
    } else {
      float t = H.t;
      bool any = false;
      const uint32_t first = nd.w0, cnt = nd.w1 & ~kLineLeaf;
      if (STATS) {
        nl++;
        nt += cnt;
      }
      for (uint32_t j = 0; j < cnt; j++) {
        const LineRec L = load_line(recs + first + j);
        float u, v;
        bool hc;
        if (cyl_isect(L, R, cap, &t, &u, &v, hc)) {
          H.t = t;
          H.u = u;
          H.v = v;
          H.cap = hc;
          H.rec = (int)(first + j);
          any = true;
        }
      }
      if (any) hitT = H.t;
    }
  }
  return H;
}

}  // namespace srt_line_walk

// ------------------------------------------------------------------ solids
namespace srt_solid_walk {

// Device node: w1 bit 31 set for a leaf (w0 = first record, low bits = count),
// else w0 = left child, w1 = right child | axis << 29.
struct alignas(16) SNode {
  float bmin[3];
  uint32_t w0;
  float bmax[3];
  uint32_t w1;
};
static_assert(sizeof(SNode) == 32, "two 16-byte loads");

constexpr uint32_t kSolidLeaf = 0x80000000u;

// floats per record: nv vertices (xyz) and the solid's index, padded to 16 bytes
__host__ __device__ constexpr int rec_floats(int nv) { return ((3 * nv + 1) + 3) / 4 * 4; }
// The same for double-precision positions: doubles per record (nv vertices,
// then the solid's index in the low word of one more double), padded to 16
// bytes.
__host__ __device__ constexpr int rec_doubles(int nv) { return ((3 * nv + 1) + 1) / 2 * 2; }
// Bytes of one record of scalar type T.
template <typename T>
__host__ __device__ constexpr int rec_bytes(int nv) {
  return sizeof(T) == 8 ? 8 * rec_doubles(nv) : 4 * rec_floats(nv);
}

// ------------------------------------------------------------------ trace
struct D3 {
  double x, y, z;
};
__device__ __forceinline__ D3 dsub(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ D3 dadd(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ D3 dscale(D3 a, double f) { return {a.x * f, a.y * f, a.z * f}; }
__device__ __forceinline__ D3 dcross(D3 a, D3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ double ddot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

// normalize (:85), then to float
__device__ __forceinline__ void s_unit(D3 a, float out[3]) {
  const double len = sqrt(a.x * a.x + a.y * a.y + a.z * a.z);
  out[0] = (float)(a.x / len);
  out[1] = (float)(a.y / len);
  out[2] = (float)(a.z / len);
}

__device__ __forceinline__ double comp(D3 a, int j) { return j == 0 ? a.x : (j == 1 ? a.y : a.z); }

// The crossing point of a face, every coordinate (FULL) or coordinate j
// only (out[j]; the one a hit's t is measured along).
// SetCrossPoint_Sq (double, :438-444): a quad face.
template <bool FULL>
__device__ __forceinline__ void s_quad(float out[3], int j, D3 v0, D3 v1, D3 v2, double ws0,
                                       double ws1, double ws2, double ws3, D3 e2, D3 e3,
                                       D3 dir) {
  const double w = ws2 + ws3 + ddot(dcross(e2, e3), dir);
  const double den = ws0 + ws1 + w;
  if (FULL) {
    const D3 p = dadd(dadd(dscale(v2, ws0), dscale(v0, ws1)), dscale(v1, w));
    out[0] = (float)(p.x / den);
    out[1] = (float)(p.y / den);
    out[2] = (float)(p.z / den);
  } else {
    const double pj = (comp(v2, j) * ws0 + comp(v0, j) * ws1) + comp(v1, j) * w;
    out[j] = (float)(pj / den);
  }
}

// A triangle face: the weighted sum in double, then the float vector
// divided by the float sum of the weights.
template <bool FULL>
__device__ __forceinline__ void s_tri(float out[3], int j, D3 a, double wa, D3 b, double wb,
                                      D3 c, double wc, double den) {
  const float f = (float)den;
  if (FULL) {
    const D3 p = dadd(dadd(dscale(a, wa), dscale(b, wb)), dscale(c, wc));
    out[0] = (float)p.x / f;
    out[1] = (float)p.y / f;
    out[2] = (float)p.z / f;
  } else {
    out[j] = (float)((comp(a, j) * wa + comp(b, j) * wb) + comp(c, j) * wc) / f;
  }
}

// Edges of each solid (GetEdges, :119-154): edge i = vertex hi[i] - vertex
// lo[i]; the Pluecker moment of edge i uses vertex i % MOD (:470).
template <int NV>
struct SolidTab;
template <>
struct SolidTab<5> {
  static constexpr int NE = 8, MOD = 4;
  __device__ static int hi(int i) {
    constexpr int t[8] = {1, 2, 3, 0, 4, 4, 4, 4};
    return t[i];
  }
  __device__ static int lo(int i) {
    constexpr int t[8] = {0, 1, 2, 3, 0, 1, 2, 3};
    return t[i];
  }
};
template <>
struct SolidTab<6> {
  static constexpr int NE = 9, MOD = 6;
  __device__ static int hi(int i) {
    constexpr int t[9] = {1, 2, 0, 4, 5, 3, 3, 4, 5};
    return t[i];
  }
  __device__ static int lo(int i) {
    constexpr int t[9] = {0, 1, 2, 3, 4, 5, 0, 1, 2};
    return t[i];
  }
};
template <>
struct SolidTab<8> {
  static constexpr int NE = 12, MOD = 8;
  __device__ static int hi(int i) {
    constexpr int t[12] = {1, 2, 3, 0, 5, 6, 7, 4, 4, 5, 6, 7};
    return t[i];
  }
  __device__ static int lo(int i) {
    constexpr int t[12] = {0, 1, 2, 3, 4, 5, 6, 7, 0, 1, 2, 3};
    return t[i];
  }
};

// One solid's vertices (floats or doubles, exactly as stored: T) read as
// doubles on use; edges are recomputed from them (the same double
// subtraction each time).
template <int NV, typename T = float>
struct SolidV {
  T x[NV][3];
  __device__ __forceinline__ D3 v(int k) const {
    return {(double)x[k][0], (double)x[k][1], (double)x[k][2]};
  }
  __device__ __forceinline__ D3 e(int i) const {
    return dsub(v(SolidTab<NV>::hi(i)), v(SolidTab<NV>::lo(i)));
  }
};

// ws[i] = dir . (e_i x v_{i % MOD}) + e_i . (dir x org) (:467-476)
template <int NV, typename T>
__device__ __forceinline__ void s_weights(const SolidV<NV, T> &S, D3 dir, D3 org,
                                          double (&ws)[SolidTab<NV>::NE]) {
  const D3 rpc = dcross(dir, org);
#pragma unroll
  for (int i = 0; i < SolidTab<NV>::NE; i++) {
    const D3 ei = S.e(i);
    ws[i] = ddot(dir, dcross(ei, S.v(i % SolidTab<NV>::MOD))) + ddot(ei, rpc);
  }
}

// The reference's Intersect{Pyramid,Prism,Hexa}D (:455-505, :559-611,
// :664-716) split in two.  face(ws, slot): the face its sign tests pick for
// crossing point `slot` (0 the first point, 1 the second; -1: the solid is
// missed).  point<FULL>(S, ws, face, ...): that face's crossing point (all
// of it and the face normal when FULL, else only coordinate j) by the same
// expressions.  A ray tests every solid's two points for t and forms the
// full point and normal only for a point that becomes its closest hit.
__device__ __forceinline__ bool s_cw(const double *ws, int side, int k) {
  return side == 0 ? ws[k] >= 0 : ws[k] <= 0;
}

template <int NV>
struct SolidFaces;

template <>
struct SolidFaces<5> {  // IntersectPyramidD: point n uses i = 1 - n
  __device__ static int face(const double (&ws)[8], int slot) {
    const int n = slot, i = 1 - slot;
    if (s_cw(ws, i, 0) && s_cw(ws, i, 1) && s_cw(ws, i, 2) && s_cw(ws, i, 3)) return 0;
    if (s_cw(ws, n, 0) && s_cw(ws, i, 4) && s_cw(ws, n, 5)) return 1;
    if (s_cw(ws, n, 1) && s_cw(ws, i, 5) && s_cw(ws, n, 6)) return 2;
    if (s_cw(ws, n, 2) && s_cw(ws, i, 6) && s_cw(ws, n, 7)) return 3;
    if (s_cw(ws, n, 3) && s_cw(ws, i, 7) && s_cw(ws, n, 4)) return 4;
    return -1;
  }
  template <bool FULL, typename T>
  __device__ static void point(const SolidV<5, T> &S, const double (&ws)[8], int f, D3 dir, int j,
                               float pos[3], float nrm[3]) {
    switch (f) {
      case 0:
        s_quad<FULL>(pos, j, S.v(0), S.v(1), S.v(2), ws[0], ws[1], ws[2], ws[3], S.e(2), S.e(3),
                     dir);
        if (FULL) s_unit(dcross(S.e(1), S.e(0)), nrm);
        break;
      case 1:
        s_tri<FULL>(pos, j, S.v(4), -ws[0], S.v(1), ws[4], S.v(0), -ws[5], -ws[0] + ws[4] - ws[5]);
        if (FULL) s_unit(dcross(S.e(4), S.e(0)), nrm);
        break;
      case 2:
        s_tri<FULL>(pos, j, S.v(4), -ws[1], S.v(2), ws[5], S.v(1), -ws[6], -ws[1] + ws[5] - ws[6]);
        if (FULL) s_unit(dcross(S.e(5), S.e(1)), nrm);
        break;
      case 3:
        s_tri<FULL>(pos, j, S.v(4), -ws[2], S.v(3), ws[6], S.v(2), -ws[7], -ws[2] + ws[6] - ws[7]);
        if (FULL) s_unit(dcross(S.e(6), S.e(2)), nrm);
        break;
      default:
        s_tri<FULL>(pos, j, S.v(4), -ws[3], S.v(0), ws[7], S.v(3), -ws[4], -ws[3] + ws[7] - ws[4]);
        if (FULL) s_unit(dcross(S.e(7), S.e(3)), nrm);
        break;
    }
  }
};

template <>
struct SolidFaces<6> {  // IntersectPrismD: point i uses n = 1 - i
  __device__ static int face(const double (&ws)[9], int slot) {
    const int i = slot, n = 1 - slot;
    if (s_cw(ws, n, 0) && s_cw(ws, n, 1) && s_cw(ws, n, 2)) return 0;
    if (s_cw(ws, i, 3) && s_cw(ws, i, 4) && s_cw(ws, i, 5)) return 1;
    if (s_cw(ws, i, 2) && s_cw(ws, i, 6) && s_cw(ws, n, 5) && s_cw(ws, n, 8)) return 2;
    if (s_cw(ws, i, 0) && s_cw(ws, i, 7) && s_cw(ws, n, 3) && s_cw(ws, n, 6)) return 3;
    if (s_cw(ws, i, 1) && s_cw(ws, i, 8) && s_cw(ws, n, 4) && s_cw(ws, n, 7)) return 4;
    return -1;
  }
  template <bool FULL, typename T>
  __device__ static void point(const SolidV<6, T> &S, const double (&ws)[9], int f, D3 dir, int j,
                               float pos[3], float nrm[3]) {
    switch (f) {
      case 0:
        s_tri<FULL>(pos, j, S.v(2), ws[0], S.v(0), ws[1], S.v(1), ws[2], ws[0] + ws[1] + ws[2]);
        if (FULL) s_unit(dcross(S.e(0), S.e(1)), nrm);
        break;
      case 1:
        s_tri<FULL>(pos, j, S.v(5), ws[3], S.v(3), ws[4], S.v(4), ws[5], ws[3] + ws[4] + ws[5]);
        if (FULL) s_unit(dcross(S.e(3), S.e(4)), nrm);
        break;
      case 2:
        s_quad<FULL>(pos, j, S.v(2), S.v(0), S.v(3), ws[2], ws[6], -ws[5], -ws[8], S.e(5),
                     S.e(8), dir);
        if (FULL) s_unit(dcross(S.e(2), S.e(6)), nrm);
        break;
      case 3:
        s_quad<FULL>(pos, j, S.v(0), S.v(1), S.v(4), ws[0], ws[7], -ws[3], -ws[6], S.e(3),
                     S.e(6), dir);
        if (FULL) s_unit(dcross(S.e(0), S.e(7)), nrm);
        break;
      default:
        s_quad<FULL>(pos, j, S.v(1), S.v(2), S.v(5), ws[1], ws[8], -ws[4], -ws[7], S.e(4),
                     S.e(7), dir);
        if (FULL) s_unit(dcross(S.e(1), S.e(8)), nrm);
        break;
    }
  }
};

template <>
struct SolidFaces<8> {  // IntersectHexaD: point i uses n = 1 - i
  __device__ static int face(const double (&ws)[12], int slot) {
    const int i = slot, n = 1 - slot;
    if (s_cw(ws, n, 0) && s_cw(ws, n, 1) && s_cw(ws, n, 2) && s_cw(ws, n, 3)) return 0;
    if (s_cw(ws, i, 4) && s_cw(ws, i, 5) && s_cw(ws, i, 6) && s_cw(ws, i, 7)) return 1;
    if (s_cw(ws, i, 0) && s_cw(ws, i, 9) && s_cw(ws, n, 4) && s_cw(ws, n, 8)) return 2;
    if (s_cw(ws, i, 1) && s_cw(ws, i, 10) && s_cw(ws, n, 5) && s_cw(ws, n, 9)) return 3;
    if (s_cw(ws, i, 2) && s_cw(ws, i, 11) && s_cw(ws, n, 6) && s_cw(ws, n, 10)) return 4;
    if (s_cw(ws, i, 3) && s_cw(ws, i, 8) && s_cw(ws, n, 7) && s_cw(ws, n, 11)) return 5;
    return -1;
  }
  template <bool FULL, typename T>
  __device__ static void point(const SolidV<8, T> &S, const double (&ws)[12], int f, D3 dir, int j,
                               float pos[3], float nrm[3]) {
    switch (f) {
      case 0:
        s_quad<FULL>(pos, j, S.v(0), S.v(1), S.v(2), ws[0], ws[1], ws[2], ws[3], S.e(2), S.e(3),
                     dir);
        if (FULL) s_unit(dcross(S.e(0), S.e(1)), nrm);
        break;
      case 1:
        s_quad<FULL>(pos, j, S.v(4), S.v(5), S.v(6), ws[4], ws[5], ws[6], ws[7], S.e(6), S.e(7),
                     dir);
        if (FULL) s_unit(dcross(S.e(4), S.e(5)), nrm);
        break;
      case 2:
        s_quad<FULL>(pos, j, S.v(0), S.v(1), S.v(5), ws[0], ws[9], -ws[4], -ws[8], S.e(4),
                     S.e(8), dir);
        if (FULL) s_unit(dcross(S.e(0), S.e(9)), nrm);
        break;
      case 3:
        s_quad<FULL>(pos, j, S.v(1), S.v(2), S.v(6), ws[1], ws[10], -ws[5], -ws[9], S.e(5),
                     S.e(9), dir);
        if (FULL) s_unit(dcross(S.e(1), S.e(10)), nrm);
        break;
      case 4:
        s_quad<FULL>(pos, j, S.v(2), S.v(3), S.v(7), ws[2], ws[11], -ws[6], -ws[10], S.e(6),
                     S.e(10), dir);
        if (FULL) s_unit(dcross(S.e(2), S.e(11)), nrm);
        break;
      default:
        s_quad<FULL>(pos, j, S.v(3), S.v(0), S.v(4), ws[3], ws[8], -ws[7], -ws[11], S.e(7),
                     S.e(11), dir);
        if (FULL) s_unit(dcross(S.e(3), S.e(8)), nrm);
        break;
    }
  }
};

// The full crossing point and normal of a hit that becomes a ray's closest
// (seldom: kept out of line so the test loop keeps its registers).
template <int NV, typename T>
__device__ __noinline__ void s_full_point(const SolidV<NV, T> &S,
                                          const double (&ws)[SolidTab<NV>::NE], int f, D3 dir,
                                          float pos[3], float nrm[3]) {
  SolidFaces<NV>::template point<true, T>(S, ws, f, dir, 0, pos, nrm);
}

// t of a crossing point along axis j (the last with |dir| > 0.1; none: 0),
// as the reference's parameter step computes it (:2280-2290).
__device__ __forceinline__ float s_t(float pj, int j, D3 org, D3 dir) {
  if (j < 0) return 0.0f;
  return (float)(((double)pj - comp(org, j)) / comp(dir, j));
}

// IntersectRayAABB (:2160-2204) with the reference's selection order.
__device__ __forceinline__ bool sbox_hit(const SNode &nd, const float org[3], const float inv[3],
                                         const int sign[3]) {
  float lo[3], hi[3];
  for (int k = 0; k < 3; k++) {
    lo[k] = sign[k] ? nd.bmax[k] : nd.bmin[k];
    hi[k] = sign[k] ? nd.bmin[k] : nd.bmax[k];
  }
  const float tx0 = (lo[0] - org[0]) * inv[0], tx1 = (hi[0] - org[0]) * inv[0];
  const float ty0 = (lo[1] - org[1]) * inv[1], ty1 = (hi[1] - org[1]) * inv[1];
  float tmin = (tx0 > ty0) ? tx0 : ty0;
  float tmax = (tx1 < ty1) ? tx1 : ty1;
  const float tz0 = (lo[2] - org[2]) * inv[2], tz1 = (hi[2] - org[2]) * inv[2];
  tmin = (tmin > tz0) ? tmin : tz0;
  tmax = (tmax < tz1) ? tmax : tz1;
  return (tmax > 0.0f) && (tmin <= tmax) && (tmin <= FLT_MAX);
}

// The reference's walk (render/render_accel_solid.cc:2345): near child first,
// every solid whose leaf box the ray enters tested (no culling by distance:
// a quad face's crossing point is an affine combination of its corners that
// can fall outside the solid's box, so a box entered beyond the running
// distance may still hold a nearer hit), the first of the smallest t kept.
// One solid (sorted record j) against a ray: the point nearer than t that
// the reference keeps (entry, then exit), its solid id, position and
// normal; a record whose id is the ray's previous primitive is skipped.
// jax: the last axis with |dir| > 0.1 (-1: none).
// recs: records of scalar type T (rec_floats / rec_doubles per solid).
template <int NV, typename T = float>
__device__ __forceinline__ void solid_test(const void *__restrict__ recs, uint32_t j,
                                           uint32_t prev, D3 dorg, D3 ddir, int jax, float &t,
                                           uint32_t &prim, float bp[3], float bn[3]) {
  SolidV<NV, T> S;
  uint32_t p;
  if constexpr (sizeof(T) == 8) {
    constexpr int RD = rec_doubles(NV);
    const double2 *r2 = reinterpret_cast<const double2 *>(recs) + (size_t)(RD / 2) * j;
    double rv[RD];
#pragma unroll
    for (int q = 0; q < RD / 2; q++) {
      const double2 v2 = __ldg(r2 + q);
      rv[2 * q] = v2.x;
      rv[2 * q + 1] = v2.y;
    }
    p = (uint32_t)__double_as_longlong(rv[3 * NV]);
    if (p == prev) return;  // Ray::prev_prim_id
#pragma unroll
    for (int c = 0; c < NV; c++)
#pragma unroll
      for (int e = 0; e < 3; e++) S.x[c][e] = rv[3 * c + e];
  } else {
    constexpr int RF = rec_floats(NV);
    const float4 *r4 = reinterpret_cast<const float4 *>(recs) + (size_t)(RF / 4) * j;
    float rv[RF];
#pragma unroll
    for (int q4 = 0; q4 < RF / 4; q4++) {
      const float4 v4 = __ldg(r4 + q4);
      rv[4 * q4] = v4.x;
      rv[4 * q4 + 1] = v4.y;
      rv[4 * q4 + 2] = v4.z;
      rv[4 * q4 + 3] = v4.w;
    }
    p = __float_as_uint(rv[3 * NV]);
    if (p == prev) return;  // Ray::prev_prim_id
#pragma unroll
    for (int c = 0; c < NV; c++)
#pragma unroll
      for (int e = 0; e < 3; e++) S.x[c][e] = rv[3 * c + e];
  }
  double ws[SolidTab<NV>::NE];
  s_weights<NV, T>(S, ddir, dorg, ws);
  const int f0 = SolidFaces<NV>::face(ws, 0);
  const int f1 = f0 < 0 ? -1 : SolidFaces<NV>::face(ws, 1);
  if (f1 < 0) return;
  float pt[3] = {0.0f, 0.0f, 0.0f}, nd3[3];
  float th[2];
#pragma unroll
  for (int h = 0; h < 2; h++) {
    if (jax >= 0)
      SolidFaces<NV>::template point<false, T>(S, ws, h ? f1 : f0, ddir, jax, pt, nd3);
    th[h] = s_t(jax >= 0 ? pt[jax] : 0.0f, jax, dorg, ddir);
  }
#pragma unroll
  for (int h = 0; h < 2; h++)
    if (th[h] >= 0.0f && th[h] < t) {
      t = th[h];
      prim = p;
      s_full_point<NV, T>(S, ws, h ? f1 : f0, ddir, bp, bn);
      if (h) {  // the second point's normal is flipped
#pragma unroll
        for (int c = 0; c < 3; c++) bn[c] = -1.0f * bn[c];
      }
    }
}

// SolidAccel::Traverse for one ray, one thread: the reference's walk (near
// child first, every solid of every entered leaf tested, no distance
// culling).  prim = 0xFFFFFFFF and t = FLT_MAX when nothing is hit.  STACK:
// the walk's stack (the tree's depth + 2 at least); returns false (the walk
// stopped) for a deeper tree.
template <int NV, int STACK, typename T = float>
__device__ __forceinline__ bool solid_walk(const SNode *__restrict__ nodes,
                                           const void *__restrict__ recs,
                                           const float org[3], const float dir[3],
                                           uint32_t prev, float &t, uint32_t &prim,
                                           float bp[3], float bn[3]) {
  int sign[3];
  float inv[3];
  int jax = -1;
#pragma unroll
  for (int c = 0; c < 3; c++) {
    sign[c] = dir[c] < 0.0f ? 1 : 0;
    inv[c] = __frcp_rn(dir[c]);
    if (dir[c] > 0.1 || dir[c] < -0.1) jax = c;
    bp[c] = bn[c] = 0.0f;
  }
  const D3 dorg = {org[0], org[1], org[2]}, ddir = {dir[0], dir[1], dir[2]};
  t = FLT_MAX;
  prim = 0xffffffffu;
  int stack[STACK];
  int sp = 0;
  stack[0] = 0;
  while (sp >= 0) {
    const float4 *q = reinterpret_cast<const float4 *>(nodes + stack[sp]);
    const float4 a = __ldg(q), b = __ldg(q + 1);
    sp--;
    const SNode nd = {{a.x, a.y, a.z}, __float_as_uint(a.w), {b.x, b.y, b.z},
                      __float_as_uint(b.w)};
    if (!sbox_hit(nd, org, inv, sign)) continue;
    if (!(nd.w1 & kSolidLeaf)) {
      const int axis = (int)(nd.w1 >> 29);
      const int right = (int)(nd.w1 & 0x1fffffffu), left = (int)nd.w0;
      const int nearc = sign[axis];
      if (sp + 2 >= STACK) return false;
      stack[++sp] = nearc ? left : right;  // far
      stack[++sp] = nearc ? right : left;  // near
      continue;
    }
    const uint32_t first = nd.w0, cnt = nd.w1 & ~kSolidLeaf;
    for (uint32_t j = first; j < first + cnt; j++)
      solid_test<NV, T>(recs, j, prev, dorg, ddir, jax, t, prim, bp, bn);
  }
  return true;
}

}  // namespace srt_solid_walk
