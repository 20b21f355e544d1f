/*
 * surface_oracle.c -- CPU restatement of SURFACE's ray-tracing core.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity oracle: it is linked by
 * the test-suite, by __graft_entry__.smoke() and by the CPU-baseline leg of
 * bench.py, and never by the product library (surface_b200/csrc).  It restates,
 * in plain C, the reference algorithms that the CUDA kernels must reproduce
 * bit-for-bit, each function citing the reference file:line it follows
 * (paths relative to the SURFACE source tree):
 *
 *   - scene bounding box       render/render_accel_triangle.cc:713-796 (eps 0),
 *                              render/render_accel_tetra.cc:973-1030 (eps 16 ulp),
 *                              render/render_accel_particle.cc:304-369 (radius+eps)
 *   - 30-bit Morton codes      render/render_prefix_tree_util.h:113-157,
 *                              render/render_prefix_tree_util.cc:151-304
 *   - stable LSD radix sort    render/render_prefix_tree_util.h:296-457
 *   - Karras radix tree        render/render_prefix_tree_util.cc:501-649
 *   - leaf collapse + emit     render/render_accel_triangle.cc:866-992,1389-1690
 *                              render/render_accel_tetra.cc:1113-1243,1579-1850
 *                              render/render_accel_particle.cc:521-661,1560-1866
 *   - closest-hit traversal    render/render_accel_triangle.cc:1815-1938,1994-2437,2511-2669
 *                              render/render_accel_tetra.cc:89-567,1934-2122,2200-2289
 *                              render/render_accel_particle.cc:1990-2035,2423-2834,3053-3218
 *   - shading records          render/render_accel_triangle.cc:2439-2507,
 *     (BuildIntersection)      render/render_accel_tetra.cc:148-241,2124-2196,
 *                              render/render_accel_particle.cc:2966-3049
 *   - trilinear 3D fetch       render/render_texture.cc:97-121,946-1058
 *   - volume march             examples/nonuniform_volume_render/input.frag:16-141
 *                              (camera, slab test, texel mapping); the
 *                              emission-absorption compositing, transfer-function
 *                              lookup and adjoint are defined here (the reference
 *                              only has a 64-step averaging march).
 *   - TinyMT64 generator       Saito & Matsumoto's published TinyMT64, used by the
 *                              reference tests as their fixture RNG
 *                              (test/cctest/test-prefix-tree.cc:10-23).
 *
 * Floating point: compile with -ffp-contract=off.  Every expression keeps the
 * reference's operand order and precision (float vs. double promotions) so that
 * results are identical to the reference build with g++ on x86-64.
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define SO_API __attribute__((visibility("default")))

enum { SO_TRI = 0, SO_TET = 1, SO_SPHERE = 2 };

/* ------------------------------------------------------------------------ */
/* TinyMT64 (fixture RNG of test/cctest/test-prefix-tree.cc:10-23)           */
/* ------------------------------------------------------------------------ */
typedef struct {
  uint64_t s0, s1;
  uint32_t mat1, mat2;
  uint64_t tmat;
} so_tinymt64;

static void tmt_step(so_tinymt64 *r) {
  uint64_t x;
  r->s0 &= UINT64_C(0x7fffffffffffffff);
  x = r->s0 ^ r->s1;
  x ^= x << 12;
  x ^= x >> 32;
  x ^= x << 32;
  x ^= x << 11;
  r->s0 = r->s1;
  r->s1 = x;
  if (x & 1) {
    r->s0 ^= (uint64_t)r->mat1;
    r->s1 ^= ((uint64_t)r->mat2) << 32;
  }
}

static uint64_t tmt_out(const so_tinymt64 *r) {
  uint64_t x = r->s0 + r->s1;
  x ^= r->s0 >> 8;
  if (x & 1) x ^= r->tmat;
  return x;
}

static void tmt_seed(so_tinymt64 *r, uint64_t seed) {
  uint64_t st[2];
  st[0] = seed ^ ((uint64_t)r->mat1 << 32);
  st[1] = (uint64_t)r->mat2 ^ r->tmat;
  for (int i = 1; i < 8; i++) {
    uint64_t p = st[(i - 1) & 1];
    st[i & 1] ^= (uint64_t)i + UINT64_C(6364136223846793005) * (p ^ (p >> 62));
  }
  if ((st[0] & UINT64_C(0x7fffffffffffffff)) == 0 && st[1] == 0) {
    st[0] = 'T';
    st[1] = 'M';
  }
  r->s0 = st[0];
  r->s1 = st[1];
}

/* n doubles in [0,1) with the parameter set the reference tests use. */
SO_API void so_tinymt64_doubles(uint64_t seed, uint32_t mat1, uint32_t mat2,
                                uint64_t tmat, size_t n, double *out) {
  so_tinymt64 r;
  r.mat1 = mat1;
  r.mat2 = mat2;
  r.tmat = tmat;
  tmt_seed(&r, seed);
  for (size_t i = 0; i < n; i++) {
    tmt_step(&r);
    out[i] = (double)tmt_out(&r) * (1.0 / 18446744073709551616.0);
  }
}

/* ------------------------------------------------------------------------ */
/* Morton codes                                                              */
/* ------------------------------------------------------------------------ */

/* Spread the low 10 bits of v so that bit k lands on bit 3k
 * (PartBy2_30, render/render_prefix_tree_util.h:113-120). */
static inline uint32_t spread10(uint32_t v) {
  v &= 0x3ffu;
  v = (v | (v << 16)) & 0x030000ffu;
  v = (v | (v << 8)) & 0x0300f00fu;
  v = (v | (v << 4)) & 0x030c30c3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}

SO_API uint32_t so_morton_bits(uint32_t ix, uint32_t iy, uint32_t iz) {
  return (spread10(ix) << 2) | (spread10(iy) << 1) | spread10(iz);
}

/* MortionCode30 (render/render_prefix_tree_util.h:143-157): quantise then
 * interleave.  The float->uint32 cast is left to the compiler exactly as the
 * reference writes it. */
static inline uint32_t morton_of(const float c[3], const float bmin[3],
                                 const float inv[3]) {
  uint32_t ix = (uint32_t)((c[0] - bmin[0]) * inv[0]);
  uint32_t iy = (uint32_t)((c[1] - bmin[1]) * inv[1]);
  uint32_t iz = (uint32_t)((c[2] - bmin[2]) * inv[2]);
  return so_morton_bits(ix, iy, iz);
}

/* inv = (float)1024 / (bmax - bmin) (render/render_prefix_tree_util.cc:235-238) */
static void morton_inv(const float bmin[3], const float bmax[3], float inv[3]) {
  int kdiv = 1 << 10;
  for (int k = 0; k < 3; k++) inv[k] = kdiv / (bmax[k] - bmin[k]);
}

SO_API void so_morton_points(const float *pts, size_t n, const float bmin[3],
                             const float bmax[3], uint32_t *codes) {
  float inv[3];
  morton_inv(bmin, bmax, inv);
  for (size_t i = 0; i < n; i++) codes[i] = morton_of(&pts[3 * i], bmin, inv);
}

/* CalculateMortonCodesTriangleFloat30 (render/render_prefix_tree_util.cc:230-265) */
SO_API void so_morton_tris(const float *v, const uint32_t *f, size_t n,
                           const float bmin[3], const float bmax[3],
                           uint32_t *codes) {
  float inv[3];
  morton_inv(bmin, bmax, inv);
  const float one_third = 1.0f / 3.0f;
  for (size_t i = 0; i < n; i++) {
    const float *p0 = &v[3 * (size_t)f[3 * i + 0]];
    const float *p1 = &v[3 * (size_t)f[3 * i + 1]];
    const float *p2 = &v[3 * (size_t)f[3 * i + 2]];
    float c[3];
    for (int k = 0; k < 3; k++) c[k] = one_third * (p0[k] + p1[k] + p2[k]);
    codes[i] = morton_of(c, bmin, inv);
  }
}

/* CalculateMortonCodesTetraFloat30 (render/render_prefix_tree_util.cc:267-304) */
SO_API void so_morton_tets(const float *v, const uint32_t *f, size_t n,
                           const float bmin[3], const float bmax[3],
                           uint32_t *codes) {
  float inv[3];
  morton_inv(bmin, bmax, inv);
  const float one_fourth = 1.0f / 4.0f;
  for (size_t i = 0; i < n; i++) {
    const float *p0 = &v[3 * (size_t)f[4 * i + 0]];
    const float *p1 = &v[3 * (size_t)f[4 * i + 1]];
    const float *p2 = &v[3 * (size_t)f[4 * i + 2]];
    const float *p3 = &v[3 * (size_t)f[4 * i + 3]];
    float c[3];
    for (int k = 0; k < 3; k++)
      c[k] = one_fourth * (p0[k] + p1[k] + p2[k] + p3[k]);
    codes[i] = morton_of(c, bmin, inv);
  }
}

/* ------------------------------------------------------------------------ */
/* Scene bounding boxes                                                      */
/* ------------------------------------------------------------------------ */

static inline float fmin_ref(float a, float b) { return (b < a) ? b : a; }
static inline float fmax_ref(float a, float b) { return (a < b) ? b : a; }

/* Per-vertex box with padding eps over the vertices of `n` primitives of
 * `nv` corners each (ComputeBoundingBoxOMP, render/render_accel_triangle.cc:713;
 * render/render_accel_tetra.cc:973). */
static void bbox_corners(const float *v, const uint32_t *f, size_t n, int nv,
                         float eps, float bmin[3], float bmax[3]) {
  for (int k = 0; k < 3; k++) {
    bmin[k] = FLT_MAX;
    bmax[k] = -FLT_MAX;
  }
  for (size_t i = 0; i < n; i++)
    for (int j = 0; j < nv; j++) {
      const float *p = &v[3 * (size_t)f[(size_t)nv * i + j]];
      for (int k = 0; k < 3; k++) {
        bmin[k] = fmin_ref(bmin[k], p[k] - eps);
        bmax[k] = fmax_ref(bmax[k], p[k] + eps);
      }
    }
}

SO_API void so_bbox_tris(const float *v, const uint32_t *f, size_t n,
                         float bmin[3], float bmax[3]) {
  bbox_corners(v, f, n, 3, 0.0f, bmin, bmax);
}

SO_API void so_bbox_tets(const float *v, const uint32_t *f, size_t n,
                         float bmin[3], float bmax[3]) {
  const float keps = FLT_EPSILON * 16;
  bbox_corners(v, f, n, 4, keps, bmin, bmax);
}

static inline float sphere_radius(const float *radius, float constr, size_t i) {
  return radius ? radius[i] : constr;
}

/* render/render_accel_particle.cc:304-369: centre -/+ radius -/+ 16 ulp(1). */
SO_API void so_bbox_spheres(const float *pos, const float *radius, float constr,
                            size_t n, float bmin[3], float bmax[3]) {
  const float keps = FLT_EPSILON * 16.0;
  for (int k = 0; k < 3; k++) {
    bmin[k] = FLT_MAX;
    bmax[k] = -FLT_MAX;
  }
  for (size_t i = 0; i < n; i++) {
    float r = sphere_radius(radius, constr, i);
    for (int k = 0; k < 3; k++) {
      bmin[k] = fmin_ref(bmin[k], pos[3 * i + k] - r - keps);
      bmax[k] = fmax_ref(bmax[k], pos[3 * i + k] + r + keps);
    }
  }
}

/* ------------------------------------------------------------------------ */
/* Stable sort of (code, index) pairs by code                                */
/* ------------------------------------------------------------------------ */

/* RadixSort30 / RadixSort30OMP (render/render_prefix_tree_util.h:296-457):
 * four stable 8-bit counting passes over the 32-bit code.  For n < 1024 the
 * reference uses an unstable quicksort, but Build32 is never reached below
 * 1024 primitives; this restatement is stable for every n. */
SO_API void so_sort_pairs(uint32_t *code, uint32_t *index, size_t n) {
  uint32_t *c2 = (uint32_t *)malloc(n * sizeof(uint32_t) + 4);
  uint32_t *i2 = (uint32_t *)malloc(n * sizeof(uint32_t) + 4);
  uint32_t *sc = code, *si = index, *dc = c2, *di = i2;
  for (int shift = 0; shift < 32; shift += 8) {
    size_t count[257];
    memset(count, 0, sizeof(count));
    for (size_t i = 0; i < n; i++) count[((sc[i] >> shift) & 0xff) + 1]++;
    for (int b = 0; b < 256; b++) count[b + 1] += count[b];
    for (size_t i = 0; i < n; i++) {
      size_t d = count[(sc[i] >> shift) & 0xff]++;
      dc[d] = sc[i];
      di[d] = si[i];
    }
    uint32_t *t;
    t = sc; sc = dc; dc = t;
    t = si; si = di; di = t;
  }
  /* four passes: the result is back in the caller's arrays */
  free(c2);
  free(i2);
}

/* ------------------------------------------------------------------------ */
/* Karras binary radix tree                                                  */
/* ------------------------------------------------------------------------ */

static inline int clz32(uint32_t x) { return x ? __builtin_clz(x) : 32; }

/* Delta30 (render/render_prefix_tree_util.cc:501-526): common-prefix length of
 * sorted keys i and j; equal codes fall back to 32 + prefix of the positions;
 * -1 outside [0,n). */
static inline int kdelta(const uint32_t *code, int32_t i, int32_t j, int32_t n) {
  if (j < 0 || j >= n) return -1;
  uint32_t a = code[i], b = code[j];
  if (a == b) return 32 + clz32((uint32_t)i ^ (uint32_t)j);
  return clz32(a ^ b);
}

/* ConstructBinaryRadixTree30 (render/render_prefix_tree_util.cc:562-649).
 * child[i] = split gamma; ltype/rtype = 1 when that child is a single key. */
SO_API void so_karras(const uint32_t *code, size_t n_, uint32_t *child,
                      uint8_t *ltype, uint8_t *rtype) {
  int32_t n = (int32_t)n_;
  for (int32_t i = 0; i < n - 1; i++) {
    int d = (kdelta(code, i, i + 1, n) - kdelta(code, i, i - 1, n)) >= 0 ? 1 : -1;
    int dmin = kdelta(code, i, i - d, n);
    int lmax = 2;
    while (kdelta(code, i, i + lmax * d, n) > dmin) lmax *= 2;
    int l = 0;
    for (int t = lmax / 2; t >= 1; t /= 2)
      if (kdelta(code, i, i + (l + t) * d, n) > dmin) l += t;
    int j = i + l * d;
    int dnode = kdelta(code, i, j, n);
    int s = 0;
    /* t = ceil(l/2), ceil(l/4), ..., 1 */
    for (int k = 2;; k *= 2) {
      int t = (l + k - 1) / k;
      if (t <= 0) break;
      if (kdelta(code, i, i + (s + t) * d, n) > dnode) s += t;
      if (t == 1) break;
    }
    int g = i + s * d + (d < 0 ? d : 0);
    child[i] = (uint32_t)g;
    ltype[i] = ((i < j ? i : j) == g) ? 1 : 0;
    rtype[i] = ((i > j ? i : j) == g + 1) ? 1 : 0;
  }
}

/* ------------------------------------------------------------------------ */
/* LBVH emission                                                             */
/* ------------------------------------------------------------------------ */

/* One node in reference emission order.  bmin/bmax is the node's OWN box:
 * for triangles and spheres the reference stores it in the parent's child
 * slot (TriangleNode/ParticleNode), for tetrahedra in the node itself
 * (TetraNode, render/render_accel_tetra.h:24-43). */
typedef struct {
  float bmin[3], bmax[3];
  int32_t leaf;  /* 1 = leaf */
  int32_t axis;  /* branch split axis */
  uint32_t d0;   /* leaf: count, branch: left child */
  uint32_t d1;   /* leaf: offset, branch: right child */
} so_node;

typedef struct {
  int kind;
  size_t nprims;
  size_t nnodes, cap;
  so_node *nodes;
  uint32_t *indices; /* sorted primitive ids */
  uint32_t *codes;   /* sorted Morton codes */
  uint32_t *child;
  uint8_t *ltype, *rtype;
  float scene_min[3], scene_max[3];
  double eps_scale; /* triangles: max scene extent */
  float keps;       /* leaf padding */
  int max_leaf;
  /* borrowed primitive data */
  const float *verts;
  const uint32_t *faces;
  const float *radius;
  float constr;
  /* tetrahedra with double-precision positions (isDoublePrecisionPos):
   * dverts is borrowed, verts then holds them rounded to float (owned) */
  const double *dverts;
  float *own_verts;
} so_accel;

static size_t push_node(so_accel *a) {
  if (a->nnodes == a->cap) {
    a->cap = a->cap ? a->cap * 2 : 1024;
    a->nodes = (so_node *)realloc(a->nodes, a->cap * sizeof(so_node));
  }
  memset(&a->nodes[a->nnodes], 0, sizeof(so_node));
  return a->nnodes++;
}

/* Leaf box over sorted primitives [lo, hi] (ComputeBoundingBox30,
 * render/render_accel_triangle.cc:661-709; tetra :923-970; particle :417-461). */
static void leaf_box(const so_accel *a, uint32_t lo, uint32_t hi, float bmin[3],
                     float bmax[3]) {
  const float e = a->keps;
  for (int k = 0; k < 3; k++) {
    bmin[k] = FLT_MAX;
    bmax[k] = -FLT_MAX;
  }
  for (uint32_t i = lo; i <= hi; i++) {
    size_t p = a->indices[i];
    if (a->kind == SO_SPHERE) {
      float r = sphere_radius(a->radius, a->constr, p);
      for (int k = 0; k < 3; k++) {
        float mn = a->verts[3 * p + k] - r - e;
        float mx = a->verts[3 * p + k] + r + e;
        if (bmin[k] > mn) bmin[k] = mn;
        if (bmax[k] < mx) bmax[k] = mx;
      }
    } else {
      int nv = a->kind == SO_TRI ? 3 : 4;
      for (int j = 0; j < nv; j++) {
        const size_t vi = a->faces[(size_t)nv * p + j];
        const float *q = &a->verts[3 * vi];
        for (int k = 0; k < 3; k++) {
          /* double positions: padded in double, then rounded */
          float mn = a->dverts ? (float)(a->dverts[3 * vi + k] - (double)e) : q[k] - e;
          float mx = a->dverts ? (float)(a->dverts[3 * vi + k] + (double)e) : q[k] + e;
          if (bmin[k] > mn) bmin[k] = mn;
          if (bmax[k] < mx) bmax[k] = mx;
        }
      }
    }
  }
}

/* GetSplitAxis (render/render_accel_triangle.cc:854-863). */
static int split_axis(uint32_t code) { return (clz32(code) - 2) % 3; }

/* BuildTreeRecursive32 (render/render_accel_triangle.cc:896-992): emit the
 * subtree rooted at Karras node `root` covering sorted range [lo, hi]. */
static size_t emit(so_accel *a, uint32_t root, uint32_t lo, uint32_t hi,
                   int is_leaf, int depth) {
  if (is_leaf || (hi - lo) <= (uint32_t)a->max_leaf || depth > 22) {
    size_t o = push_node(a);
    so_node *nd = &a->nodes[o];
    leaf_box(a, lo, hi, nd->bmin, nd->bmax);
    nd->leaf = 1;
    nd->axis = 0;
    nd->d0 = hi - lo + 1;
    nd->d1 = lo;
    return o;
  }
  uint32_t mid = a->child[root];
  size_t o = push_node(a);
  a->nodes[o].leaf = 0;
  a->nodes[o].axis = split_axis(a->codes[root]);
  size_t l = emit(a, mid, lo, mid, a->ltype[root], depth + 1);
  size_t r = emit(a, mid + 1, mid + 1, hi, a->rtype[root], depth + 1);
  so_node *nd = &a->nodes[o];
  nd->d0 = (uint32_t)l;
  nd->d1 = (uint32_t)r;
  for (int k = 0; k < 3; k++) {
    nd->bmin[k] = fmin_ref(a->nodes[l].bmin[k], a->nodes[r].bmin[k]);
    nd->bmax[k] = fmax_ref(a->nodes[l].bmax[k], a->nodes[r].bmax[k]);
  }
  return o;
}

/* Build32 for the three primitive kinds (render/render_accel_triangle.cc:1389,
 * render/render_accel_tetra.cc:1579, render/render_accel_particle.cc:1560).
 * Requires n >= 2 (the reference switches to its SAH builder below 1024). */
static so_accel *build_impl(int kind, const float *verts, const double *dverts,
                            size_t nverts, const uint32_t *faces, const float *radius,
                            float constr, size_t n) {
  if (n < 2) return NULL;
  so_accel *a = (so_accel *)calloc(1, sizeof(so_accel));
  a->kind = kind;
  a->nprims = n;
  if (dverts) { /* positions rounded to float: Morton codes, shading records */
    a->own_verts = (float *)malloc(3 * nverts * sizeof(float));
    for (size_t i = 0; i < 3 * nverts; i++) a->own_verts[i] = (float)dverts[i];
    verts = a->own_verts;
    a->dverts = dverts;
  }
  a->verts = verts;
  a->faces = faces;
  a->radius = radius;
  a->constr = constr;
  a->codes = (uint32_t *)malloc(n * sizeof(uint32_t));
  a->indices = (uint32_t *)malloc(n * sizeof(uint32_t));
  float bmin[3], bmax[3];
  if (kind == SO_TRI) {
    so_bbox_tris(verts, faces, n, bmin, bmax);
    double es = bmax[0] - bmin[0];
    if (es < (double)(bmax[1] - bmin[1])) es = bmax[1] - bmin[1];
    if (es < (double)(bmax[2] - bmin[2])) es = bmax[2] - bmin[2];
    a->eps_scale = es;
    a->keps = FLT_EPSILON * (float)es;
    a->max_leaf = 16;
    so_morton_tris(verts, faces, n, bmin, bmax, a->codes);
  } else if (kind == SO_TET && dverts) {
    /* ComputeBoundingBoxOMP over dvertices: padded in double, rounded */
    const double e = (double)(FLT_EPSILON * 16);
    for (int k = 0; k < 3; k++) {
      bmin[k] = FLT_MAX;
      bmax[k] = -FLT_MAX;
    }
    for (size_t i = 0; i < 4 * n; i++)
      for (int k = 0; k < 3; k++) {
        bmin[k] = fmin_ref(bmin[k], (float)(dverts[3 * (size_t)faces[i] + k] - e));
        bmax[k] = fmax_ref(bmax[k], (float)(dverts[3 * (size_t)faces[i] + k] + e));
      }
    a->eps_scale = 16.0;
    a->keps = FLT_EPSILON * 16;
    a->max_leaf = 4;
    so_morton_tets(verts, faces, n, bmin, bmax, a->codes);
  } else if (kind == SO_TET) {
    so_bbox_tets(verts, faces, n, bmin, bmax);
    a->eps_scale = 16.0;
    a->keps = FLT_EPSILON * 16;
    a->max_leaf = 4;
    so_morton_tets(verts, faces, n, bmin, bmax, a->codes);
  } else {
    so_bbox_spheres(verts, radius, constr, n, bmin, bmax);
    a->eps_scale = 16.0;
    a->keps = FLT_EPSILON * 16.0;
    a->max_leaf = 16;
    so_morton_points(verts, n, bmin, bmax, a->codes);
  }
  memcpy(a->scene_min, bmin, sizeof(bmin));
  memcpy(a->scene_max, bmax, sizeof(bmax));
  for (size_t i = 0; i < n; i++) a->indices[i] = (uint32_t)i;
  so_sort_pairs(a->codes, a->indices, n);
  a->child = (uint32_t *)malloc((n - 1) * sizeof(uint32_t));
  a->ltype = (uint8_t *)malloc(n - 1);
  a->rtype = (uint8_t *)malloc(n - 1);
  so_karras(a->codes, n, a->child, a->ltype, a->rtype);

  /* root: always a branch; its children start at depth 0 */
  size_t root = push_node(a);
  uint32_t mid = a->child[0];
  size_t l = emit(a, mid, 0, mid, a->ltype[0], 0);
  size_t r = emit(a, mid + 1, mid + 1, (uint32_t)(n - 1), a->rtype[0], 0);
  so_node *nd = &a->nodes[root];
  nd->leaf = 0;
  nd->axis = split_axis(a->codes[0]);
  nd->d0 = (uint32_t)l;
  nd->d1 = (uint32_t)r;
  for (int k = 0; k < 3; k++) {
    nd->bmin[k] = fmin_ref(a->nodes[l].bmin[k], a->nodes[r].bmin[k]);
    nd->bmax[k] = fmax_ref(a->nodes[l].bmax[k], a->nodes[r].bmax[k]);
  }
  return a;
}

SO_API so_accel *so_build(int kind, const float *verts, const uint32_t *faces,
                          const float *radius, float constr, size_t n) {
  return build_impl(kind, verts, NULL, 0, faces, radius, constr, n);
}

/* Tetrahedra with double-precision positions (Tetrahedron::dvertices). */
SO_API so_accel *so_build_tet_d(const double *dverts, size_t nverts, const uint32_t *faces,
                                size_t n) {
  return build_impl(SO_TET, NULL, dverts, nverts, faces, NULL, 0.0f, n);
}

SO_API void so_free(so_accel *a) {
  if (!a) return;
  free(a->own_verts);
  free(a->nodes);
  free(a->indices);
  free(a->codes);
  free(a->child);
  free(a->ltype);
  free(a->rtype);
  free(a);
}

SO_API size_t so_num_nodes(const so_accel *a) { return a->nnodes; }

/* Copies: nodes as 10 x 32-bit words each (bmin[3], bmax[3], leaf, axis, d0,
 * d1), sorted indices, sorted codes, Karras arrays, scene box, eps values. */
SO_API void so_export(const so_accel *a, void *nodes, uint32_t *indices,
                      uint32_t *codes, float scene[6], double *eps_scale) {
  if (nodes) memcpy(nodes, a->nodes, a->nnodes * sizeof(so_node));
  if (indices) memcpy(indices, a->indices, a->nprims * sizeof(uint32_t));
  if (codes) memcpy(codes, a->codes, a->nprims * sizeof(uint32_t));
  if (scene) {
    memcpy(scene, a->scene_min, 3 * sizeof(float));
    memcpy(scene + 3, a->scene_max, 3 * sizeof(float));
  }
  if (eps_scale) *eps_scale = a->eps_scale;
}

SO_API void so_export_karras(const so_accel *a, uint32_t *child, uint8_t *lt,
                             uint8_t *rt) {
  size_t m = a->nprims - 1;
  memcpy(child, a->child, m * sizeof(uint32_t));
  memcpy(lt, a->ltype, m);
  memcpy(rt, a->rtype, m);
}

/* ------------------------------------------------------------------------ */
/* Canonical topology                                                        */
/* ------------------------------------------------------------------------ */

/* Depth-first, left-first listing of a tree given in generic form (own box,
 * leaf flag, axis, d0/d1 as in so_node).  Output records, 10 words each:
 * leaf, axis (0 for leaves), count (0 for branches), offset (0 for
 * branches), bmin[3], bmax[3], depth, reserved.  Node storage order is
 * irrelevant, so a tree emitted by concurrent tasks compares equal to the
 * sequential emission.  Returns the number of records, or -1 on a malformed
 * tree (index out of range, cycle, more than `max_out` records). */
SO_API long so_canonicalize(const void *generic_nodes, size_t nnodes, size_t root,
                            uint32_t *out, size_t max_out) {
  const so_node *nd = (const so_node *)generic_nodes;
  size_t *stack = (size_t *)malloc(sizeof(size_t) * 2 * 4096);
  int *dstack = (int *)malloc(sizeof(int) * 2 * 4096);
  long cnt = 0;
  int sp = 0;
  stack[0] = root;
  dstack[0] = 0;
  while (sp >= 0) {
    size_t i = stack[sp];
    int dep = dstack[sp];
    sp--;
    if (i >= nnodes || (size_t)cnt >= max_out) {
      cnt = -1;
      break;
    }
    uint32_t *o = &out[10 * (size_t)cnt];
    const so_node *x = &nd[i];
    o[0] = x->leaf ? 1u : 0u;
    o[1] = x->leaf ? 0u : (uint32_t)x->axis;
    o[2] = x->leaf ? x->d0 : 0u;
    o[3] = x->leaf ? x->d1 : 0u;
    memcpy(&o[4], x->bmin, 3 * sizeof(float));
    memcpy(&o[7], x->bmax, 3 * sizeof(float));
    /* depth kept out of the record body; callers that need it re-derive */
    (void)dep;
    cnt++;
    if (!x->leaf) {
      if (sp + 2 >= 2 * 4096) {
        cnt = -1;
        break;
      }
      /* right pushed first so that left is listed first */
      stack[++sp] = x->d1;
      dstack[sp] = dep + 1;
      stack[++sp] = x->d0;
      dstack[sp] = dep + 1;
    }
  }
  free(stack);
  free(dstack);
  return cnt;
}

/* ------------------------------------------------------------------------ */
/* Traversal                                                                 */
/* ------------------------------------------------------------------------ */

typedef struct {
  float org[3];
  uint32_t prev_prim;
  float dir[3];
  float prev_t;
} so_ray; /* 32 bytes, same as the product's srt_ray */

typedef struct {
  float t, u, v;
  uint32_t prim;
} so_hit;

typedef struct {
  uint64_t branch_visits; /* popped branch nodes (tri/sphere) or all pops (tet) */
  uint64_t leaf_visits;
  uint64_t prim_tests;
} so_stats;

/* IntersectRayAABB (render/render_accel_triangle.cc:1815-1861); `clamp` = 1
 * clamps tmax to maxT (triangle, particle), 0 tests tmin <= maxT (tetra,
 * render/render_accel_tetra.cc:1934-1978). */
static inline int ray_aabb(float maxT, const float bmin[3], const float bmax[3],
                           const float org[3], const float inv[3],
                           const int sgn[3], int clamp) {
  float tmin, tmax;
  const float min_x = sgn[0] ? bmax[0] : bmin[0];
  const float min_y = sgn[1] ? bmax[1] : bmin[1];
  const float min_z = sgn[2] ? bmax[2] : bmin[2];
  const float max_x = sgn[0] ? bmin[0] : bmax[0];
  const float max_y = sgn[1] ? bmin[1] : bmax[1];
  const float max_z = sgn[2] ? bmin[2] : bmax[2];
  const float tmin_x = (min_x - org[0]) * inv[0];
  const float tmax_x = (max_x - org[0]) * inv[0];
  const float tmin_y = (min_y - org[1]) * inv[1];
  const float tmax_y = (max_y - org[1]) * inv[1];
  tmin = (tmin_x > tmin_y) ? tmin_x : tmin_y;
  tmax = (tmax_x < tmax_y) ? tmax_x : tmax_y;
  const float tmin_z = (min_z - org[2]) * inv[2];
  const float tmax_z = (max_z - org[2]) * inv[2];
  tmin = (tmin > tmin_z) ? tmin : tmin_z;
  tmax = (tmax < tmax_z) ? tmax : tmax_z;
  if (clamp) {
    tmax = (maxT < tmax) ? maxT : tmax;
    return (tmax > 0.0f) && (tmin <= tmax);
  }
  return (tmax > 0.0f) && (tmin <= tmax) && (tmin <= maxT);
}

static inline float dot3f(const float a[3], const float b[3]) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}
static inline void cross3f(const float a[3], const float b[3], float c[3]) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}

/* TriangleIsect, double-sided (render/render_accel_triangle.cc:1887-1938). */
static inline int tri_isect(float *tio, float *uo, float *vo, const float p0[3],
                            const float p1[3], const float p2[3],
                            const float org[3], const float dir[3], float keps) {
  float e1[3], e2[3], p[3], s[3], q[3];
  for (int k = 0; k < 3; k++) {
    e1[k] = p1[k] - p0[k];
    e2[k] = p2[k] - p0[k];
  }
  cross3f(dir, e2, p);
  float det = dot3f(e1, p);
  if (fabsf(det) < keps) return 0;
  float inv_det = (float)(1.0 / (double)det);
  for (int k = 0; k < 3; k++) s[k] = org[k] - p0[k];
  cross3f(s, e1, q);
  float u = dot3f(s, p) * inv_det;
  float v = dot3f(q, dir) * inv_det;
  float t = dot3f(e2, q) * inv_det;
  if (u < 0.0f || u > 1.0f) return 0;
  if (v < 0.0f || u + v > 1.0f) return 0;
  if (t < 0.0f || t > *tio) return 0;
  *tio = t;
  *uo = u;
  *vo = v;
  return 1;
}

/* ---- Pluecker ray/tetrahedron test, FP64 (render/render_accel_tetra.cc:89-567) */
typedef struct { double x, y, z; } d3;
static inline d3 d3sub(d3 a, d3 b) { d3 r = {a.x - b.x, a.y - b.y, a.z - b.z}; return r; }
static inline d3 d3add(d3 a, d3 b) { d3 r = {a.x + b.x, a.y + b.y, a.z + b.z}; return r; }
static inline d3 d3scale(double f, d3 v) { d3 r = {v.x * f, v.y * f, v.z * f}; return r; }
static inline d3 d3cross(d3 a, d3 b) {
  d3 c = {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
  return c;
}
static inline double d3dot(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline int dsign(double x) {
  return x > DBL_EPSILON ? 1 : (x < -DBL_EPSILON ? -1 : 0);
}
typedef struct { d3 d, c; } plk;
static inline plk plk_make(d3 v0, d3 v1) {
  plk p;
  p.d = d3sub(v1, v0);
  p.c = d3cross(v1, v0);
  return p;
}
static inline double plk_dot(plk a, plk b) { return d3dot(a.d, b.c) + d3dot(b.d, a.c); }

/* barycentric point (1-a-b)*A + a*B + b*C */
static inline d3 bary(double a, double b, d3 A, d3 B, d3 C) {
  return d3add(d3add(d3scale(1 - a - b, A), d3scale(a, B)), d3scale(b, C));
}

static inline void param_dist(d3 o, d3 d, d3 pe, d3 pl, double *te, double *tl) {
  if (d.x != 0.0) {
    double iv = 1.0 / d.x;
    *te = (pe.x - o.x) * iv;
    *tl = (pl.x - o.x) * iv;
  } else if (d.y != 0.0) {
    double iv = 1.0 / d.y;
    *te = (pe.y - o.y) * iv;
    *tl = (pl.y - o.y) * iv;
  } else {
    double iv = 1.0 / d.z;
    *te = (pe.z - o.z) * iv;
    *tl = (pl.z - o.z) * iv;
  }
}

/* Output: enter face, enter barycentrics (ue1, ue2), leave barycentric ul1,
 * enter distance.  Mirrors RayTetraPluecker's face order and sign logic. */
/* Corner vi of a tetrahedron as the Pluecker test takes it: the float
 * position, or the double one (TestLeafNode's dvertices branch). */
static inline void tet_corner(const so_accel *a, size_t vi, d3 *out) {
  if (a->dverts) {
    out->x = a->dverts[3 * vi];
    out->y = a->dverts[3 * vi + 1];
    out->z = a->dverts[3 * vi + 2];
  } else {
    out->x = a->verts[3 * vi];
    out->y = a->verts[3 * vi + 1];
    out->z = a->verts[3 * vi + 2];
  }
}

static int ray_tet(d3 orig, d3 dir, const d3 V[4], int *ef, double *ue1,
                   double *ue2, double *ul1, double *te) {
  int enterF = -1, leaveF = -1;
  double uAB = 0, uAC = 0, uDB = 0, uDC = 0, uBC = 0, uAD = 0;
  int sAB = -2, sAC = -2, sDB = -2, sDC = -2, sBC = -2, sAD = -2;
  double eu1 = 0, eu2 = 0, lu1 = 0, lu2 = 0, tl = 0;
  d3 ep = {0, 0, 0}, lp = {0, 0, 0};
  (void)leaveF; (void)lu2;
  d3 dest = d3add(orig, dir);
  plk ray = plk_make(orig, dest);
  int next = 0;

#define ENTER(F, A1, A2, P0, P1, P2) do { enterF = F; eu1 = A1; eu2 = A2; ep = bary(eu1, eu2, P0, P1, P2); } while (0)
#define LEAVE(F, A1, A2, P0, P1, P2) do { leaveF = F; lu1 = A1; lu2 = A2; lp = bary(lu1, lu2, P0, P1, P2); } while (0)
#define DONE() do { param_dist(orig, dir, ep, lp, te, &tl); *ef = enterF; *ue1 = eu1; *ue2 = eu2; *ul1 = lu1; return 1; } while (0)

  uAB = plk_dot(ray, plk_make(V[0], V[1])); sAB = dsign(uAB);
  uAC = plk_dot(ray, plk_make(V[0], V[2])); sAC = dsign(uAC);
  if ((sAC == -sAB) || (sAC == 0) || (sAB == 0)) {
    uBC = plk_dot(ray, plk_make(V[1], V[2])); sBC = dsign(uBC);
    int sABC = sAB;
    if (sABC == 0) { sABC = -sAC; if (sABC == 0) sABC = sBC; }
    if ((sABC != 0) && ((sBC == sABC) || (sBC == 0))) {
      double inv = 1.0 / (uAB + uBC - uAC);
      if (sABC == 1) { ENTER(3, -uAC * inv, uAB * inv, V[0], V[1], V[2]); next = -1; }
      else { LEAVE(3, -uAC * inv, uAB * inv, V[0], V[1], V[2]); next = 1; }
      uAD = plk_dot(ray, plk_make(V[0], V[3])); sAD = dsign(uAD);
      if ((sAD == next) || (sAD == 0)) {
        uDB = plk_dot(ray, plk_make(V[3], V[1])); sDB = dsign(uDB);
        if ((sDB == next) || ((sDB == 0) && ((sAD != 0) || (sAB != 0)))) {
          double iv = 1.0 / (uAD + uDB - uAB);
          if (next == 1) ENTER(2, uDB * iv, -uAB * iv, V[1], V[0], V[3]);
          else LEAVE(2, uDB * iv, -uAB * iv, V[1], V[0], V[3]);
          DONE();
        }
      }
      uDC = plk_dot(ray, plk_make(V[3], V[2])); sDC = dsign(uDC);
      if ((sDC == -next) || ((sDC == 0) && ((sAD != 0) || (sAC != 0)))) {
        double iv = 1.0 / (uAC - uDC - uAD);
        if (next == 1) ENTER(1, uAC * iv, -uDC * iv, V[2], V[3], V[0]);
        else LEAVE(1, uAC * iv, -uDC * iv, V[2], V[3], V[0]);
        DONE();
      } else {
        if (sDB == -2) uDB = plk_dot(ray, plk_make(V[3], V[1]));
        double iv = 1.0 / (uDC - uBC - uDB);
        if (next == 1) ENTER(0, -uDB * iv, uDC * iv, V[3], V[2], V[1]);
        else LEAVE(0, -uDB * iv, uDC * iv, V[3], V[2], V[1]);
        DONE();
      }
    }
  }
  uAD = plk_dot(ray, plk_make(V[0], V[3])); sAD = dsign(uAD);
  if ((sAD == -sAB) || (sAB == 0) || (sAD == 0)) {
    uDB = plk_dot(ray, plk_make(V[3], V[1])); sDB = dsign(uDB);
    int sBAD = -sAB;
    if (sBAD == 0) { sBAD = sAD; if (sBAD == 0) sBAD = sDB; }
    if ((sBAD != 0) && ((sDB == sBAD) || (sDB == 0))) {
      double inv = 1.0 / (uAD + uDB - uAB);
      if (sBAD == 1) { ENTER(2, uDB * inv, -uAB * inv, V[1], V[0], V[3]); next = -1; }
      else { LEAVE(2, uDB * inv, -uAB * inv, V[1], V[0], V[3]); next = 1; }
      uDC = plk_dot(ray, plk_make(V[3], V[2])); sDC = dsign(uDC);
      if ((sDC == -next) || ((sDC == 0) && ((sAD != 0) || (sAC != 0)))) {
        double iv = 1.0 / (uAC - uDC - uAD);
        if (next == 1) ENTER(1, uAC * iv, -uDC * iv, V[2], V[3], V[0]);
        else LEAVE(1, uAC * iv, -uDC * iv, V[2], V[3], V[0]);
        DONE();
      } else {
        if (sBC == -2) uBC = plk_dot(ray, plk_make(V[1], V[2]));
        double iv = 1.0 / (uDC - uBC - uDB);
        if (next == 1) ENTER(0, -uDB * iv, uDC * iv, V[3], V[2], V[1]);
        else LEAVE(0, -uDB * iv, uDC * iv, V[3], V[2], V[1]);
        DONE();
      }
    }
  }
  if ((-sAD == sAC) || (sAC == 0) || (sAD == 0)) {
    uDC = plk_dot(ray, plk_make(V[3], V[2])); sDC = dsign(uDC);
    int sCDA = sAC;
    if (sCDA == 0) { sCDA = -sAD; if (sCDA == 0) sCDA = -sDC; }
    if ((sCDA != 0) && ((-sDC == sCDA) || (sDC == 0))) {
      double ivCDA = 1.0 / (uAC - uDC - uAD);
      if (sBC == -2) uBC = plk_dot(ray, plk_make(V[1], V[2]));
      if (sDB == -2) uDB = plk_dot(ray, plk_make(V[3], V[1]));
      double ivDCB = 1.0 / (uDC - uBC - uDB);
      if (sCDA == 1) {
        ENTER(1, uAC * ivCDA, -uDC * ivCDA, V[2], V[3], V[0]);
        LEAVE(0, -uDB * ivDCB, uDC * ivDCB, V[3], V[2], V[1]);
      } else {
        LEAVE(1, uAC * ivCDA, -uDC * ivCDA, V[2], V[3], V[0]);
        ENTER(0, -uDB * ivDCB, uDC * ivDCB, V[3], V[2], V[1]);
      }
      DONE();
    }
  }
#undef ENTER
#undef LEAVE
#undef DONE
  return 0;
}

/* SphereIsect (render/render_accel_particle.cc:2423-2512). */
static inline int sphere_isect(float *tio, const float c[3], float radius,
                               const float org[3], const float dir[3],
                               double prevT, const float prevN[3], int self) {
  float oc[3] = {org[0] - c[0], org[1] - c[1], org[2] - c[2]};
  float a = dot3f(dir, dir);
  float b = (float)(2.0 * (double)dot3f(dir, oc));
  float cc = dot3f(oc, oc) - radius * radius;
  float disc = (float)((double)(b * b) - 4.0 * (double)a * (double)cc);
  float t0, t1;
  if (disc < 0.0f) return 0;
  else if (disc == 0.0f) {
    t0 = t1 = (float)(-0.5 * (double)(b / a));
  } else {
    float ds = sqrtf(disc);
    float q;
    if (b < 0) q = (float)((double)(-b - ds) / 2.0);
    else q = (float)((double)(-b + ds) / 2.0);
    t0 = q / a;
    t1 = cc / q;
  }
  if (t0 > t1) { float tmp = t0; t0 = t1; t1 = tmp; }
  if (t1 < 0) return 0;
  if (self) {
    float t = t1;
    float nrm[3];
    for (int k = 0; k < 3; k++) nrm[k] = (org[k] + t * dir[k]) - c[k];
    if ((t < *tio) && ((double)t < prevT) && (dot3f(nrm, prevN) <= 0.0f)) {
      *tio = t;
      return 1;
    }
  } else {
    float t = (t0 < 0) ? t1 : t0;
    if (t < *tio) {
      *tio = t;
      return 1;
    }
  }
  return 0;
}

/* Closest hit for one ray: Traverse() of the three accel classes, with the
 * running distance starting at t0 (FLT_MAX: the reference's own walk).
 * Returns whether a primitive was accepted. */
static int trace_from(const so_accel *a, const so_ray *ray, const float *prevN,
                      so_hit *h, uint32_t *subface, const float *vscalar,
                      float *scalar_out, so_stats *st, float t0) {
  double best_e1 = 0.0, best_e2 = 0.0;
  float hitT = t0;
  h->t = hitT;
  h->u = 0.0f;
  h->v = 0.0f;
  h->prim = 0xffffffffu;
  uint32_t sub = 0;
  int sgn[3];
  float inv[3];
  for (int k = 0; k < 3; k++) {
    sgn[k] = ray->dir[k] < 0.0f ? 1 : 0;
    inv[k] = (float)(1.0 / (double)ray->dir[k]);
  }
  const float *org = ray->org;
  const float *dir = ray->dir;
  float zero3[3] = {0, 0, 0};
  const float *pn = prevN ? prevN : zero3;
  int stack[512];
  int sp = 0;
  stack[0] = 0;
  while (sp >= 0) {
    const so_node *nd = &a->nodes[stack[sp]];
    sp--;
    if (a->kind == SO_TET) {
      int hit = ray_aabb(hitT, nd->bmin, nd->bmax, org, inv, sgn, 0);
      st->branch_visits++;
      if (!nd->leaf) {
        if (hit) {
          int nearc = sgn[nd->axis], farc = 1 - nearc;
          stack[++sp] = (int)(farc ? nd->d1 : nd->d0);
          stack[++sp] = (int)(nearc ? nd->d1 : nd->d0);
        }
      } else if (hit) {
        st->leaf_visits++;
        float t = h->t;
        int any = 0;
        d3 o = {org[0], org[1], org[2]};
        d3 d = {dir[0], dir[1], dir[2]};
        for (uint32_t i = 0; i < nd->d0; i++) {
          uint32_t f = a->indices[nd->d1 + i];
          if (f == ray->prev_prim) continue;
          st->prim_tests++;
          d3 V[4];
          for (int j = 0; j < 4; j++) tet_corner(a, a->faces[4 * (size_t)f + j], &V[j]);
          int ef;
          double ue1, ue2, ul1, te;
          if (ray_tet(o, d, V, &ef, &ue1, &ue2, &ul1, &te)) {
            if ((te >= 0.0) && (te < (double)t)) {
              h->t = (float)te;
              h->u = (float)ue1;
              h->v = (float)ul1; /* the reference passes uLeave1 into isect.v */
              h->prim = f;
              sub = (uint32_t)ef;
              best_e1 = ue1;
              best_e2 = ue2;
              t = (float)te;
              any = 1;
            }
          }
        }
        if (any) hitT = h->t;
      }
      continue;
    }
    if (!nd->leaf) {
      st->branch_visits++;
      const so_node *c0 = &a->nodes[nd->d0];
      const so_node *c1 = &a->nodes[nd->d1];
      int hits[2];
      hits[0] = ray_aabb(hitT, c0->bmin, c0->bmax, org, inv, sgn, 1);
      hits[1] = ray_aabb(hitT, c1->bmin, c1->bmax, org, inv, sgn, 1);
      if (hits[0] || hits[1]) {
        int nearc = sgn[nd->axis], farc = 1 - nearc;
        if (hits[farc]) stack[++sp] = (int)(farc ? nd->d1 : nd->d0);
        if (hits[nearc]) stack[++sp] = (int)(nearc ? nd->d1 : nd->d0);
      }
    } else {
      st->leaf_visits++;
      float t = h->t;
      int any = 0;
      for (uint32_t i = 0; i < nd->d0; i++) {
        uint32_t f = a->indices[nd->d1 + i];
        if (a->kind == SO_TRI) {
          if (f == ray->prev_prim) continue;
          st->prim_tests++;
          const float *p0 = &a->verts[3 * (size_t)a->faces[3 * (size_t)f + 0]];
          const float *p1 = &a->verts[3 * (size_t)a->faces[3 * (size_t)f + 1]];
          const float *p2 = &a->verts[3 * (size_t)a->faces[3 * (size_t)f + 2]];
          float u, v;
          if (tri_isect(&t, &u, &v, p0, p1, p2, org, dir, a->keps)) {
            h->t = t;
            h->u = u;
            h->v = v;
            h->prim = f;
            any = 1;
          }
        } else {
          st->prim_tests++;
          float r = sphere_radius(a->radius, a->constr, f);
          if (sphere_isect(&t, &a->verts[3 * (size_t)f], r, org, dir,
                           (double)ray->prev_t, pn, ray->prev_prim == f)) {
            h->t = t;
            h->prim = f;
            any = 1;
          }
        }
      }
      if (any) hitT = h->t;
    }
  }
  if (h->prim == 0xffffffffu || !(h->t < FLT_MAX)) {
    h->t = FLT_MAX;
    h->u = 0.0f;
    h->v = 0.0f;
    h->prim = 0xffffffffu;
  }
  if (subface) *subface = sub;
  if (scalar_out) {
    /* scalar at the entering point: (1-a-b)*s_A + a*s_B + b*s_C over the
     * entering face's vertices in the order the Pluecker test forms its
     * barycentric point (face 3: 0,1,2; 2: 1,0,3; 1: 2,3,0; 0: 3,2,1) */
    float sv = 0.0f;
    if (h->prim != 0xffffffffu && vscalar && a->kind == SO_TET) {
      static const int fa[4] = {3, 2, 1, 0}, fb[4] = {2, 3, 0, 1}, fc[4] = {1, 0, 3, 2};
      const uint32_t *tv = &a->faces[4 * (size_t)h->prim];
      double sa = vscalar[tv[fa[sub]]], sb = vscalar[tv[fb[sub]]], sc = vscalar[tv[fc[sub]]];
      sv = (float)((1.0 - best_e1 - best_e2) * sa + best_e1 * sb + best_e2 * sc);
    }
    *scalar_out = sv;
  }
  return h->prim != 0xffffffffu;
}

static void trace_one(const so_accel *a, const so_ray *ray, const float *prevN,
                      so_hit *h, uint32_t *subface, const float *vscalar,
                      float *scalar_out, so_stats *st) {
  trace_from(a, ray, prevN, h, subface, vscalar, scalar_out, st, FLT_MAX);
}

/* ---- two-pass walk (restatement of the product's default traversal) ----
 * Pass 1: front-to-back (nearer child box first), pruning boxes entered
 * after bound(m), m = running smallest hit distance.  Pass 2: the
 * reference's depth-first order through boxes entered before bound(m),
 * applying the reference's acceptance rule to the candidates at m
 * (tetrahedra: within 8 float steps of m).  This equals the reference's
 * result unless one of those candidates reports a distance below the entry
 * distance of its own leaf box (the same float the reference's box test
 * computes): a box around a primitive at or beyond its entry is entered
 * no later than that primitive's distance, so it is pruned only for a
 * running distance below it, i.e. by a nearer candidate.  The walk then
 * falls back to the reference's walk. */
static inline float bound_rel(float m, float rel) {
  return (m < FLT_MAX) ? m + fabsf(m) * rel + 1e-30f : FLT_MAX;
}
#define SO_REL_TRI 3.90625e-3f      /* 2^-8 */
#define SO_REL_TET 1.52587890625e-5f /* 2^-16 */
/* candidate t below its leaf box entry (NaN counts as below) */
static inline int below_entry(double t, float entry) {
  return !(t >= (double)entry);
}

static inline int ray_aabb_t(float maxT, const float bmin[3], const float bmax[3],
                             const float org[3], const float inv[3], const int sgn[3],
                             int clamp, float *tmin_out) {
  float tmin, tmax;
  const float min_x = sgn[0] ? bmax[0] : bmin[0];
  const float min_y = sgn[1] ? bmax[1] : bmin[1];
  const float min_z = sgn[2] ? bmax[2] : bmin[2];
  const float max_x = sgn[0] ? bmin[0] : bmax[0];
  const float max_y = sgn[1] ? bmin[1] : bmax[1];
  const float max_z = sgn[2] ? bmin[2] : bmax[2];
  const float tmin_x = (min_x - org[0]) * inv[0];
  const float tmax_x = (max_x - org[0]) * inv[0];
  const float tmin_y = (min_y - org[1]) * inv[1];
  const float tmax_y = (max_y - org[1]) * inv[1];
  tmin = (tmin_x > tmin_y) ? tmin_x : tmin_y;
  tmax = (tmax_x < tmax_y) ? tmax_x : tmax_y;
  const float tmin_z = (min_z - org[2]) * inv[2];
  const float tmax_z = (max_z - org[2]) * inv[2];
  tmin = (tmin > tmin_z) ? tmin : tmin_z;
  tmax = (tmax < tmax_z) ? tmax : tmax_z;
  *tmin_out = tmin;
  if (clamp) {
    tmax = (maxT < tmax) ? maxT : tmax;
    return (tmax > 0.0f) && (tmin <= tmax);
  }
  return (tmax > 0.0f) && (tmin <= tmax) && (tmin <= maxT);
}

/* One primitive's hit distance for the two-pass walk; returns 1 on a hit
 * whose distance is stored in *tc (double for tetrahedra).  The per-kind
 * acceptance state is handled by the caller. */
static inline int prim_candidate(const so_accel *a, uint32_t f, const so_ray *ray,
                                 const float *org, const float *dir, const float *pn,
                                 d3 o, d3 d, float tio, double *tc, float *u, float *v,
                                 int *ef, double *e1, double *e2, double *ul1) {
  if (a->kind == SO_TRI) {
    if (f == ray->prev_prim) return 0;
    const float *p0 = &a->verts[3 * (size_t)a->faces[3 * (size_t)f + 0]];
    const float *p1 = &a->verts[3 * (size_t)a->faces[3 * (size_t)f + 1]];
    const float *p2 = &a->verts[3 * (size_t)a->faces[3 * (size_t)f + 2]];
    float t = tio;
    if (!tri_isect(&t, u, v, p0, p1, p2, org, dir, a->keps)) return 0;
    *tc = t;
    return 1;
  }
  if (a->kind == SO_SPHERE) {
    float r = sphere_radius(a->radius, a->constr, f);
    float t = tio;
    if (!sphere_isect(&t, &a->verts[3 * (size_t)f], r, org, dir, (double)ray->prev_t, pn,
                      ray->prev_prim == f))
      return 0;
    *tc = t;
    return 1;
  }
  if (f == ray->prev_prim) return 0;
  d3 V[4];
  for (int j = 0; j < 4; j++) tet_corner(a, a->faces[4 * (size_t)f + j], &V[j]);
  double te;
  if (!ray_tet(o, d, V, ef, e1, e2, ul1, &te) || !(te >= 0.0)) return 0;
  *tc = te;
  return 1;
}

/* window membership: triangles and spheres t == m (float); tetrahedra
 * within 8 float steps above m */
static inline double window_hi(double m, int tet) {
  if (!tet) return m;
  float wf = (float)m;
  for (int k = 0; k < 8; k++) wf = nextafterf(wf, FLT_MAX);
  return (double)wf;
}

typedef struct {
  double t, e1, e2, ul1;
  float u, v;
  uint32_t prim;
  int ef;
  int viol;    /* distance below its own leaf box's entry */
  float entry; /* that entry */
} so_cand;

static void trace2_one(const so_accel *a, const so_ray *ray, const float *prevN,
                       so_hit *h, uint32_t *subface, float *scal, const float *vscalar,
                       so_stats *st, int *fallback) {
  int sgn[3];
  float inv[3];
  for (int k = 0; k < 3; k++) {
    sgn[k] = ray->dir[k] < 0.0f ? 1 : 0;
    inv[k] = (float)(1.0 / (double)ray->dir[k]);
  }
  const float *org = ray->org, *dir = ray->dir;
  float zero3[3] = {0, 0, 0};
  const float *pn = prevN ? prevN : zero3;
  const int tet = a->kind == SO_TET;
  const int clamp = !tet;
  const float rel = tet ? SO_REL_TET : SO_REL_TRI;
  d3 o = {org[0], org[1], org[2]}, d = {dir[0], dir[1], dir[2]};
  int stk[512];
  float stt[512];
  int sp, viol = 0;
  /* ---- pass 1: front to back, collecting the candidates in the window */
  double m = DBL_MAX;
  so_cand win[4];
  int nwin = 0, overflow = 0, viol_lost = 0;
  double m2 = DBL_MAX; /* second smallest distance */
  sp = -1;
  {
    float t0;
    if (!tet || ray_aabb_t(FLT_MAX, a->nodes[0].bmin, a->nodes[0].bmax, org, inv, sgn, 0, &t0)) {
      stk[0] = 0;
      stt[0] = tet ? t0 : -FLT_MAX;
      sp = 0;
    }
  }
  while (sp >= 0) {
    const int ni = stk[sp];
    const float et = stt[sp];
    sp--;
    const float bnd = (m < DBL_MAX) ? bound_rel((float)m, rel) : FLT_MAX;
    if (et > bnd) continue;
    const so_node *nd = &a->nodes[ni];
    if (!nd->leaf) {
      st->branch_visits++;
      float t0, t1;
      const so_node *c0 = &a->nodes[nd->d0], *c1 = &a->nodes[nd->d1];
      int h0 = ray_aabb_t(bnd, c0->bmin, c0->bmax, org, inv, sgn, clamp, &t0);
      int h1 = ray_aabb_t(bnd, c1->bmin, c1->bmax, org, inv, sgn, clamp, &t1);
      if (h0 && h1) {
        int first1 = t1 < t0;
        stk[++sp] = first1 ? (int)nd->d0 : (int)nd->d1; stt[sp] = first1 ? t0 : t1;
        stk[++sp] = first1 ? (int)nd->d1 : (int)nd->d0; stt[sp] = first1 ? t1 : t0;
      } else if (h0) {
        stk[++sp] = (int)nd->d0; stt[sp] = t0;
      } else if (h1) {
        stk[++sp] = (int)nd->d1; stt[sp] = t1;
      }
      continue;
    }
    st->leaf_visits++;
    for (uint32_t i = 0; i < nd->d0; i++) {
      uint32_t f = a->indices[nd->d1 + i];
      st->prim_tests++;
      so_cand c;
      if (!prim_candidate(a, f, ray, org, dir, pn, o, d, FLT_MAX, &c.t, &c.u, &c.v, &c.ef,
                          &c.e1, &c.e2, &c.ul1))
        continue;
      c.prim = f;
      c.viol = below_entry(c.t, et);
      c.entry = et;
      if (c.t < m) {
        m2 = m;
        m = c.t;
        /* drop the candidates that fell out of the window */
        double whi = window_hi(m, tet);
        int k2 = 0;
        for (int k = 0; k < nwin; k++)
          if (win[k].t <= whi) win[k2++] = win[k];
        nwin = k2;
      }
      else if (c.t < m2) {
        m2 = c.t;
      }
      if (c.t <= window_hi(m, tet)) {
        if (nwin < 4) {
          win[nwin++] = c;
        } else {
          overflow = 1;
          viol_lost |= c.viol;
        }
      }
    }
  }
  /* only the candidates left in the window at m can be hidden by the
   * reference's pruning; a dropped candidate's violation is kept.  A single
   * candidate below its box's entry e can only be pruned for a running
   * distance below e, i.e. by another primitive nearer than e: none when the
   * second smallest distance m2 >= e (every such primitive was tested, e
   * lying below pass 1's pruning bound). */
  viol = viol_lost;
  for (int k = 0; k < nwin; k++) viol |= win[k].viol;
  if (viol && nwin == 1 && !overflow)
    viol = !(m2 >= (double)win[0].entry) || !(win[0].entry < bound_rel((float)m, rel));
  h->t = FLT_MAX;
  h->u = 0.0f;
  h->v = 0.0f;
  h->prim = 0xffffffffu;
  uint32_t sub = 0;
  double be1 = 0.0, be2 = 0.0;
  if (!viol && m < DBL_MAX && nwin == 1 && !overflow) {
    /* one candidate in the window: it is the reference's answer */
    h->t = (float)win[0].t;
    h->prim = win[0].prim;
    if (tet) {
      h->u = (float)win[0].e1;
      h->v = (float)win[0].ul1;
      sub = (uint32_t)win[0].ef;
      be1 = win[0].e1;
      be2 = win[0].e2;
    } else if (a->kind == SO_TRI) {
      h->u = win[0].u;
      h->v = win[0].v;
    }
  } else if (!viol && m < DBL_MAX) {
    /* ---- pass 2: several candidates at m; the reference's order decides */
    float bnd, t;
    double whi = window_hi(m, tet);
    if (tet) {
      bnd = bound_rel((float)whi, rel);
      t = FLT_MAX;
    } else {
      bnd = bound_rel((float)m, rel);
      t = (a->kind == SO_TRI) ? (float)m : nextafterf((float)m, FLT_MAX);
    }
    sp = 0;
    stk[0] = 0;
    while (sp >= 0) {
      const so_node *nd = &a->nodes[stk[sp]];
      sp--;
      if (tet) {
        float tm;
        int hit = ray_aabb_t(bnd, nd->bmin, nd->bmax, org, inv, sgn, 0, &tm);
        st->branch_visits++;
        if (!hit) continue;
        if (!nd->leaf) {
          int nearc = sgn[nd->axis], farc = 1 - nearc;
          stk[++sp] = (int)(farc ? nd->d1 : nd->d0);
          stk[++sp] = (int)(nearc ? nd->d1 : nd->d0);
          continue;
        }
      } else if (!nd->leaf) {
        st->branch_visits++;
        const so_node *c0 = &a->nodes[nd->d0], *c1 = &a->nodes[nd->d1];
        int hits[2];
        hits[0] = ray_aabb(bnd, c0->bmin, c0->bmax, org, inv, sgn, 1);
        hits[1] = ray_aabb(bnd, c1->bmin, c1->bmax, org, inv, sgn, 1);
        if (hits[0] || hits[1]) {
          int nearc = sgn[nd->axis], farc = 1 - nearc;
          if (hits[farc]) stk[++sp] = (int)(farc ? nd->d1 : nd->d0);
          if (hits[nearc]) stk[++sp] = (int)(nearc ? nd->d1 : nd->d0);
        }
        continue;
      }
      st->leaf_visits++;
      for (uint32_t i = 0; i < nd->d0; i++) {
        uint32_t f = a->indices[nd->d1 + i];
        st->prim_tests++;
        so_cand c;
        if (!prim_candidate(a, f, ray, org, dir, pn, o, d, FLT_MAX, &c.t, &c.u, &c.v, &c.ef,
                            &c.e1, &c.e2, &c.ul1))
          continue;
        if (tet) {
          if (c.t <= whi && c.t < (double)t) {
            h->t = (float)c.t; h->u = (float)c.e1; h->v = (float)c.ul1; h->prim = f;
            sub = (uint32_t)c.ef;
            be1 = c.e1;
            be2 = c.e2;
            t = (float)c.t;
          }
        } else if (a->kind == SO_TRI) {
          if ((float)c.t <= t) {
            t = (float)c.t; h->t = t; h->u = c.u; h->v = c.v; h->prim = f;
          }
        } else if ((float)c.t < t) {
          t = (float)c.t; h->t = t; h->prim = f;
        }
      }
    }
  }
  if (viol) {
    /* a candidate reported a distance below its leaf box's entry: the
     * reference's pruning may matter, so take its walk.  Started from the
     * pruning bound T of pass 1 it returns the same primitive: the answer
     * and every primitive that can prune its boxes lie below T by more than
     * the float error of a distance, so a running distance at or above T
     * (which the full walk may hold on the way) prunes none of them.  If
     * nothing is accepted below T, the full walk decides. */
    if (!trace_from(a, ray, prevN, h, subface, vscalar, scal, st, bound_rel((float)m, rel)))
      trace_one(a, ray, prevN, h, subface, vscalar, scal, st);
    if (fallback) *fallback = 1;
    return;
  }
  if (subface) *subface = sub;
  if (scal) {
    float sv = 0.0f;
    if (h->prim != 0xffffffffu && vscalar && tet) {
      static const int fa[4] = {3, 2, 1, 0}, fb[4] = {2, 3, 0, 1}, fc[4] = {1, 0, 3, 2};
      const uint32_t *tv = &a->faces[4 * (size_t)h->prim];
      double sa = vscalar[tv[fa[sub]]], sb = vscalar[tv[fb[sub]]], sc = vscalar[tv[fc[sub]]];
      sv = (float)((1.0 - be1 - be2) * sa + be1 * sb + be2 * sc);
    }
    *scal = sv;
  }
}

/* ---- BuildIntersection: the shading record of a hit ----------------------
 * The fields the reference's Traverse fills after the closest hit is known
 * and the GLSL stage reads (gles/gles_common.cc:1007-1141).  Record layout
 * (80 bytes, the product's srt_isect): position, f0, normal, f1, tangent, f2,
 * binormal, f3, d[4]; a miss is all zero.  Float arithmetic in the
 * reference's order; the spheres' angles from the C library's double atan2
 * and acos, which is what the reference's unqualified atan2 / acos calls on
 * floats resolve to in its build (checked against its outputs). */
typedef struct {
  float position[3];
  uint32_t f0;
  float normal[3];
  uint32_t f1;
  float tangent[3];
  uint32_t f2;
  float binormal[3];
  uint32_t f3;
  float d[4];
} so_isect;

static inline void sub3f(const float a[3], const float b[3], float c[3]) {
  c[0] = a[0] - b[0];
  c[1] = a[1] - b[1];
  c[2] = a[2] - b[2];
}
/* real3::length (render/render_common.h) */
static inline float len3f(const float a[3]) {
  return (float)sqrt((double)(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]));
}
/* real3::normalize (render/render_common.h): scale by 1/sqrt in double */
static inline void normalize_real3(float n[3]) {
  double l2 = n[0] * n[0] + n[1] * n[1] + n[2] * n[2];
  double len = 0.0;
  if (fabs(l2) > 1.0e-30) len = 1.0 / sqrt(l2);
  for (int k = 0; k < 3; k++) n[k] = (float)(n[k] * len);
}
/* vnormalize (render/render_accel_particle.cc:2041-2056) */
static inline void vnormalize_p(float n[3]) {
  const float kEPS = FLT_EPSILON * 16.0;
  float len = (float)sqrt((double)dot3f(n, n));
  if (len > kEPS) {
    float inv = (float)(1.0 / len);
    n[0] *= inv;
    n[1] *= inv;
    n[2] *= inv;
  }
}
/* Spherical (u, v) of a unit normal (render/render_accel_particle.cc:3013-3014) */
static inline void sphere_uv_ref(const float n[3], float *u, float *v) {
  *u = (float)((atan2((double)n[0], (double)n[2]) + M_PI) * 0.5 * (1.0 / M_PI));
  *v = (float)(acos((double)n[1]) / M_PI);
}

/* InterpolateTetra (render/render_accel_tetra.cc:148-241), mode 0. */
static void interpolate_tetra(const float pt[3], const float V[4][3], float dout[4]) {
  static const int fl[4][3] = {{0, 2, 1}, {1, 2, 3}, {0, 3, 2}, {0, 1, 3}};
  const float kEPS = 0.001;
  float E[6][3];
  sub3f(V[1], V[0], E[0]);
  sub3f(V[2], V[1], E[1]);
  sub3f(V[0], V[2], E[2]);
  sub3f(V[3], V[0], E[3]);
  sub3f(V[3], V[1], E[4]);
  sub3f(V[3], V[2], E[5]);
  for (int v = 0; v < 4; v++) {
    const float *ro = V[v];
    float rd[3], pc[3], tmp[3];
    sub3f(pt, ro, rd);
    cross3f(rd, ro, pc);
    sub3f(pt, ro, tmp);
    float d = len3f(tmp);
    float ws[6];
    int cw0[6], cw1[6];
    for (int i = 0; i < 6; i++) {
      float cv[3];
      cross3f(E[i], V[i % 3], cv);
      ws[i] = dot3f(rd, cv) + dot3f(E[i], pc);
      cw0[i] = ws[i] >= -kEPS;
      cw1[i] = ws[i] <= kEPS;
    }
    int in[4];
    for (int f = 0; f < 4; f++) in[f] = fl[f][0] == v || fl[f][1] == v || fl[f][2] == v;
    float cp[3] = {1e16f, 1e16f, 1e16f};
    if (cw0[0] && cw0[1] && cw0[2] && !in[0]) {
      float s = ws[0] + ws[1] + ws[2];
      for (int k = 0; k < 3; k++) cp[k] = (V[2][k] * ws[0] + V[0][k] * ws[1] + V[1][k] * ws[2]) / s;
    } else if (cw1[1] && cw0[4] && cw1[5] && !in[1]) {
      float s = ws[5] + ws[1] - ws[4];
      for (int k = 0; k < 3; k++) cp[k] = (V[3][k] * ws[1] + V[1][k] * ws[5] - V[2][k] * ws[4]) / s;
    } else if (cw1[2] && cw1[3] && cw0[5] && !in[2]) {
      float s = ws[2] + ws[3] - ws[5];
      for (int k = 0; k < 3; k++) cp[k] = (V[3][k] * ws[2] + V[2][k] * ws[3] - V[0][k] * ws[5]) / s;
    } else if (cw1[0] && cw0[3] && cw1[4] && !in[3]) {
      float s = ws[0] + ws[4] - ws[3];
      for (int k = 0; k < 3; k++) cp[k] = (V[3][k] * ws[0] + V[0][k] * ws[4] - V[1][k] * ws[3]) / s;
    }
    float cr[3];
    sub3f(cp, ro, cr);
    dout[v] = d / len3f(cr);
    if (dout[v] < 0) {
      dout[v] = 0;
    } else if (!(dout[v] < 1) && !(dout[v] > 0)) {
      dout[v] = 1;
    }
    dout[v] = 1 - dout[v];
  }
  float ds = 0, dd[4], w = 0;
  for (int i = 0; i < 4; i++) {
    float r[3];
    sub3f(pt, V[i], r);
    ds += len3f(r);
  }
  for (int i = 0; i < 4; i++) {
    float r[3];
    sub3f(pt, V[i], r);
    dd[i] = ds / len3f(r);
  }
  for (int i = 0; i < 4; i++) {
    dout[i] *= dd[i];
    w += dout[i];
  }
  for (int i = 0; i < 4; i++) dout[i] = dout[i] / w;
}

static void build_isect(const so_accel *a, const so_ray *ray, const so_hit *h, uint32_t sub,
                        so_isect *o) {
  memset(o, 0, sizeof(*o));
  if (h->prim == 0xffffffffu) return;
  const uint32_t prim = h->prim;
  for (int k = 0; k < 3; k++) o->position[k] = ray->org[k] + h->t * ray->dir[k];
  if (a->kind == SO_TRI) {
    const uint32_t *fv = &a->faces[3 * (size_t)prim];
    o->f0 = fv[0];
    o->f1 = fv[1];
    o->f2 = fv[2];
    const float *p0 = &a->verts[3 * (size_t)fv[0]], *p1 = &a->verts[3 * (size_t)fv[1]],
                *p2 = &a->verts[3 * (size_t)fv[2]];
    float e1[3], e2[3];
    sub3f(p1, p0, e1);
    sub3f(p2, p0, e2);
    cross3f(e1, e2, o->normal);
    normalize_real3(o->normal);
  } else if (a->kind == SO_TET) {
    static const int ft[4][3] = {{0, 1, 3}, {1, 2, 3}, {2, 0, 3}, {0, 1, 2}};
    const uint32_t *fv = &a->faces[4 * (size_t)prim];
    o->f0 = fv[0];
    o->f1 = fv[1];
    o->f2 = fv[2];
    o->f3 = fv[3];
    float p[4][3];
    for (int j = 0; j < 4; j++)
      for (int k = 0; k < 3; k++) p[j][k] = a->verts[3 * (size_t)fv[j] + k];
    float e1[3], e2[3];
    sub3f(p[ft[sub & 3][1]], p[ft[sub & 3][0]], e1);
    sub3f(p[ft[sub & 3][2]], p[ft[sub & 3][0]], e2);
    cross3f(e1, e2, o->normal);
    normalize_real3(o->normal);
    interpolate_tetra(o->position, (const float(*)[3])p, o->d);
  } else {
    o->f0 = o->f1 = o->f2 = prim;
    const float *c = &a->verts[3 * (size_t)prim];
    float *n = o->normal;
    sub3f(o->position, c, n);
    vnormalize_p(n);
    float xz2 = n[0] * n[0] + n[2] * n[2];
    if (xz2 > 0.0) {
      float xz = sqrtf(xz2);
      float inv = (float)(1.0 / xz);
      o->tangent[0] = (float)(-2.0 * M_PI * n[0]);
      o->tangent[1] = (float)(2.0 * M_PI * n[2]);
      o->tangent[2] = 0.0f;
      o->binormal[0] = (float)(-M_PI * n[2] * inv * n[1]);
      o->binormal[1] = (float)(-M_PI * n[0] * inv * n[1]);
      o->binormal[2] = (float)(M_PI * xz);
    } else {
      o->tangent[2] = 1.0f;
      o->binormal[0] = n[1] > 0.0 ? 1.0f : -1.0f;
    }
  }
}

/* The sphere hit's (u, v) as the reference's Traverse returns them: the
 * spherical coordinates BuildIntersection computes from its normal. */
static void sphere_finish(const so_accel *a, const so_ray *ray, so_hit *h) {
  if (a->kind != SO_SPHERE || h->prim == 0xffffffffu) return;
  so_isect r;
  build_isect(a, ray, h, 0, &r);
  sphere_uv_ref(r.normal, &h->u, &h->v);
}

/* Shading records of n traced rays (hits and, for tetrahedra, entering
 * faces from so_trace / so_trace2). */
SO_API void so_isect_records(const so_accel *a, const so_ray *rays, size_t n,
                             const so_hit *hits, const uint32_t *subface, so_isect *out,
                             int nthreads) {
#ifdef _OPENMP
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(static) num_threads(nthreads)
#endif
  for (long long i = 0; i < (long long)n; i++)
    build_isect(a, &rays[i], &hits[i], subface ? subface[i] : 0u, &out[i]);
}

/* stats (optional): 4 x uint64 (branch visits, leaf visits, primitive
 * tests, rays that fell back to the reference's walk). */
SO_API void so_trace2(const so_accel *a, const so_ray *rays, size_t n,
                      const float *prev_normals, so_hit *hits, uint32_t *subface,
                      uint64_t *stats, int nthreads) {
  uint64_t bv = 0, lv = 0, pt = 0, fb = 0;
#ifdef _OPENMP
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 256) num_threads(nthreads) reduction(+ : bv, lv, pt, fb)
#endif
  for (long long i = 0; i < (long long)n; i++) {
    so_stats st = {0, 0, 0};
    int fall = 0;
    trace2_one(a, &rays[i], prev_normals ? &prev_normals[3 * i] : NULL, &hits[i],
               subface ? &subface[i] : NULL, NULL, NULL, &st, &fall);
    sphere_finish(a, &rays[i], &hits[i]);
    bv += st.branch_visits;
    lv += st.leaf_visits;
    pt += st.prim_tests;
    fb += (uint64_t)fall;
  }
  if (stats) {
    stats[0] = bv;
    stats[1] = lv;
    stats[2] = pt;
    stats[3] = fb;
  }
}

/* Trace `n` rays.  prev_normals: 3 floats per ray or NULL.  subface: per-ray
 * output for tetrahedra or NULL.  vscalar/scalar_out: per-vertex scalar and
 * its value at the entering point (tetrahedra).  stats (optional): 3 x uint64
 * totals (branch visits, leaf visits, primitive tests). */
SO_API void so_trace(const so_accel *a, const so_ray *rays, size_t n,
                     const float *prev_normals, so_hit *hits, uint32_t *subface,
                     const float *vscalar, float *scalar_out, uint64_t *stats,
                     int nthreads) {
  uint64_t bv = 0, lv = 0, pt = 0;
#ifdef _OPENMP
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 256) num_threads(nthreads) reduction(+ : bv, lv, pt)
#endif
  for (long long i = 0; i < (long long)n; i++) {
    so_stats st = {0, 0, 0};
    trace_one(a, &rays[i], prev_normals ? &prev_normals[3 * i] : NULL, &hits[i],
              subface ? &subface[i] : NULL, vscalar,
              scalar_out ? &scalar_out[i] : NULL, &st);
    sphere_finish(a, &rays[i], &hits[i]);
    bv += st.branch_visits;
    lv += st.leaf_visits;
    pt += st.prim_tests;
  }
  if (stats) {
    stats[0] = bv;
    stats[1] = lv;
    stats[2] = pt;
  }
}

/* ------------------------------------------------------------------------ */
/* Trilinear 3D fetch (FilterTexture3DFloat, render/render_texture.cc:946)   */
/* ------------------------------------------------------------------------ */

static inline int floor_ref(float x) { /* fasterfloorf, render_texture.cc:106 */
  if (x >= 0) return (int)x;
  int y = (int)x;
  if (fabsf(x - (float)y) <= FLT_EPSILON) {
  } else {
    y = y - 1;
  }
  return y;
}
static inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
/* local::remap (gles/gles_common.h:264-269) */
static inline float remap_ref(float x, const float *table, int n) {
  int idx = (int)(x * n);
  idx = idx > n - 1 ? n - 1 : idx;
  idx = idx < 0 ? 0 : idx;
  return table[idx];
}
static inline float lerpf(float t, float a, float b) { return (1.f - t) * a + t * b; }

/* Scalar (1-component) volume fetch with the reference's texel-corner
 * mapping vox = u * (dim - 1). */
static float tex3d_f32(const float *img, const int dim[3], float u, float v,
                       float r, int clamp_s, int clamp_t, int clamp_r) {
  float uu = clamp_s ? u : u - floor_ref(u);
  float vv = clamp_t ? v : v - floor_ref(v);
  float rr = clamp_r ? r : r - floor_ref(r);
  float vox0 = uu * (dim[0] - 1.0f);
  float vox1 = vv * (dim[1] - 1.0f);
  float vox2 = rr * (dim[2] - 1.0f);
  int vx = clampi((int)vox0, 0, dim[0] - 1);
  int vy = clampi((int)vox1, 0, dim[1] - 1);
  int vz = clampi((int)vox2, 0, dim[2] - 1);
  int vx1 = vx + 1 < dim[0] - 1 ? vx + 1 : dim[0] - 1;
  int vy1 = vy + 1 < dim[1] - 1 ? vy + 1 : dim[1] - 1;
  int vz1 = vz + 1 < dim[2] - 1 ? vz + 1 : dim[2] - 1;
  float dx = vox0 - vx, dy = vox1 - vy, dz = vox2 - vz;
#define A(x, y, z) img[(size_t)(z) * dim[0] * dim[1] + (size_t)(y) * dim[0] + (x)]
  float d00 = lerpf(dx, A(vx, vy, vz), A(vx1, vy, vz));
  float d10 = lerpf(dx, A(vx, vy1, vz), A(vx1, vy1, vz));
  float d01 = lerpf(dx, A(vx, vy, vz1), A(vx1, vy, vz1));
  float d11 = lerpf(dx, A(vx, vy1, vz1), A(vx1, vy1, vz1));
#undef A
  float d0 = lerpf(dy, d00, d10);
  float d1 = lerpf(dy, d01, d11);
  return lerpf(dz, d0, d1);
}

SO_API void so_tex3d(const float *img, const int dim[3], const float *uvw,
                     size_t m, int clamp_s, int clamp_t, int clamp_r, float *out) {
  for (size_t i = 0; i < m; i++)
    out[i] = tex3d_f32(img, dim, uvw[3 * i], uvw[3 * i + 1], uvw[3 * i + 2],
                       clamp_s, clamp_t, clamp_r);
}

/* ------------------------------------------------------------------------ */
/* Emission-absorption volume march                                          */
/* ------------------------------------------------------------------------ */

/* Parameters shared with the CUDA kernel (srt_volume_params in the C ABI).
 * The camera frame is precomputed once on the host (so_volume_camera). */
typedef struct {
  int width, height;        /* image size */
  int max_steps;            /* hard cap on samples per ray */
  int reserved;
  float eye[3];
  float corner[3];          /* image-plane corner */
  float du[3], dv[3];       /* per-pixel image-plane steps */
  float step;               /* world-space distance between samples */
  float sigma_scale;        /* extinction = sigma_scale * tf.a */
  float alpha_max;          /* per-sample opacity clamp (< 1) */
} so_vol_params;

/* build_cameraframe (examples/nonuniform_volume_render/input.frag:16-29),
 * FP32, including the shader's 3.14 for pi. */
SO_API void so_volume_camera(int W, int H, const float eye[3],
                             const float lookat[3], const float up[3],
                             float fov_deg, float corner[3], float du[3],
                             float dv[3]) {
  float look[3], tmp[3];
  for (int k = 0; k < 3; k++) look[k] = lookat[k] - eye[k];
  float ll = sqrtf(dot3f(look, look));
  for (int k = 0; k < 3; k++) look[k] = look[k] / ll;
  cross3f(look, up, tmp);
  float lu = sqrtf(dot3f(tmp, tmp));
  for (int k = 0; k < 3; k++) du[k] = tmp[k] / lu;
  cross3f(look, du, tmp);
  float lv = sqrtf(dot3f(tmp, tmp));
  for (int k = 0; k < 3; k++) dv[k] = tmp[k] / lv;
  float flen = 0.5f * (float)H / (float)tan(0.5 * ((double)fov_deg * 3.14 / 180.0));
  for (int k = 0; k < 3; k++) {
    float lk = flen * look[k] + eye[k];
    corner[k] = lk - 0.5f * ((float)W * du[k] + (float)H * dv[k]);
  }
}

/* Ray through fragment centre (px+0.5, py+0.5) (input.frag:101-108). */
static void vol_ray_f32(const so_vol_params *P, int px, int py, float org[3],
                        float dir[3]) {
  float fx = (float)px + 0.5f, fy = (float)py + 0.5f;
  float d[3];
  for (int k = 0; k < 3; k++)
    d[k] = (P->corner[k] + fx * P->du[k] + fy * P->dv[k]) - P->eye[k];
  float dl = sqrtf(dot3f(d, d));
  for (int k = 0; k < 3; k++) {
    dir[k] = d[k] / dl;
    org[k] = P->eye[k];
  }
}

/* IntersectP against [-1,1]^3 (input.frag:59-97). */
static int vol_slab_f32(const float o[3], const float d[3], float *t0o, float *t1o) {
  float t0 = -10000.0f, t1 = 10000.0f;
  for (int k = 0; k < 3; k++) {
    float tn = (-1.0f - o[k]) / d[k];
    float tf = (1.0f - o[k]) / d[k];
    if (tn > tf) { float x = tn; tn = tf; tf = x; }
    t0 = tn > t0 ? tn : t0;
    t1 = tf < t1 ? tf : t1;
  }
  *t0o = t0;
  *t1o = t1;
  return t0 <= t1;
}

static inline int vol_inside_f(const float p[3]) {
  return p[0] >= -1.0f && p[0] < 1.0f && p[1] >= -1.0f && p[1] < 1.0f &&
         p[2] >= -1.0f && p[2] < 1.0f;
}

/* Forward march, FP32.  img: width*height*4 (RGB premultiplied, A = 1 - T). */
/* The density texture's sampling state (srt_volume_sampling): per-axis
 * remap tables (local::remap) and clamp-to-edge flags (0: repeat wrap).
 * NULL: clamp-to-edge, no remap. */
typedef struct {
  const float *remap[3];
  uint32_t remap_n[3];
  int32_t clamp[3];
} so_sampling;

static inline float samp_f32(const so_sampling *S, int k, float u) {
  if (!S) return u;
  if (S->remap[k] && S->remap_n[k]) u = remap_ref(u, S->remap[k], (int)S->remap_n[k]);
  if (!S->clamp[k]) u = u - floor_ref(u);
  return u;
}

static inline double samp_f64(const so_sampling *S, int k, double q) {
  if (!S) return q;
  if (S->remap[k] && S->remap_n[k]) {
    const int n = (int)S->remap_n[k];
    int idx = (int)(q * n);
    idx = idx > n - 1 ? n - 1 : (idx < 0 ? 0 : idx);
    q = S->remap[k][idx];
  }
  if (!S->clamp[k]) q = q - floor(q);
  return q;
}

static void vol_fwd_f32(const so_vol_params *P, const so_sampling *S, const float *dens,
                        const int dim[3], const float *tf, float *img, int nthreads);

SO_API void so_volume_fwd_f32(const so_vol_params *P, const float *dens,
                              const int dim[3], const float *tf, float *img,
                              int nthreads) {
  vol_fwd_f32(P, NULL, dens, dim, tf, img, nthreads);
}

SO_API void so_volume_fwd_f32_ex(const so_vol_params *P, const so_sampling *S,
                                 const float *dens, const int dim[3], const float *tf,
                                 float *img, int nthreads) {
  vol_fwd_f32(P, S, dens, dim, tf, img, nthreads);
}

static void vol_fwd_f32(const so_vol_params *P, const so_sampling *S, const float *dens,
                        const int dim[3], const float *tf, float *img, int nthreads) {
  int W = P->width, H = P->height;
#ifdef _OPENMP
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 4) num_threads(nthreads)
#endif
  for (int py = 0; py < H; py++) {
    for (int px = 0; px < W; px++) {
      float o[3], d[3], t0, t1;
      vol_ray_f32(P, px, py, o, d);
      float C[3] = {0, 0, 0}, T = 1.0f;
      if (vol_slab_f32(o, d, &t0, &t1)) {
        int ns = (int)((t1 - t0) / P->step);
        if (ns > P->max_steps) ns = P->max_steps;
        for (int s = 0; s < ns; s++) {
          float t = t0 + ((float)s + 0.5f) * P->step;
          float p[3] = {o[0] + t * d[0], o[1] + t * d[1], o[2] + t * d[2]};
          if (!vol_inside_f(p)) continue;
          float rho = tex3d_f32(dens, dim, samp_f32(S, 0, 0.5f * p[0] + 0.5f),
                                samp_f32(S, 1, 0.5f * p[1] + 0.5f),
                                samp_f32(S, 2, 0.5f * p[2] + 0.5f), 1, 1, 1);
          float x = rho * 255.0f;
          x = x < 0.0f ? 0.0f : (x > 255.0f ? 255.0f : x);
          int i0 = (int)x;
          int i1 = i0 + 1 < 255 ? i0 + 1 : 255;
          float f = x - (float)i0;
          float c[4];
          for (int k = 0; k < 4; k++) c[k] = lerpf(f, tf[4 * i0 + k], tf[4 * i1 + k]);
          float sig = P->sigma_scale * c[3];
          float al = 1.0f - expf(-sig * P->step);
          if (al > P->alpha_max) al = P->alpha_max;
          float w = T * al;
          for (int k = 0; k < 3; k++) C[k] += w * c[k];
          T = T * (1.0f - al);
        }
      }
      float *out = &img[4 * ((size_t)py * W + px)];
      out[0] = C[0];
      out[1] = C[1];
      out[2] = C[2];
      out[3] = 1.0f - T;
    }
  }
}

/* ---- FP64 forward + analytic adjoint (reference gradient) --------------- */


static void vol_ray_f64(const so_vol_params *P, int px, int py, double o[3], double dir[3]) {
  /* same construction as the FP32 path, in double, so that the ray set is
   * the FP32 one to within rounding */
  float of[3], df[3];
  vol_ray_f32(P, px, py, of, df);
  for (int k = 0; k < 3; k++) {
    o[k] = of[k];
    dir[k] = df[k];
  }
}

static double tex3d_f64(const double *img, const int dim[3], const double q[3],
                        int cx[8], double w[8]) {
  double vox[3];
  int v0[3], v1[3];
  double fr[3];
  for (int k = 0; k < 3; k++) {
    vox[k] = q[k] * (dim[k] - 1.0);
    int vi = (int)vox[k];
    vi = clampi(vi, 0, dim[k] - 1);
    v0[k] = vi;
    v1[k] = vi + 1 < dim[k] - 1 ? vi + 1 : dim[k] - 1;
    fr[k] = vox[k] - vi;
  }
  double val = 0.0;
  for (int c = 0; c < 8; c++) {
    int ix = (c & 1) ? v1[0] : v0[0];
    int iy = (c & 2) ? v1[1] : v0[1];
    int iz = (c & 4) ? v1[2] : v0[2];
    double wx = (c & 1) ? fr[0] : 1.0 - fr[0];
    double wy = (c & 2) ? fr[1] : 1.0 - fr[1];
    double wz = (c & 4) ? fr[2] : 1.0 - fr[2];
    cx[c] = (iz * dim[1] + iy) * dim[0] + ix;
    w[c] = wx * wy * wz;
    val += w[c] * img[cx[c]];
  }
  return val;
}

/* FP64 march.  If target != NULL returns loss = sum((img - target)^2) and,
 * when grad_dens/grad_tf are non-NULL, accumulates the analytic gradients
 * (reverse-order transmittance recomputation, the same scheme as the CUDA
 * adjoint).  img (optional): width*height*4 output. */
static double vol_f64(const so_vol_params *P, const so_sampling *S, const double *dens,
                      const int dim[3], const double *tf, const float *target, double *img,
                      double *grad_dens, double *grad_tf, const uint32_t *pixels,
                      size_t npix);

SO_API double so_volume_f64(const so_vol_params *P, const double *dens,
                            const int dim[3], const double *tf,
                            const float *target, double *img, double *grad_dens,
                            double *grad_tf) {
  return vol_f64(P, NULL, dens, dim, tf, target, img, grad_dens, grad_tf, NULL, 0);
}

/* The loss over a subset of pixels (indices py * W + px) -- for finite
 * differences of a local perturbation, which changes only the pixels whose
 * rays pass near it. */
SO_API double so_volume_f64_pixels(const so_vol_params *P, const double *dens,
                                   const int dim[3], const double *tf, const float *target,
                                   const uint32_t *pixels, size_t npix) {
  return vol_f64(P, NULL, dens, dim, tf, target, NULL, NULL, NULL, pixels, npix);
}

SO_API double so_volume_f64_ex(const so_vol_params *P, const so_sampling *S,
                               const double *dens, const int dim[3], const double *tf,
                               const float *target, double *img, double *grad_dens,
                               double *grad_tf) {
  return vol_f64(P, S, dens, dim, tf, target, img, grad_dens, grad_tf, NULL, 0);
}

/* pixels: NULL for every pixel of the image, else the npix pixel indices
 * (py * W + px) whose loss (and gradient) is taken.  Pixels run in parallel;
 * gradients are accumulated with atomic adds (the order of the double sums
 * then varies from run to run, within rounding). */
static double vol_f64(const so_vol_params *P, const so_sampling *S, const double *dens,
                      const int dim[3], const double *tf, const float *target, double *img,
                      double *grad_dens, double *grad_tf, const uint32_t *pixels,
                      size_t npix) {
  int W = P->width, H = P->height;
  double loss = 0.0;
  const double step = P->step;
  const int maxs = P->max_steps;
  const long long count = pixels ? (long long)npix : (long long)W * H;
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : loss)
#endif
  for (long long item = 0; item < count; item++) {
    {
      const long long pix = pixels ? (long long)pixels[item] : item;
      const int py = (int)(pix / W), px = (int)(pix % W);
      double o[3], d[3];
      vol_ray_f64(P, px, py, o, d);
      /* slab test in double mirroring the FP32 one */
      double t0 = -10000.0, t1 = 10000.0;
      for (int k = 0; k < 3; k++) {
        double tn = (-1.0 - o[k]) / d[k], tf_ = (1.0 - o[k]) / d[k];
        if (tn > tf_) { double x = tn; tn = tf_; tf_ = x; }
        t0 = tn > t0 ? tn : t0;
        t1 = tf_ < t1 ? tf_ : t1;
      }
      double C[3] = {0, 0, 0}, T = 1.0;
      int ns = 0;
      if (t0 <= t1) {
        /* the sample count is taken from the FP32 path so both march the
         * same samples */
        float of[3], df[3], f0, f1;
        vol_ray_f32(P, px, py, of, df);
        vol_slab_f32(of, df, &f0, &f1);
        ns = (int)((f1 - f0) / P->step);
        if (ns > maxs) ns = maxs;
      }
      for (int s = 0; s < ns; s++) {
        double t = t0 + (s + 0.5) * step;
        double p[3] = {o[0] + t * d[0], o[1] + t * d[1], o[2] + t * d[2]};
        if (!(p[0] >= -1 && p[0] < 1 && p[1] >= -1 && p[1] < 1 && p[2] >= -1 && p[2] < 1))
          continue;
        double q[3] = {samp_f64(S, 0, 0.5 * p[0] + 0.5), samp_f64(S, 1, 0.5 * p[1] + 0.5),
                       samp_f64(S, 2, 0.5 * p[2] + 0.5)};
        int cx[8];
        double w[8];
        double rho = tex3d_f64(dens, dim, q, cx, w);
        double x = rho * 255.0;
        x = x < 0 ? 0 : (x > 255 ? 255 : x);
        int i0 = (int)x, i1 = i0 + 1 < 255 ? i0 + 1 : 255;
        double f = x - i0;
        double c[4];
        for (int k = 0; k < 4; k++) c[k] = (1 - f) * tf[4 * i0 + k] + f * tf[4 * i1 + k];
        double al = 1.0 - exp(-P->sigma_scale * c[3] * step);
        if (al > P->alpha_max) al = P->alpha_max;
        for (int k = 0; k < 3; k++) C[k] += T * al * c[k];
        T *= (1.0 - al);
      }
      double out[4] = {C[0], C[1], C[2], 1.0 - T};
      if (img)
        for (int k = 0; k < 4; k++) img[4 * ((size_t)py * W + px) + k] = out[k];
      if (!target) continue;
      const float *tg = &target[4 * ((size_t)py * W + px)];
      double dC[4];
      for (int k = 0; k < 4; k++) {
        double e = out[k] - tg[k];
        loss += e * e;
        dC[k] = 2.0 * e;
      }
      if (!grad_dens && !grad_tf) continue;
      /* reverse pass: T_k = T_{k+1} / (1 - a_k); Cb = colour of the samples behind k */
      double Tn = T;         /* transmittance after the current sample */
      double Cb[3] = {0, 0, 0}; /* accumulated color of samples behind */
      for (int s = ns - 1; s >= 0; s--) {
        double t = t0 + (s + 0.5) * step;
        double p[3] = {o[0] + t * d[0], o[1] + t * d[1], o[2] + t * d[2]};
        if (!(p[0] >= -1 && p[0] < 1 && p[1] >= -1 && p[1] < 1 && p[2] >= -1 && p[2] < 1))
          continue;
        double q[3] = {samp_f64(S, 0, 0.5 * p[0] + 0.5), samp_f64(S, 1, 0.5 * p[1] + 0.5),
                       samp_f64(S, 2, 0.5 * p[2] + 0.5)};
        int cx[8];
        double w[8];
        double rho = tex3d_f64(dens, dim, q, cx, w);
        double xr = rho * 255.0;
        int inr = (xr > 0.0 && xr < 255.0);
        double x = xr < 0 ? 0 : (xr > 255 ? 255 : xr);
        int i0 = (int)x, i1 = i0 + 1 < 255 ? i0 + 1 : 255;
        double f = x - i0;
        double c[4];
        for (int k = 0; k < 4; k++) c[k] = (1 - f) * tf[4 * i0 + k] + f * tf[4 * i1 + k];
        double e = exp(-P->sigma_scale * c[3] * step);
        double al = 1.0 - e;
        int clamped = al > P->alpha_max;
        if (clamped) al = P->alpha_max;
        double Tk = Tn / (1.0 - al);
        /* dL/dc_rgb = dC * T_k * a_k */
        double gc[4];
        for (int k = 0; k < 3; k++) gc[k] = dC[k] * Tk * al;
        /* dL/da_k */
        double ga = 0.0;
        for (int k = 0; k < 3; k++) ga += dC[k] * (Tk * c[k] - Cb[k] / (1.0 - al));
        ga += dC[3] * (T / (1.0 - al)); /* dA/da_k = T_final / (1 - a_k) */
        /* a = 1 - exp(-s*c_a*step) -> da/dc_a = s*step*exp(...) */
        gc[3] = clamped ? 0.0 : ga * P->sigma_scale * step * e;
        if (grad_tf) {
          for (int k = 0; k < 4; k++) {
            const double g0 = (1 - f) * gc[k], g1 = f * gc[k];
#ifdef _OPENMP
#pragma omp atomic
#endif
            grad_tf[4 * i0 + k] += g0;
#ifdef _OPENMP
#pragma omp atomic
#endif
            grad_tf[4 * i1 + k] += g1;
          }
        }
        if (grad_dens && inr) {
          double drho = 0.0;
          for (int k = 0; k < 4; k++) drho += gc[k] * (tf[4 * i1 + k] - tf[4 * i0 + k]);
          drho *= 255.0;
          for (int cc = 0; cc < 8; cc++) {
            const double g = w[cc] * drho;
#ifdef _OPENMP
#pragma omp atomic
#endif
            grad_dens[cx[cc]] += g;
          }
        }
        for (int k = 0; k < 3; k++) Cb[k] += Tk * al * c[k];
        Tn = Tk;
      }
    }
  }
  return loss;
}

/* ======================================================== eye rays, frames
 * RaytraceEngine::OnData's eye rays and framebuffer write for one sample per
 * pixel (gles/gles_raytrace_engine.cc:547-879), restated:
 *   - Camera::buildFrame (render/render_camera.cc:17-63), float arithmetic
 *     with real3::normalize's double reciprocal length
 *     (render/render_common.h:69-83);
 *   - ViewportConversion (gles/gles_raytrace_engine.cc:530-544);
 *   - per pixel (x, y) of the render region in steps of `step`: the
 *     viewport-converted pixel (px, py), and the ray through
 *     corner + (px + step/2) u + (py - step/2 + 1) v (:770-795);
 *   - the write of a hit: the step x step block at (x + u, height - y - 1 + v)
 *     gets the colour (RGBA8 via clamp() (:50-58) or RGBA32F) and the depth t
 *     (:840-877).  Rows above the framebuffer are skipped (the reference
 *     would write outside it). */

static void cam_norm(float v[3]) {
  double l2 = (double)(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  double l = 0.0;
  if (fabs(l2) > 1.0e-30) l = 1.0 / sqrt(l2);
  for (int k = 0; k < 3; k++) v[k] = (float)((double)v[k] * l);
}

static void cam_cross(const float a[3], const float b[3], float o[3]) {
  o[0] = a[1] * b[2] - a[2] * b[1];
  o[1] = a[2] * b[0] - a[0] * b[2];
  o[2] = a[0] * b[1] - a[1] * b[0];
}

/* out = corner[3], u[3], v[3] */
SO_API void so_camera_frame(const float eye[3], const float lookat[3], const float up[3],
                            float fov, int ortho, int width, int height, float out[9]) {
  float look[3], u[3], v[3], corner[3];
  for (int k = 0; k < 3; k++) look[k] = lookat[k] - eye[k];
  cam_cross(look, up, u);
  cam_norm(u);
  cam_cross(look, u, v);
  cam_norm(v);
  cam_norm(look);
  if (ortho) {
    for (int k = 0; k < 3; k++) {
      u[k] = u[k] / (float)width;
      v[k] = v[k] / (float)height;
    }
    for (int k = 0; k < 3; k++) corner[k] = -(u[k] * (float)width + v[k] * (float)height);
    for (int k = 0; k < 3; k++) {
      u[k] = 2.0f * u[k];
      v[k] = 2.0f * v[k];
    }
  } else {
    const float flen =
        (float)(0.5f * (float)height / tan(0.5 * ((double)fov * 3.14159265358979323846 / 180.0)));
    for (int k = 0; k < 3; k++) look[k] = look[k] * flen + eye[k];
    for (int k = 0; k < 3; k++) {
      const float s = u[k] * (float)width + v[k] * (float)height;
      corner[k] = look[k] - s * 0.5f;
    }
  }
  for (int k = 0; k < 3; k++) {
    out[k] = corner[k];
    out[3 + k] = u[k];
    out[6 + k] = v[k];
  }
}

/* Viewport conversion of loop pixel x (axis 0) or y (axis 1). */
static int cam_viewport(int x, int axis, int size, int vp_off, int vp_size) {
  const float inv = 1.0f / (float)size;
  const float x01 = ((float)x + 0.5f) * inv;
  const float nd = 2.0f * (x01 - 0.5f);
  const float w = (nd + 1.0f) * (0.5f * (float)vp_size);
  return axis == 0 ? (int)(w - (float)vp_off) : (int)(w + (float)vp_off);
}

/* cam: eye[3], lookat[3], up[3], fov; ints: ortho, width, height, vx, vy,
 * vw, vh, x0, y0, x1, y1, step.  Writes the rays (row-major over the loop
 * pixels whose converted pixel is on screen) and each ray's loop pixel
 * (y << 16 | x); returns the count. */
SO_API size_t so_camera_rays(const float cam[10], const int ints[12], so_ray *rays,
                             uint32_t *pixel) {
  const int ortho = ints[0], W = ints[1], H = ints[2], vx = ints[3], vy = ints[4],
            vw = ints[5], vh = ints[6], x0 = ints[7], y0 = ints[8], x1 = ints[9],
            y1 = ints[10], step = ints[11];
  float fr[9];
  so_camera_frame(cam, cam + 3, cam + 6, cam[9], ortho, W, H, fr);
  const float *corner = fr, *ud = fr + 3, *vd = fr + 6;
  float look[3];
  cam_cross(ud, vd, look);
  cam_norm(look);
  /* kept loop pixels per axis (the conversion is separable), then one ray
   * per kept (y, x) in row-major order, rows in parallel */
  int nx = 0, ny = 0;
  for (int x = x0; x < x1; x += step) {
    const int px = cam_viewport(x, 0, W, vx, vw);
    if (px >= 0 && px < W) nx++;
  }
  for (int y = y0; y < y1; y += step) {
    const int py = cam_viewport(y, 1, H, vy, vh);
    if (py >= 0 && py < H) ny++;
  }
  int *xs = (int *)malloc(sizeof(int) * (size_t)(nx > 0 ? nx : 1));
  int *ys = (int *)malloc(sizeof(int) * (size_t)(ny > 0 ? ny : 1));
  nx = ny = 0;
  for (int x = x0; x < x1; x += step) {
    const int px = cam_viewport(x, 0, W, vx, vw);
    if (px >= 0 && px < W) xs[nx++] = x;
  }
  for (int y = y0; y < y1; y += step) {
    const int py = cam_viewport(y, 1, H, vy, vh);
    if (py >= 0 && py < H) ys[ny++] = y;
  }
#pragma omp parallel for schedule(static)
  for (int j = 0; j < ny; j++) {
    const int y = ys[j];
    const int py = cam_viewport(y, 1, H, vy, vh);
    for (int i = 0; i < nx; i++) {
      const int x = xs[i];
      const int px = cam_viewport(x, 0, W, vx, vw);
      const float a = ((float)px + 0.0f) + (float)step / 2.0f;
      const float b = (((float)py + 0.0f) - (float)step / 2.0f) + 1.0f;
      float o[3], d[3];
      for (int k = 0; k < 3; k++) {
        const float p = (corner[k] + ud[k] * a) + vd[k] * b;
        if (ortho) {
          o[k] = p;
          d[k] = look[k];
        } else {
          o[k] = cam[k];
          d[k] = p - cam[k];
        }
      }
      cam_norm(d);
      const size_t n = (size_t)j * nx + i;
      so_ray *r = &rays[n];
      for (int k = 0; k < 3; k++) {
        r->org[k] = o[k];
        r->dir[k] = d[k];
      }
      r->prev_prim = 0xffffffffu;
      r->prev_t = 0.0f;
      pixel[n] = ((uint32_t)y << 16) | (uint32_t)x;
    }
  }
  free(xs);
  free(ys);
  return (size_t)nx * ny;
}

static unsigned char fb_clamp(float f) {
  const double d = (double)f * 255.0;
  int i = (d >= -2147483648.0 && d < 2147483648.0) ? (int)d : INT32_MIN; /* x86 cvttsd2si */
  if (i < 0) i = 0;
  if (i > 255) i = 255;
  return (unsigned char)i;
}

/* format 0: RGBA8, 1: RGBA32F.  rgba: per-ray colour or NULL (1,1,1,1). */
SO_API void so_framebuffer_write(int width, int height, int step, const so_hit *hits,
                                 const uint32_t *pixel, const float *rgba, size_t n,
                                 int format, void *color, float *depth) {
#pragma omp parallel for schedule(static)
  for (long ii = 0; ii < (long)n; ii++) {
    const size_t i = (size_t)ii;
    if (hits[i].prim == 0xffffffffu) continue;
    const int x = (int)(pixel[i] & 0xffffu), y = (int)(pixel[i] >> 16);
    float c[4] = {1.0f, 1.0f, 1.0f, 1.0f};
    if (rgba)
      for (int k = 0; k < 4; k++) c[k] = rgba[4 * i + k];
    for (int vv = 0; vv < step; vv++) {
      const int row = height - y - 1 + vv;
      if (row > height - 1 || row < 0) continue;
      for (int uu = 0; uu < step; uu++) {
        const int col = x + uu;
        if (col > width - 1) continue;
        const size_t p = (size_t)row * width + col;
        if (color && format == 0) {
          unsigned char *o = (unsigned char *)color + 4 * p;
          for (int k = 0; k < 4; k++) o[k] = fb_clamp(c[k] * 1.0f);
        } else if (color) {
          float *o = (float *)color + 4 * p;
          for (int k = 0; k < 4; k++) o[k] = c[k] * 1.0f;
        }
        if (depth) depth[p] = hits[i].t * 1.0f;
      }
    }
  }
}

/* ---- several samples per pixel and the stereo environment camera
 * OnData with sampleCoverage (gles/gles_raytrace_engine.cc:549-553,
 * 747-800): per loop pixel subSamples^2 rays, (vv, uu) row-major, at
 * u = (uu + ju) / S, v = (vv + jv) / S where ju (uu != 0) and then jv
 * (vv != 0) are draws of randomreal: (float) of TinyMT64's double, the
 * serial renderer's single stream seeded 1234 with gles_common.cc's
 * parameters (initialize_random, :260-280), consumed in pixel order (rows,
 * then x) over the kept pixels -- `offset` draws already consumed.  The
 * write averages each pixel's hits: colour sum * (1 / S^2), depth sum *
 * (1 / S^2), for pixels with at least one hit (:826-877). */

/* Camera::generateStereoEnvRay (render/render_camera.cc:65-118) for the
 * stereo camera of render/render_camera.h:44-60 (m_uvw = (normalize(up x
 * look), normalize(look x u), normalize(look))). */
SO_API void so_stereo_env_ray(const float eye[3], const float lookat[3], const float up[3],
                              float zero_parallax, float eye_sep, float image_u, float image_v,
                              int width, int height, float org[3], float dir[3]) {
  float look[3], u[3], v[3];
  for (int k = 0; k < 3; k++) look[k] = lookat[k] - eye[k];
  cam_cross(up, look, u);
  cam_norm(u);
  cam_cross(look, u, v);
  cam_norm(v);
  cam_norm(look);
  const int is_left = image_v < (float)(height / 2);
  const float focal = zero_parallax, r = eye_sep;
  const float theta = (float)(M_PI * fmod(2.0 * image_v / height, 1.0));
  const float phi = (float)(2.0 * M_PI * (image_u / (float)width));
  float dir_o[3];
  dir_o[0] = sinf(theta) * cosf(phi);
  dir_o[1] = cosf(theta);
  dir_o[2] = sinf(theta) * sinf(phi);
  float par[3];
  if (is_left) {
    par[0] = -dir_o[2];
    par[1] = 0.0f;
    par[2] = dir_o[0];
  } else {
    par[0] = dir_o[2];
    par[1] = 0.0f;
    par[2] = -dir_o[0];
  }
  cam_norm(par);
  for (int k = 0; k < 3; k++) par[k] = par[k] * r;
  for (int k = 0; k < 3; k++) org[k] = eye[k] + par[k];
  float psi = (float)atan2((double)r, (double)focal);
  if (is_left) psi = -psi;
  float d[3];
  d[0] = (float)(dir_o[0] * cos((double)psi) - dir_o[2] * sin((double)psi));
  d[1] = dir_o[1];
  d[2] = (float)(dir_o[0] * sin((double)psi) + dir_o[2] * cos((double)psi));
  for (int k = 0; k < 3; k++) dir[k] = u[k] * d[0] + v[k] * d[1] + look[k] * d[2];
}

/* cam, ints as so_camera_rays; smp_i: subsamples, stereo; smp_f: zero
 * parallax, eye separation.  Rays: per kept loop pixel (rows, then x) its
 * S^2 rays; pixel: each ray's loop pixel.  Returns the ray count. */
SO_API size_t so_camera_rays_ex(const float cam[10], const int ints[12], const int smp_i[2],
                                const float smp_f[2], uint64_t seed, uint64_t offset,
                                so_ray *rays, uint32_t *pixel) {
  const int ortho = ints[0], W = ints[1], H = ints[2], vx = ints[3], vy = ints[4],
            vw = ints[5], vh = ints[6], x0 = ints[7], y0 = ints[8], x1 = ints[9],
            y1 = ints[10], step = ints[11];
  const int S = smp_i[0], stereo = smp_i[1];
  float fr[9];
  so_camera_frame(cam, cam + 3, cam + 6, cam[9], ortho, W, H, fr);
  const float *corner = fr, *ud = fr + 3, *vd = fr + 6;
  float look[3];
  cam_cross(ud, vd, look);
  cam_norm(look);
  so_tinymt64 rng;
  rng.mat1 = 0xfa051f40u;
  rng.mat2 = 0xffd0fff4u;
  rng.tmat = UINT64_C(0x58d02ffeffbfffbc);
  tmt_seed(&rng, seed);
  for (uint64_t i = 0; i < offset; i++) tmt_step(&rng);
  size_t n = 0;
  for (int y = y0; y < y1; y += step) {
    const int py = cam_viewport(y, 1, H, vy, vh);
    if (py < 0 || py >= H) continue;
    for (int x = x0; x < x1; x += step) {
      const int px = cam_viewport(x, 0, W, vx, vw);
      if (px < 0 || px >= W) continue;
      for (int vv = 0; vv < S; vv++)
        for (int uu = 0; uu < S; uu++) {
          float ju = 0.0f, jv = 0.0f;
          if (uu != 0) {
            tmt_step(&rng);
            ju = (float)((double)tmt_out(&rng) * (1.0 / 18446744073709551616.0));
          }
          if (vv != 0) {
            tmt_step(&rng);
            jv = (float)((double)tmt_out(&rng) * (1.0 / 18446744073709551616.0));
          }
          const float su = ((float)uu + ju) / (float)S, sv = ((float)vv + jv) / (float)S;
          const float a = ((float)px + su) + (float)step / 2.0f;
          const float b = (((float)py + sv) - (float)step / 2.0f) + 1.0f;
          float o[3], d[3];
          if (stereo) {
            so_stereo_env_ray(cam, cam + 3, cam + 6, smp_f[0], smp_f[1], a, b, W, H, o, d);
          } else {
            for (int k = 0; k < 3; k++) {
              const float p = (corner[k] + ud[k] * a) + vd[k] * b;
              if (ortho) {
                o[k] = p;
                d[k] = look[k];
              } else {
                o[k] = cam[k];
                d[k] = p - cam[k];
              }
            }
          }
          cam_norm(d);
          so_ray *r = &rays[n];
          for (int k = 0; k < 3; k++) {
            r->org[k] = o[k];
            r->dir[k] = d[k];
          }
          r->prev_prim = 0xffffffffu;
          r->prev_t = 0.0f;
          pixel[n] = ((uint32_t)y << 16) | (uint32_t)x;
          n++;
        }
    }
  }
  return n;
}

/* The write of n rays made S^2 per loop pixel by so_camera_rays_ex. */
SO_API void so_framebuffer_write_ex(int width, int height, int step, int S, const so_hit *hits,
                                    const uint32_t *pixel, const float *rgba, size_t n,
                                    int format, void *color, float *depth) {
  const size_t per = (size_t)S * S;
  const float inv_n = 1.0f / (float)(S * S);
  for (size_t g = 0; g + per <= n; g += per) {
    float fc[4] = {0.0f, 0.0f, 0.0f, 0.0f}, dv = 0.0f;
    int frag = 0;
    for (size_t q = g; q < g + per; q++) {
      if (hits[q].prim == 0xffffffffu) continue;
      for (int k = 0; k < 4; k++) fc[k] += rgba ? rgba[4 * q + k] : 1.0f;
      dv += hits[q].t;
      frag = 1;
    }
    if (!frag) continue;
    dv *= inv_n;
    const int x = (int)(pixel[g] & 0xffffu), y = (int)(pixel[g] >> 16);
    for (int vv = 0; vv < step; vv++) {
      const int row = height - y - 1 + vv;
      if (row > height - 1 || row < 0) continue;
      for (int uu = 0; uu < step; uu++) {
        const int col = x + uu;
        if (col > width - 1) continue;
        const size_t p = (size_t)row * width + col;
        if (color && format == 0) {
          unsigned char *o = (unsigned char *)color + 4 * p;
          for (int k = 0; k < 4; k++) o[k] = fb_clamp(fc[k] * inv_n);
        } else if (color) {
          float *o = (float *)color + 4 * p;
          for (int k = 0; k < 4; k++) o[k] = fc[k] * inv_n;
        }
        if (depth) depth[p] = dv;
      }
    }
  }
}

/* ======================================================== scenes
 * RenderGraph::Build / Trace (gles/gles_render_graph.cc:104-314) over
 * elements = (accel, T, invT, invT33, world box), restated:
 *   - BVHTree::BuildTree / ConstructTree (render/render_bvh_tree.cc:319-500):
 *     spatial median on the longest axis (axis retries in the order
 *     {0,1,2},{1,2,0},{2,0,1}), PartitionNodes' in-place swap order
 *     (:83-130), object median fallback, child boxes widened by 1e-6 of their
 *     extent, root = the unwidened scene box;
 *   - BVHTree::Trace (:504-585): SetupRay's reciprocals (|d| <= 2e-15 gives
 *     +-FLT_MAX), TestRayAABB in double, leaves tested with their own box,
 *     near child by ray sign first, candidates sorted by entry distance
 *     (std::sort: insertion sort, stable, for up to 16 candidates);
 *   - per candidate: skipped when beyond the nearest world hit so far;
 *     local ray by Matrixd::MultV with invT / invT33 (double) stored as
 *     float; the element's reference walk; world point by MultV with T of
 *     the float local point; world distance = float length; strictly nearer
 *     wins.  prev_prim / prev_t / prev_normal apply only in prev_element.
 * so_scene_trace walks each element with the reference's walk, or with
 * walk2 with the two-pass walk restated (the same hits); visits (optional)
 * receives per ray the node and primitive visits of its element walks. */
typedef struct {
  double bmin[3], bmax[3];
  int child[2], axis, leaf;
  uint32_t id;
} so_top;

typedef struct {
  double bmin[3], bmax[3];
  uint32_t id;
} so_topdata;

typedef struct {
  size_t n, nn, cap;
  const so_accel **acc; /* per element: so_accel, or so_lines / so_solids (kind) */
  int *kind;            /* 0: so_accel; 3: so_lines; 4: so_solids */
  double *T, *invT, *invT33;
  so_top *nodes;
} so_scene;

/* The closest hit of a local ray in a line (kind 3) or solid (kind 4)
 * element: LineAccel::Traverse / SolidAccel::Traverse, defined with them
 * below. */
static void scene_other_trace(int kind, const void *obj, const so_ray *lr, so_hit *h);

static size_t top_partition(so_topdata *d, size_t l, size_t r, double pos, int axis) {
  so_topdata leftmost = d[l];
  size_t pivot = l;
  for (size_t i = l + 1; i < r; i++) {
    if (d[i].bmax[axis] < pos) {
      pivot++;
      so_topdata t = d[pivot];
      d[pivot] = d[i];
      d[i] = t;
    }
  }
  d[l] = d[pivot];
  d[pivot] = leftmost;
  size_t split = l;
  for (size_t i = l; i < r; i++)
    if (d[i].bmax[axis] < pos) split++;
  return split;
}

static void top_box(const so_topdata *d, size_t s, size_t e, double bmin[3], double bmax[3]) {
  for (int k = 0; k < 3; k++) {
    bmin[k] = d[s].bmin[k];
    bmax[k] = d[s].bmax[k];
  }
  for (size_t i = s + 1; i < e; i++)
    for (int k = 0; k < 3; k++) {
      if (d[i].bmin[k] < bmin[k]) bmin[k] = d[i].bmin[k];
      if (bmax[k] < d[i].bmax[k]) bmax[k] = d[i].bmax[k];
    }
}

static size_t top_push(so_scene *s, const double bmin[3], const double bmax[3]) {
  if (s->nn == s->cap) {
    s->cap = s->cap ? 2 * s->cap : 16;
    s->nodes = (so_top *)realloc(s->nodes, s->cap * sizeof(so_top));
  }
  so_top *t = &s->nodes[s->nn];
  memset(t, 0, sizeof(*t));
  for (int k = 0; k < 3; k++) {
    t->bmin[k] = bmin[k];
    t->bmax[k] = bmax[k];
  }
  return s->nn++;
}

static void top_construct(so_scene *s, so_topdata *d, size_t root, size_t l, size_t r) {
  static const int axl[3][3] = {{0, 1, 2}, {1, 2, 0}, {2, 0, 1}};
  const size_t n = r - l;
  if (n == 1) {
    s->nodes[root].leaf = 1;
    s->nodes[root].child[0] = s->nodes[root].child[1] = 0;
    s->nodes[root].id = d[l].id;
    return;
  }
  double bsize[3], bmin[3];
  for (int k = 0; k < 3; k++) {
    bsize[k] = s->nodes[root].bmax[k] - s->nodes[root].bmin[k];
    bmin[k] = s->nodes[root].bmin[k];
  }
  double maxlen = bsize[0];
  int at = 0;
  if (maxlen < bsize[1]) {
    maxlen = bsize[1];
    at = 1;
  }
  if (maxlen < bsize[2]) {
    maxlen = bsize[2];
    at = 2;
  }
  size_t split = l, nl = 0, nr = n;
  int axis = 0;
  for (int i = 0; i < 3; i++) {
    axis = axl[at][i];
    split = top_partition(d, l, r, bmin[axis] + bsize[axis] * 0.5, axis);
    if (split != l && split != r) {
      nl = split - l;
      nr = n - nl;
      break;
    }
  }
  if (split == l || split == r) {
    nl = n / 2;
    nr = n - nl;
    split = l + (r - l) / 2;
  }
  s->nodes[root].axis = axis;
  s->nodes[root].leaf = 0;
  for (int side = 0; side < 2; side++) {
    const size_t cnt = side ? nr : nl;
    if (!cnt) {
      s->nodes[root].child[side] = 0;
      continue;
    }
    const size_t a = side ? split : l, b = side ? r : split;
    double cb[3], ce[3];
    top_box(d, a, b, cb, ce);
    for (int k = 0; k < 3; k++) {
      double ext = ce[k] - cb[k];
      cb[k] = cb[k] - ext * 1.0e-6;
      ce[k] = ce[k] + ext * 1.0e-6;
    }
    size_t child = top_push(s, cb, ce);
    s->nodes[root].child[side] = (int)child;
    top_construct(s, d, child, a, b);
  }
}

SO_API so_scene *so_scene_build(const so_accel *const *acc, const double *T,
                                const double *invT, const double *invT33, const double *bmin,
                                const double *bmax, size_t n) {
  so_scene *s = (so_scene *)calloc(1, sizeof(so_scene));
  s->n = n;
  s->acc = (const so_accel **)malloc(n * sizeof(*s->acc));
  s->T = (double *)malloc(n * 16 * sizeof(double));
  s->invT = (double *)malloc(n * 16 * sizeof(double));
  s->invT33 = (double *)malloc(n * 16 * sizeof(double));
  s->kind = (int *)calloc(n ? n : 1, sizeof(int));
  memcpy(s->acc, acc, n * sizeof(*s->acc));
  memcpy(s->T, T, n * 16 * sizeof(double));
  memcpy(s->invT, invT, n * 16 * sizeof(double));
  memcpy(s->invT33, invT33, n * 16 * sizeof(double));
  so_topdata *d = (so_topdata *)malloc(n * sizeof(so_topdata));
  for (size_t i = 0; i < n; i++) {
    for (int k = 0; k < 3; k++) {
      d[i].bmin[k] = bmin[3 * i + k];
      d[i].bmax[k] = bmax[3 * i + k];
    }
    d[i].id = (uint32_t)i;
  }
  double sb[3], se[3];
  top_box(d, 0, n, sb, se);
  top_push(s, sb, se);
  top_construct(s, d, 0, 0, n);
  free(d);
  return s;
}

/* Element e is a line (3) or solid (4) accel: acc[e] holds an so_lines /
 * so_solids (RenderGraph::Trace's PRIMITIVE_LINES and solid cases,
 * gles/gles_render_graph.cc:239-260). */
SO_API void so_scene_set_kind(so_scene *s, size_t e, int kind) {
  if (s && e < s->n) s->kind[e] = kind;
}

SO_API void so_scene_free(so_scene *s) {
  if (!s) return;
  free(s->kind);
  free(s->acc);
  free(s->T);
  free(s->invT);
  free(s->invT33);
  free(s->nodes);
  free(s);
}

SO_API size_t so_scene_top_nodes(const so_scene *s, double *boxes, int32_t *ints, size_t cap) {
  for (size_t i = 0; i < s->nn && i < cap; i++) {
    for (int k = 0; k < 3; k++) {
      boxes[6 * i + k] = s->nodes[i].bmin[k];
      boxes[6 * i + 3 + k] = s->nodes[i].bmax[k];
    }
    ints[5 * i + 0] = s->nodes[i].child[0];
    ints[5 * i + 1] = s->nodes[i].child[1];
    ints[5 * i + 2] = s->nodes[i].axis;
    ints[5 * i + 3] = s->nodes[i].leaf;
    ints[5 * i + 4] = (int32_t)s->nodes[i].id;
  }
  return s->nn;
}

static int top_aabb(const so_top *t, const double o[3], const double inv[3], const int sgn[3],
                    double *tmin, double *tmax) {
  double mn[3], mx[3];
  for (int k = 0; k < 3; k++) {
    mn[k] = sgn[k] ? t->bmax[k] : t->bmin[k];
    mx[k] = sgn[k] ? t->bmin[k] : t->bmax[k];
  }
  const double tminx = (mn[0] - o[0]) * inv[0], tmaxx = (mx[0] - o[0]) * inv[0];
  const double tminy = (mn[1] - o[1]) * inv[1], tmaxy = (mx[1] - o[1]) * inv[1];
  double a = (tminx > tminy) ? tminx : tminy;
  double b = (tmaxx < tmaxy) ? tmaxx : tmaxy;
  const double tminz = (mn[2] - o[2]) * inv[2], tmaxz = (mx[2] - o[2]) * inv[2];
  a = (a > tminz) ? a : tminz;
  b = (b < tmaxz) ? b : tmaxz;
  if ((b > 0.0) && (a <= b)) {
    *tmin = a;
    *tmax = b;
    return 1;
  }
  return 0;
}

/* candidates of one ray in sorted order; returns their number */
SO_API size_t so_scene_candidates(const so_scene *s, const double o[3], const double dir[3],
                                  double *ct, uint32_t *cid, size_t cap) {
  int sgn[3];
  double inv[3];
  for (int k = 0; k < 3; k++) {
    sgn[k] = dir[k] < 0.0 ? 1 : 0;
    inv[k] = fabs(dir[k]) > 2.0e-15 ? 1.0 / dir[k] : (dir[k] < 0.0 ? -FLT_MAX : FLT_MAX);
  }
  size_t nc = 0;
  int stk[256], sp = 0, node = 0;
  for (;;) {
    const so_top *t = &s->nodes[node];
    if (t->leaf) {
      double a, b;
      if (top_aabb(t, o, inv, sgn, &a, &b) && nc < cap) {
        ct[nc] = a;
        cid[nc] = t->id;
        nc++;
      }
      if (sp < 1) break;
      node = stk[--sp];
    } else {
      double a0 = 0, b0 = 0, a1 = 0, b1 = 0;
      int h0 = t->child[0] > 0 && top_aabb(&s->nodes[t->child[0]], o, inv, sgn, &a0, &b0);
      int h1 = t->child[1] > 0 && top_aabb(&s->nodes[t->child[1]], o, inv, sgn, &a1, &b1);
      if (!h0 && !h1) {
        if (sp < 1) break;
        node = stk[--sp];
      } else if (h0 && !h1) {
        node = t->child[0];
      } else if (h1 && !h0) {
        node = t->child[1];
      } else {
        int order = sgn[t->axis];
        stk[sp++] = t->child[1 - order];
        node = t->child[order];
      }
    }
  }
  for (size_t a = 1; a < nc; a++) { /* stable insertion sort */
    double kt = ct[a];
    uint32_t kid = cid[a];
    size_t b = a;
    while (b > 0 && kt < ct[b - 1]) {
      ct[b] = ct[b - 1];
      cid[b] = cid[b - 1];
      b--;
    }
    ct[b] = kt;
    cid[b] = kid;
  }
  return nc;
}

static void scene_multv(const double *m, const double v[3], double o[3]) {
  for (int k = 0; k < 3; k++) o[k] = ((m[k] * v[0] + m[4 + k] * v[1]) + m[8 + k] * v[2]) + m[12 + k];
}

SO_API void so_scene_trace(const so_scene *s, const so_ray *rays, size_t n,
                           const uint32_t *prev_element, const float *prev_normals,
                           so_hit *hits, uint32_t *element, uint32_t *visits, int walk2,
                           int nthreads) {
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 64)
#endif
  for (long ii = 0; ii < (long)n; ii++) {
    const size_t i = (size_t)ii;
    const so_ray *r = &rays[i];
    const double ro[3] = {r->org[0], r->org[1], r->org[2]};
    const double rd[3] = {r->dir[0], r->dir[1], r->dir[2]};
    double ct[64];
    uint32_t cid[64];
    size_t nc = so_scene_candidates(s, ro, rd, ct, cid, 64);
    double tnear = DBL_MAX;
    uint64_t nvis = 0;
    so_hit best = {FLT_MAX, 0.0f, 0.0f, 0xffffffffu};
    uint32_t be = 0xffffffffu;
    for (size_t c = 0; c < nc; c++) {
      if (tnear < ct[c]) continue;
      const uint32_t e = cid[c];
      double lo[3], ld[3];
      scene_multv(&s->invT[16 * e], ro, lo);
      scene_multv(&s->invT33[16 * e], rd, ld);
      const int same = prev_element && prev_element[i] == e;
      so_ray lr;
      for (int k = 0; k < 3; k++) {
        lr.org[k] = (float)lo[k];
        lr.dir[k] = (float)ld[k];
      }
      lr.prev_prim = same ? r->prev_prim : 0xffffffffu;
      lr.prev_t = same ? r->prev_t : 0.0f;
      float zero3[3] = {0, 0, 0};
      const float *pn = (same && prev_normals) ? &prev_normals[3 * i] : zero3;
      so_hit h;
      so_stats st = {0, 0, 0};
      if (s->kind[e] != 0) {
        scene_other_trace(s->kind[e], s->acc[e], &lr, &h);
      } else if (walk2) {
        int fall = 0;
        trace2_one(s->acc[e], &lr, pn, &h, NULL, NULL, NULL, &st, &fall);
      } else {
        trace_one(s->acc[e], &lr, pn, &h, NULL, NULL, NULL, &st);
      }
      nvis += st.branch_visits + st.prim_tests;
      if (h.prim == 0xffffffffu || !(h.t < FLT_MAX)) continue;
      if (s->kind[e] == 0) sphere_finish(s->acc[e], &lr, &h); /* the element's Traverse */
      double lp[3], wp[3];
      for (int k = 0; k < 3; k++) lp[k] = (double)(float)(lo[k] + (double)h.t * ld[k]);
      scene_multv(&s->T[16 * e], lp, wp);
      float po[3];
      for (int k = 0; k < 3; k++) po[k] = (float)wp[k] - r->org[k];
      const float tw = sqrtf(po[0] * po[0] + po[1] * po[1] + po[2] * po[2]);
      if ((double)tw < tnear) {
        tnear = tw;
        best = h;
        best.t = tw;
        be = e;
      }
    }
    hits[i] = best;
    if (element) element[i] = be;
    if (visits) visits[i] = (uint32_t)(nvis < 0xffffffffu ? nvis : 0xffffffffu);
  }
}

/* Matrixd::Inverse (render/render_matrix.h:40-134), written out entry by
 * entry in the routine's operation order (s = m transposed; the m[3][3]
 * entry keeps the reference's s[0] factor). */
SO_API void so_matrix_inverse(double m[16]) {
  double s[16], p[12];
  for (int r = 0; r < 4; r++)
    for (int c = 0; c < 4; c++) s[4 * c + r] = m[4 * r + c];
#define PAIRS(o)                                                               \
  p[0] = s[10 - o] * s[15 - o]; p[1] = s[11 - o] * s[14 - o];                  \
  p[2] = s[9 - o] * s[15 - o];  p[3] = s[11 - o] * s[13 - o];                  \
  p[4] = s[9 - o] * s[14 - o];  p[5] = s[10 - o] * s[13 - o];                  \
  p[6] = s[8 - o] * s[15 - o];  p[7] = s[11 - o] * s[12 - o];                  \
  p[8] = s[8 - o] * s[14 - o];  p[9] = s[10 - o] * s[12 - o];                  \
  p[10] = s[8 - o] * s[13 - o]; p[11] = s[9 - o] * s[12 - o];
#define E(e, a0, b0, a1, b1, a2, b2, c0, d0, c1, d1, c2, d2)                   \
  m[e] = p[a0] * s[b0] + p[a1] * s[b1] + p[a2] * s[b2];                        \
  m[e] -= p[c0] * s[d0] + p[c1] * s[d1] + p[c2] * s[d2];
  PAIRS(0)
  E(0, 0, 5, 3, 6, 4, 7, 1, 5, 2, 6, 5, 7)
  E(1, 1, 4, 6, 6, 9, 7, 0, 4, 7, 6, 8, 7)
  E(2, 2, 4, 7, 5, 10, 7, 3, 4, 6, 5, 11, 7)
  E(3, 5, 4, 8, 5, 11, 6, 4, 4, 9, 5, 10, 6)
  E(4, 1, 1, 2, 2, 5, 3, 0, 1, 3, 2, 4, 3)
  E(5, 0, 0, 7, 2, 8, 3, 1, 0, 6, 2, 9, 3)
  E(6, 3, 0, 6, 1, 11, 3, 2, 0, 7, 1, 10, 3)
  E(7, 4, 0, 9, 1, 10, 2, 5, 0, 8, 1, 11, 2)
  PAIRS(8)
  E(8, 0, 13, 3, 14, 4, 15, 1, 13, 2, 14, 5, 15)
  E(9, 1, 12, 6, 14, 9, 15, 0, 12, 7, 14, 8, 15)
  E(10, 2, 12, 7, 13, 10, 15, 3, 12, 6, 13, 11, 15)
  E(11, 5, 12, 8, 13, 11, 14, 4, 12, 9, 13, 10, 14)
  E(12, 2, 10, 5, 11, 1, 9, 4, 11, 0, 9, 3, 10)
  E(13, 8, 11, 0, 8, 7, 10, 6, 10, 9, 11, 1, 8)
  E(14, 6, 9, 11, 11, 3, 8, 10, 11, 2, 8, 7, 9)
  E(15, 10, 10, 4, 8, 9, 9, 8, 9, 11, 0, 5, 8)
#undef E
#undef PAIRS
  double det = s[0] * m[0] + s[1] * m[1] + s[2] * m[2] + s[3] * m[3];
  det = 1.0 / det;
  for (int e = 0; e < 16; e++) m[e] *= det;
}

/* RenderElement::Update (gles/gles_render_graph.cc:17-101): world box of
 * the local box's corners (corner order of TransformBoundingBox), invT,
 * invT33 (T without translation, inverted). */
SO_API void so_element_update(const double T[16], const double lbmin[3], const double lbmax[3],
                              double invT[16], double invT33[16], double wbmin[3],
                              double wbmax[3]) {
  for (int c = 0; c < 8; c++) {
    double v[3], x[3];
    v[0] = (c & 1) ? lbmax[0] : lbmin[0];
    v[1] = (c & 2) ? lbmax[1] : lbmin[1];
    v[2] = (c & 4) ? lbmax[2] : lbmin[2];
    for (int k = 0; k < 3; k++) x[k] = T[k] * v[0] + T[4 + k] * v[1] + T[8 + k] * v[2] + T[12 + k];
    for (int k = 0; k < 3; k++) {
      if (c == 0) {
        wbmin[k] = x[k];
        wbmax[k] = x[k];
      } else {
        if (!(wbmin[k] < x[k])) wbmin[k] = x[k];
        if (!(x[k] < wbmax[k])) wbmax[k] = x[k];
      }
    }
  }
  memcpy(invT, T, 16 * sizeof(double));
  memcpy(invT33, T, 16 * sizeof(double));
  so_matrix_inverse(invT);
  invT33[12] = invT33[13] = invT33[14] = 0.0;
  so_matrix_inverse(invT33);
}

/* ======================================================= texture fetch
 * Texture::Fetch for 3D textures (gles/gles_common.h:344-399), restated:
 *   dense: per-axis remap (local::remap, gles/gles_common.h:264-269: idx =
 *   (int)(x * n) clamped to [0, n-1], table[idx]) then FilterTexture3D{Byte,
 *   Float,Double} (render/render_texture.cc:832-1175): wrap by fasterfloorf
 *   unless clamp-to-edge, vox = u * (dim - 1), texel-corner trilinear with
 *   Lerp (float; dlerp for doubles), bytes read as v / 255.5f, one component
 *   replicated to rgba;
 *   sparse: position = u * globalDim, the first block the BVHTree's Locate
 *   (render/render_bvh_tree.cc:587-655) reaches, then
 *   SparseVolumeAccel::Sample (render/render_accel_volume.cc:61-139): the
 *   nearest texel (local offset times size/extent of x for all three axes),
 *   bytes as v / 255.0f, doubles through float, alpha 1 when fewer than four
 *   components, (0,0,0,0) outside every block.
 * Formats: 0 byte, 1 float, 2 double (LSGL_RENDER_TEXTURE3D_FORMAT_*). */

static double texel_d(int fmt, const void *img, size_t k) {
  if (fmt == 0) return (double)(((const unsigned char *)img)[k] / 255.5f);
  if (fmt == 1) return (double)((const float *)img)[k];
  return ((const double *)img)[k];
}

SO_API void so_tex_fetch(int fmt, const void *img, const int dim[3], int comps,
                         const int clamp[3], const float *const remap[3], const int nremap[3],
                         const float *uvw, size_t n, float *rgba) {
  for (size_t i = 0; i < n; i++) {
    float c[3];
    for (int k = 0; k < 3; k++) {
      c[k] = uvw[3 * i + k];
      if (remap[k] && nremap[k] > 0) c[k] = remap_ref(c[k], remap[k], nremap[k]);
      if (!clamp[k]) c[k] = c[k] - floor_ref(c[k]);
    }
    float vox[3];
    int v0[3], v1[3];
    for (int k = 0; k < 3; k++) {
      vox[k] = c[k] * (dim[k] - 1.0f);
      v0[k] = clampi((int)vox[k], 0, dim[k] - 1);
      v1[k] = v0[k] + 1 < dim[k] - 1 ? v0[k] + 1 : dim[k] - 1;
    }
    float vals[4] = {0, 0, 0, 0};
    for (int ch = 0; ch < comps && ch < 4; ch++) {
#define T(x, y, z)                                                                          \
  texel_d(fmt, img,                                                                         \
          (size_t)comps * ((size_t)(z) * dim[0] * dim[1] + (size_t)(y) * dim[0] + (x)) + ch)
      if (fmt == 2) {
        const double dx = vox[0] - v0[0], dy = vox[1] - v0[1], dz = vox[2] - v0[2];
#define DL(t, a, b) ((1.0 - (t)) * (a) + (t) * (b))
        double d00 = DL(dx, T(v0[0], v0[1], v0[2]), T(v1[0], v0[1], v0[2]));
        double d10 = DL(dx, T(v0[0], v1[1], v0[2]), T(v1[0], v1[1], v0[2]));
        double d01 = DL(dx, T(v0[0], v0[1], v1[2]), T(v1[0], v0[1], v1[2]));
        double d11 = DL(dx, T(v0[0], v1[1], v1[2]), T(v1[0], v1[1], v1[2]));
        double d0 = DL(dy, d00, d10), d1 = DL(dy, d01, d11);
        vals[ch] = (float)DL(dz, d0, d1);
#undef DL
      } else {
        const float dx = vox[0] - v0[0], dy = vox[1] - v0[1], dz = vox[2] - v0[2];
        float d00 = lerpf(dx, (float)T(v0[0], v0[1], v0[2]), (float)T(v1[0], v0[1], v0[2]));
        float d10 = lerpf(dx, (float)T(v0[0], v1[1], v0[2]), (float)T(v1[0], v1[1], v0[2]));
        float d01 = lerpf(dx, (float)T(v0[0], v0[1], v1[2]), (float)T(v1[0], v0[1], v1[2]));
        float d11 = lerpf(dx, (float)T(v0[0], v1[1], v1[2]), (float)T(v1[0], v1[1], v1[2]));
        float d0 = lerpf(dy, d00, d10), d1 = lerpf(dy, d01, d11);
        vals[ch] = lerpf(dz, d0, d1);
      }
#undef T
    }
    float *o = &rgba[4 * i];
    if (comps == 1) {
      o[0] = o[1] = o[2] = o[3] = vals[0];
    } else {
      o[0] = vals[0]; o[1] = vals[1]; o[2] = vals[2]; o[3] = vals[3];
    }
  }
}

typedef struct {
  int offset[3], extent[3], size[3], level;
  uint64_t data_offset; /* bytes into the data pool */
} so_block;

/* BVHTree::Locate: the first leaf (depth first, left child first) whose box
 * holds p (inclusive); -1 if none. */
static int top_locate(const so_scene *s, const double p[3]) {
  int stk[256], sp = 0, node = 0;
  for (;;) {
    const so_top *t = &s->nodes[node];
    if (t->leaf) {
      if (p[0] >= t->bmin[0] && p[0] <= t->bmax[0] && p[1] >= t->bmin[1] &&
          p[1] <= t->bmax[1] && p[2] >= t->bmin[2] && p[2] <= t->bmax[2])
        return (int)t->id;
      if (sp < 1) return -1;
      node = stk[--sp];
    } else {
      int h[2];
      for (int c = 0; c < 2; c++) {
        const so_top *u = t->child[c] > 0 ? &s->nodes[t->child[c]] : NULL;
        h[c] = u && p[0] >= u->bmin[0] && p[0] <= u->bmax[0] && p[1] >= u->bmin[1] &&
               p[1] <= u->bmax[1] && p[2] >= u->bmin[2] && p[2] <= u->bmax[2];
      }
      if (!h[0] && !h[1]) {
        if (sp < 1) return -1;
        node = stk[--sp];
      } else if (h[0] && !h[1]) {
        node = t->child[0];
      } else if (h[1] && !h[0]) {
        node = t->child[1];
      } else {
        stk[sp++] = t->child[1];
        node = t->child[0];
      }
    }
  }
}

SO_API so_scene *so_sparse_tree(const so_block *b, size_t n) {
  double *lo = (double *)malloc(n * 3 * sizeof(double));
  double *hi = (double *)malloc(n * 3 * sizeof(double));
  const so_accel **acc = (const so_accel **)calloc(n, sizeof(*acc));
  double *z = (double *)calloc(n * 16, sizeof(double));
  for (size_t i = 0; i < n; i++)
    for (int k = 0; k < 3; k++) {
      lo[3 * i + k] = (double)b[i].offset[k];
      hi[3 * i + k] = (double)(b[i].offset[k] + b[i].extent[k]);
    }
  so_scene *s = so_scene_build(acc, z, z, z, lo, hi, n);
  free(lo);
  free(hi);
  free((void *)acc);
  free(z);
  return s;
}

SO_API void so_sparse_fetch(const so_scene *tree, const so_block *b, const void *pool, int fmt,
                            int comps, const int gdim[3], const float *uvw, size_t n,
                            float *rgba) {
  for (size_t i = 0; i < n; i++) {
    double p[3];
    for (int k = 0; k < 3; k++) p[k] = (double)(uvw[3 * i + k] * gdim[k]);
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    const int id = top_locate(tree, p);
    if (id >= 0) {
      const so_block *bl = &b[id];
      const int nc = comps >= 4 ? 4 : comps;
      v[3] = 1.0;
      double x = p[0] - bl->offset[0], y = p[1] - bl->offset[1], z = p[2] - bl->offset[2];
      const double sx = bl->size[0] / (double)bl->extent[0];
      x = x * sx;
      y = y * sx; /* the reference scales all three axes by x's ratio */
      z = z * sx;
      int ix = (int)x, iy = (int)y, iz = (int)z;
      ix = ix > bl->size[0] - 1 ? bl->size[0] - 1 : ix;
      iy = iy > bl->size[1] - 1 ? bl->size[1] - 1 : iy;
      iz = iz > bl->size[2] - 1 ? bl->size[2] - 1 : iz;
      ix = ix < 0 ? 0 : ix;
      iy = iy < 0 ? 0 : iy;
      iz = iz < 0 ? 0 : iz;
      const size_t idx = (size_t)iz * bl->size[0] * bl->size[1] + (size_t)iy * bl->size[0] + ix;
      const unsigned char *base = (const unsigned char *)pool + bl->data_offset;
      for (int c = 0; c < nc; c++) {
        const size_t k = (size_t)nc * idx + c; /* the stride is the clamped count */
        if (fmt == 0) v[c] = base[k] / 255.0f;
        else if (fmt == 1) v[c] = ((const float *)base)[k];
        else v[c] = (float)((const double *)base)[k];
      }
    }
    for (int k = 0; k < 4; k++) rgba[4 * i + k] = (float)v[k];
  }
}

/* ------------------------------------------------------------------------ */
/* Lines: LineAccel (render/render_accel_line.cc), capped cylinders between  */
/* segment end points, a spatial-median BVH built top-down and a closest-hit */
/* walk that tests each popped branch's own box.  Float throughout, except   */
/* where the reference's unqualified sqrt/fabs resolve to the double C       */
/* functions (the quadratic's first root is formed and divided in double).   */
/* ------------------------------------------------------------------------ */

typedef struct {
  float bmin[3], bmax[3];
  int32_t flag, axis; /* flag 1: leaf (data = count, first); 0: branch (children) */
  uint32_t data[2];
} so_line_node; /* 40 bytes, the reference's LineNode and Dump() record */

typedef struct {
  const float *pos, *radius;
  float constr;
  const uint32_t *seg;
  size_t n;
  int min_leaf, max_depth, cap, depth_seen;
  so_line_node *nodes;
  size_t nnodes, ncap;
  uint32_t *idx;
} so_lines;

static inline float line_r(const so_lines *L, uint32_t v) {
  return L->radius ? L->radius[v] : L->constr;
}

/* GetBoundingBoxOfLine (:83-116): both end points +-r, then widened by
 * FLT_EPSILON * 16 of each coordinate's own magnitude. */
static void line_box(const so_lines *L, uint32_t i, float bmin[3], float bmax[3]) {
  const uint32_t a = L->seg[2 * i], b = L->seg[2 * i + 1];
  const float r0 = line_r(L, a), r1 = line_r(L, b);
  float pt[4][3];
  for (int k = 0; k < 3; k++) {
    pt[0][k] = L->pos[3 * a + k] - r0;
    pt[1][k] = L->pos[3 * a + k] + r0;
    pt[2][k] = L->pos[3 * b + k] - r1;
    pt[3][k] = L->pos[3 * b + k] + r1;
  }
  for (int k = 0; k < 3; k++) bmin[k] = bmax[k] = pt[0][k];
  for (int q = 1; q < 4; q++)
    for (int k = 0; k < 3; k++) {
      bmin[k] = (bmin[k] < pt[q][k]) ? bmin[k] : pt[q][k];
      bmax[k] = (bmax[k] > pt[q][k]) ? bmax[k] : pt[q][k];
    }
  const float eps = FLT_EPSILON * 16.0f;
  for (int k = 0; k < 3; k++) {
    bmin[k] -= bmin[k] * eps;
    bmax[k] += bmax[k] * eps;
  }
}

/* ComputeBoundingBox (:142-163) over idx[l, r). */
static void line_range_box(const so_lines *L, size_t l, size_t r, float bmin[3],
                           float bmax[3]) {
  line_box(L, L->idx[l], bmin, bmax);
  for (size_t i = l; i < r; i++) {
    float c0[3], c1[3];
    line_box(L, L->idx[i], c0, c1);
    for (int k = 0; k < 3; k++) {
      bmin[k] = (bmin[k] < c0[k]) ? bmin[k] : c0[k];
      bmax[k] = (bmax[k] > c1[k]) ? bmax[k] : c1[k];
    }
  }
}

/* PartPred (:118-139): the segment's midpoint (p0 + p1) * 0.5 below pos. */
static inline int line_left(const so_lines *L, uint32_t i, int axis, float pos) {
  const uint32_t a = L->seg[2 * i], b = L->seg[2 * i + 1];
  const float c = (L->pos[3 * a + axis] + L->pos[3 * b + axis]) * 0.5f;
  return c < pos;
}

/* The two-ended partition of libstdc++'s std::partition for bidirectional
 * iterators: skip left-side items from the front and right-side items from
 * the back, swap the two that stop the scans, repeat. */
static size_t line_partition(so_lines *L, size_t first, size_t last, int axis, float pos) {
  for (;;) {
    for (;;) {
      if (first == last) return first;
      if (line_left(L, L->idx[first], axis, pos))
        first++;
      else
        break;
    }
    last--;
    for (;;) {
      if (first == last) return first;
      if (!line_left(L, L->idx[last], axis, pos))
        last--;
      else
        break;
    }
    const uint32_t t = L->idx[first];
    L->idx[first] = L->idx[last];
    L->idx[last] = t;
    first++;
  }
}

static size_t line_push(so_lines *L) {
  if (L->nnodes == L->ncap) {
    L->ncap = L->ncap ? 2 * L->ncap : 64;
    L->nodes = (so_line_node *)realloc(L->nodes, L->ncap * sizeof(so_line_node));
  }
  memset(&L->nodes[L->nnodes], 0, sizeof(so_line_node));
  return L->nnodes++;
}

/* LineAccel::BuildTree (:167-296): a leaf below min_leaf lines or at
 * max_depth; else the spatial median of the longest axis first (the cut
 * position formed in double, stored as float), then the next axes, and the
 * object median when no axis splits. */
static size_t line_build(so_lines *L, size_t l, size_t r, int depth) {
  const size_t off = line_push(L);
  if (L->depth_seen < depth) L->depth_seen = depth;
  float bmin[3], bmax[3];
  line_range_box(L, l, r, bmin, bmax);
  const size_t n = r - l;
  if (n < (size_t)L->min_leaf || depth >= L->max_depth) {
    so_line_node *nd = &L->nodes[off];
    memcpy(nd->bmin, bmin, sizeof(bmin));
    memcpy(nd->bmax, bmax, sizeof(bmax));
    nd->flag = 1;
    nd->data[0] = (uint32_t)n;
    nd->data[1] = (uint32_t)l;
    return off;
  }
  float bsize[3];
  for (int k = 0; k < 3; k++) bsize[k] = bmax[k] - bmin[k];
  float maxsize = bsize[0];
  int longest = 0;
  if (maxsize < bsize[1]) {
    maxsize = bsize[1];
    longest = 1;
  }
  if (maxsize < bsize[2]) {
    maxsize = bsize[2];
    longest = 2;
  }
  size_t mid = 0;
  int axis = 0;
  for (int t = 0; t < 3; t++) {
    axis = (longest + t) % 3;
    const float pos = (float)((double)bmin[axis] + 0.5 * (double)bsize[axis]);
    mid = line_partition(L, l, r, axis, pos);
    if (mid == l || mid == r)
      mid = l + (n >> 1);
    else
      break;
  }
  L->nodes[off].axis = axis;
  const size_t left = line_build(L, l, mid, depth + 1);
  const size_t right = line_build(L, mid, r, depth + 1);
  so_line_node *nd = &L->nodes[off];
  nd->data[0] = (uint32_t)left;
  nd->data[1] = (uint32_t)right;
  memcpy(nd->bmin, bmin, sizeof(bmin));
  memcpy(nd->bmax, bmax, sizeof(bmax));
  return off;
}

SO_API so_lines *so_line_build(const float *pos, const float *radius, float const_radius,
                               const uint32_t *seg, size_t n, int min_leaf, int max_depth,
                               int cap) {
  so_lines *L = (so_lines *)calloc(1, sizeof(so_lines));
  L->pos = pos;
  L->radius = radius;
  L->constr = const_radius;
  L->seg = seg;
  L->n = n;
  L->min_leaf = min_leaf > 0 ? min_leaf : 4;
  L->max_depth = max_depth > 0 ? max_depth : 512;
  L->cap = cap;
  L->idx = (uint32_t *)malloc((n ? n : 1) * sizeof(uint32_t));
  for (size_t i = 0; i < n; i++) L->idx[i] = (uint32_t)i;
  if (n) line_build(L, 0, n, 0);
  return L;
}

SO_API void so_line_free(so_lines *L) {
  if (!L) return;
  free(L->nodes);
  free(L->idx);
  free(L);
}

SO_API size_t so_line_num_nodes(const so_lines *L) { return L->nnodes; }
SO_API int so_line_depth(const so_lines *L) { return L->depth_seen; }

SO_API void so_line_export(const so_lines *L, so_line_node *nodes, uint32_t *idx) {
  if (nodes) memcpy(nodes, L->nodes, L->nnodes * sizeof(so_line_node));
  if (idx) memcpy(idx, L->idx, L->n * sizeof(uint32_t));
}

static inline float ldot(const float a[3], const float b[3]) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

/* vnormalize (:439-454): the length through the double sqrt, unchanged when
 * not above FLT_EPSILON * 16. */
static inline void lnormalize(const float a[3], float out[3]) {
  const float len = (float)sqrt((double)ldot(a, a));
  out[0] = a[0];
  out[1] = a[1];
  out[2] = a[2];
  if (len > FLT_EPSILON * 16.0f) {
    const float inv = (float)(1.0 / (double)len);
    for (int k = 0; k < 3; k++) out[k] *= inv;
  }
}

/* solve2e (:456-486); returns the smaller root in root0. */
static int line_solve(float *root0, float A, float B, float C) {
  if (fabsf(A) <= FLT_EPSILON) {
    *root0 = -C / B;
    return 1;
  }
  const float D = B * B - A * C;
  if (D < 0) return 0;
  if (D == 0) {
    *root0 = -B / A;
    return 1;
  }
  float x1 = (float)(((double)fabsf(B) + sqrt((double)D)) / (double)A);
  if (B >= 0.0f) x1 = -x1;
  const float x2 = C / (A * x1);
  *root0 = x1 > x2 ? x2 : x1;
  return 2;
}

/* CylinderIsect (:488-577): the two end planes (caps) first, then the side
 * surface of the cylinder of radius max(r0, r1). */
static int line_isect(float *pt, float *pu, float *pv, int *hit_cap, const float p0[3],
                      float r0, const float p1[3], float r1, const float org[3],
                      const float dir[3], int cap) {
  const float tmax = *pt;
  const float rr = r0 > r1 ? r0 : r1;
  float d[3], m[3];
  for (int k = 0; k < 3; k++) {
    d[k] = p1[k] - p0[k];
    m[k] = org[k] - p0[k];
  }
  const float md = ldot(m, d), nd = ldot(dir, d), dd = ldot(d, d);
  *hit_cap = 0;
  float capT = FLT_MAX;
  if (cap) {
    float dn0[3], dn1[3], rd[3], e[3];
    for (int k = 0; k < 3; k++) e[k] = p0[k] - p1[k];
    lnormalize(e, dn0);
    for (int k = 0; k < 3; k++) dn1[k] = -dn0[k];
    lnormalize(dir, rd);
    if (fabsf(ldot(dir, dn0)) > 1.0e-6f) {
      const float p0D = -ldot(p0, dn0), p1D = -ldot(p1, dn1);
      const float p0T = -(ldot(org, dn0) + p0D) / ldot(rd, dn0);
      const float p1T = -(ldot(org, dn1) + p1D) / ldot(rd, dn1);
      float q0[3], q1[3];
      for (int k = 0; k < 3; k++) {
        q0[k] = org[k] + rd[k] * p0T;
        q1[k] = org[k] + rd[k] * p1T;
      }
      float a0[3], a1[3];
      for (int k = 0; k < 3; k++) {
        a0[k] = q0[k] - p0[k];
        a1[k] = q1[k] - p1[k];
      }
      const float s0 = ldot(a0, a0), s1 = ldot(a1, a1);
      if (p0T > 0.0f && p0T < tmax && (s0 < rr * rr)) {
        *hit_cap = 1;
        capT = p0T;
        *pt = capT;
        *pu = (float)sqrt((double)s0);
        *pv = 0.0f;
      }
      if (p1T > 0.0f && p1T < tmax && p1T < capT && (s1 < rr * rr)) {
        *hit_cap = 1;
        capT = p1T;
        *pt = capT;
        *pu = (float)sqrt((double)s1);
        *pv = 1.0f;
      }
    }
  }
  if (md <= 0.0f && nd <= 0.0f) return *hit_cap;
  if (md >= dd && nd >= 0.0f) return *hit_cap;
  const float nn = ldot(dir, dir), mn = ldot(m, dir);
  const float A = dd * nn - nd * nd;
  const float kk = ldot(m, m) - rr * rr;
  const float C = dd * kk - md * md;
  const float B = dd * mn - nd * md;
  float t;
  if (line_solve(&t, A, B, C)) {
    if (0 <= t && t <= tmax && t <= capT) {
      float s = md + t * nd;
      s /= dd;
      if (0 <= s && s <= 1) {
        *hit_cap = 0;
        *pt = t;
        *pu = 0.0f;
        *pv = s;
        return 1;
      }
    }
  }
  return *hit_cap;
}

/* IntersectRayAABB (:377-420) with the reference's selection order. */
static inline int line_box_hit(const so_line_node *nd, const float org[3], const float inv[3],
                               const int sign[3], float maxT) {
  float lo[3], hi[3];
  for (int k = 0; k < 3; k++) {
    lo[k] = sign[k] ? nd->bmax[k] : nd->bmin[k];
    hi[k] = sign[k] ? nd->bmin[k] : nd->bmax[k];
  }
  const float tx0 = (lo[0] - org[0]) * inv[0], tx1 = (hi[0] - org[0]) * inv[0];
  const float ty0 = (lo[1] - org[1]) * inv[1], ty1 = (hi[1] - org[1]) * inv[1];
  float tmin = (tx0 > ty0) ? tx0 : ty0;
  float tmax = (tx1 < ty1) ? tx1 : ty1;
  const float tz0 = (lo[2] - org[2]) * inv[2], tz1 = (hi[2] - org[2]) * inv[2];
  tmin = (tmin > tz0) ? tmin : tz0;
  tmax = (tmax < tz1) ? tmax : tz1;
  return (tmax > 0.0f) && (tmin <= tmax) && (tmin <= maxT);
}

/* LineAccel::Traverse (:704-774) and BuildIntersection (:654-701). */
static void line_trace_one(const so_lines *L, const so_ray *ray, so_hit *hit, float *normal) {
  float hitT = FLT_MAX, it = FLT_MAX, iu = 0.0f, iv = 0.0f;
  int icap = 0;
  uint32_t prim = 0xffffffffu;
  int sign[3];
  float inv[3];
  for (int k = 0; k < 3; k++) {
    sign[k] = ray->dir[k] < 0.0f ? 1 : 0;
    inv[k] = (float)(1.0 / (double)ray->dir[k]);
  }
  int stack[520];
  int sp = 0;
  stack[0] = 0;
  while (L->nnodes && sp >= 0) {
    const so_line_node *nd = &L->nodes[stack[sp]];
    sp--;
    if (nd->flag == 0) {
      if (line_box_hit(nd, ray->org, inv, sign, hitT)) {
        const int nearc = sign[nd->axis];
        stack[++sp] = (int)nd->data[1 - nearc];
        stack[++sp] = (int)nd->data[nearc];
      }
    } else {
      float t = it;
      int any = 0;
      for (uint32_t j = 0; j < nd->data[0]; j++) {
        const uint32_t i = L->idx[nd->data[1] + j];
        const uint32_t a = L->seg[2 * i], b = L->seg[2 * i + 1];
        float u, v;
        int hc = 0;
        if (line_isect(&t, &u, &v, &hc, &L->pos[3 * a], line_r(L, a), &L->pos[3 * b],
                       line_r(L, b), ray->org, ray->dir, L->cap)) {
          it = t;
          iu = u;
          iv = v;
          icap = hc;
          prim = i;
          any = 1;
        }
      }
      if (any) hitT = it;
    }
  }
  if (it < FLT_MAX) {
    hit->t = it;
    hit->u = iu;
    hit->v = iv;
    hit->prim = prim;
    if (normal) {
      const uint32_t a = L->seg[2 * prim], b = L->seg[2 * prim + 1];
      const float *p0 = &L->pos[3 * a], *p1 = &L->pos[3 * b];
      float p[3], d[3], n[3];
      for (int k = 0; k < 3; k++) {
        p[k] = ray->org[k] + it * ray->dir[k];
        d[k] = p1[k] - p0[k];
      }
      if (icap) {
        float c[3], pc[3];
        for (int k = 0; k < 3; k++) c[k] = d[k] * 0.5f + p0[k];
        lnormalize(d, n);
        for (int k = 0; k < 3; k++) pc[k] = p[k] - c[k];
        if (!(ldot(pc, n) > 0.0f))
          for (int k = 0; k < 3; k++) n[k] = -n[k];
      } else {
        float e[3];
        for (int k = 0; k < 3; k++) e[k] = p[k] - (p0[k] + iv * d[k]);
        lnormalize(e, n);
      }
      for (int k = 0; k < 3; k++) normal[k] = n[k];
    }
  } else {
    hit->t = FLT_MAX;
    hit->u = hit->v = 0.0f;
    hit->prim = 0xffffffffu;
    if (normal) normal[0] = normal[1] = normal[2] = 0.0f;
  }
}

SO_API void so_line_trace(const so_lines *L, const so_ray *rays, size_t n, so_hit *hits,
                          float *normals, int nthreads) {
#ifdef _OPENMP
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 256) num_threads(nthreads)
#endif
  for (long long i = 0; i < (long long)n; i++)
    line_trace_one(L, &rays[i], &hits[i], normals ? &normals[3 * i] : NULL);
}

/* ------------------------------------------------------------------------ */
/* Solids: SolidAccel (render/render_accel_solid.cc) -- pyramids (5          */
/* vertices), prisms (6) and hexahedra (8).  Build32 (:1795-2124): the LBVH  */
/* of the tetrahedra with the solid's centroid (the running sum of its       */
/* vertices times 1.0f / nv); Traverse (:2345-2435): every popped node tests */
/* its own box, leaves test their solids in double (Intersect*D, :455-717).  */
/* The reference's TestLeafNode returns a shadowed flag (always false), so   */
/* the walk never lowers its distance bound: no box is culled by distance.   */
/* ------------------------------------------------------------------------ */

typedef struct {
  float bmin[3], bmax[3];
  int32_t flag, axis;
  uint32_t data[2];
} so_solid_node; /* 40 bytes, the reference's SolidNode and Dump() record */

typedef struct {
  int nv;
  const float *v;
  const uint32_t *ix;
  size_t n;
  so_solid_node *nodes;
  size_t nnodes, ncap;
  uint32_t *sidx, *code, *child;
  uint8_t *lt, *rt;
  const double *dv; /* double-precision positions (isDoublePrecisionPos), else NULL */
} so_solids;

/* Vertex coordinates: as float, as double, and padded by FLT_EPSILON * 16
 * (ComputeBoundingBox*: float positions in float; double positions in
 * double, then rounded to float). */
static inline float s_f(const so_solids *S, size_t f, int k) {
  return S->dv ? (float)S->dv[3 * f + k] : S->v[3 * f + k];
}
static inline double s_d(const so_solids *S, size_t f, int k) {
  return S->dv ? S->dv[3 * f + k] : (double)S->v[3 * f + k];
}
static inline float s_lo(const so_solids *S, size_t f, int k) {
  const float eps = FLT_EPSILON * 16;
  return S->dv ? (float)(S->dv[3 * f + k] - (double)eps) : S->v[3 * f + k] - eps;
}
static inline float s_hi(const so_solids *S, size_t f, int k) {
  const float eps = FLT_EPSILON * 16;
  return S->dv ? (float)(S->dv[3 * f + k] + (double)eps) : S->v[3 * f + k] + eps;
}

/* Leaf box over sorted solids [l, r) (ComputeBoundingBox30, :1121-1169). */
static void solid_box(const so_solids *S, size_t l, size_t r, float bmin[3], float bmax[3]) {
  const uint32_t f0 = S->ix[(size_t)S->nv * S->sidx[l]];
  for (int k = 0; k < 3; k++) {
    bmin[k] = s_lo(S, f0, k);
    bmax[k] = s_hi(S, f0, k);
  }
  for (size_t i = l; i < r; i++)
    for (int j = 0; j < S->nv; j++) {
      const uint32_t f = S->ix[(size_t)S->nv * S->sidx[i] + j];
      for (int k = 0; k < 3; k++) {
        const float lo = s_lo(S, f, k), hi = s_hi(S, f, k);
        if (bmin[k] > lo) bmin[k] = lo;
        if (bmax[k] < hi) bmax[k] = hi;
      }
    }
}

static inline int solid_axis(uint32_t code) { return (clz32(code) - 2) % 3; }

static size_t solid_push(so_solids *S) {
  if (S->nnodes == S->ncap) {
    S->ncap = S->ncap ? 2 * S->ncap : 64;
    S->nodes = (so_solid_node *)realloc(S->nodes, S->ncap * sizeof(so_solid_node));
  }
  memset(&S->nodes[S->nnodes], 0, sizeof(so_solid_node));
  return S->nnodes++;
}

/* BuildTreeRecursive32 (:1361-1453): keys [l, r] inclusive. */
static size_t solid_emit(so_solids *S, uint32_t root, uint32_t l, uint32_t r, int leaf,
                         int depth, float bmin[3], float bmax[3]) {
  if (leaf || (r - l) <= 4 || depth > 22) {
    const size_t off = solid_push(S);
    solid_box(S, l, (size_t)r + 1, bmin, bmax);
    so_solid_node *nd = &S->nodes[off];
    memcpy(nd->bmin, bmin, 12);
    memcpy(nd->bmax, bmax, 12);
    nd->flag = 1;
    nd->data[0] = r + 1 - l;
    nd->data[1] = l;
    return off;
  }
  const uint32_t mid = S->child[root];
  const size_t off = solid_push(S);
  float lb0[3], lb1[3], rb0[3], rb1[3];
  const size_t left = solid_emit(S, mid, l, mid, S->lt[root], depth + 1, lb0, lb1);
  const size_t right = solid_emit(S, mid + 1, mid + 1, r, S->rt[root], depth + 1, rb0, rb1);
  for (int k = 0; k < 3; k++) { /* MergeBoundingBox: std::min / std::max */
    bmin[k] = (rb0[k] < lb0[k]) ? rb0[k] : lb0[k];
    bmax[k] = (lb1[k] < rb1[k]) ? rb1[k] : lb1[k];
  }
  so_solid_node *nd = &S->nodes[off];
  nd->axis = solid_axis(S->code[root]);
  nd->data[0] = (uint32_t)left;
  nd->data[1] = (uint32_t)right;
  memcpy(nd->bmin, bmin, 12);
  memcpy(nd->bmax, bmax, 12);
  return off;
}

/* SolidAccel::Build (:1612-1793, binned SAH on 64 bins, costTaabb 0.2,
 * minLeafPrimitives 4, maxTreeDepth 256), which Build32 runs below 1024
 * solids (:1806-1809).  Float arithmetic in the reference's order. */
static size_t sah_vert(const so_solids *S, uint32_t solid, int j) {
  return S->ix[(size_t)S->nv * solid + j];
}

/* CalculateSurfaceArea (:791-799) */
static float sah_area(const float lo[3], const float hi[3]) {
  const float b0 = hi[0] - lo[0], b1 = hi[1] - lo[1], b2 = hi[2] - lo[2];
  const float sum = (b0 * b1 + b1 * b2) + b2 * b0;
  return (float)(2.0 * (double)sum);
}

/* SAHPred / SAHPredD (:1034-1074): a float sum (double addends added in
 * double) against pos * nv (float; double for double positions) */
static int sah_left(const so_solids *S, uint32_t solid, int axis, float pos) {
  float c = 0.0f;
  if (S->dv) {
    for (int j = 0; j < S->nv; j++) c = (float)((double)c + s_d(S, sah_vert(S, solid, j), axis));
    return (double)c < (double)pos * (double)(float)S->nv;
  }
  for (int j = 0; j < S->nv; j++) c += s_f(S, sah_vert(S, solid, j), axis);
  return c < pos * (float)S->nv;
}

/* std::partition of libstdc++ on bidirectional iterators (both ends) */
static uint32_t sah_partition(so_solids *S, uint32_t first, uint32_t last, int axis, float pos) {
  for (;;) {
    for (;;) {
      if (first == last) return first;
      if (sah_left(S, S->sidx[first], axis, pos)) first++;
      else break;
    }
    last--;
    for (;;) {
      if (first == last) return first;
      if (!sah_left(S, S->sidx[last], axis, pos)) last--;
      else break;
    }
    const uint32_t t = S->sidx[first];
    S->sidx[first] = S->sidx[last];
    S->sidx[last] = t;
    first++;
  }
}

static size_t sah_build(so_solids *S, uint32_t l, uint32_t r, int depth) {
  const float eps = FLT_EPSILON * 16;
  enum { BINS = 64 };
  /* ComputeBoundingBox (:1076-1118) */
  float bmin[3], bmax[3];
  const size_t p0 = sah_vert(S, S->sidx[l], 0);
  for (int k = 0; k < 3; k++) {
    bmin[k] = s_lo(S, p0, k);
    bmax[k] = s_hi(S, p0, k);
  }
  for (uint32_t i = l; i < r; i++)
    for (int j = 0; j < S->nv; j++) {
      const size_t pj = sah_vert(S, S->sidx[i], j);
      for (int k = 0; k < 3; k++) {
        const float mn = s_lo(S, pj, k), mx = s_hi(S, pj, k);
        if (bmin[k] > mn) bmin[k] = mn;
        if (bmax[k] < mx) bmax[k] = mx;
      }
    }
  const size_t me = solid_push(S);
  so_solid_node *nd = &S->nodes[me];
  for (int k = 0; k < 3; k++) {
    nd->bmin[k] = bmin[k];
    nd->bmax[k] = bmax[k];
  }
  const uint32_t n = r - l;
  if (n < 4 || depth >= 256) {
    nd->flag = 1;
    nd->data[0] = n;
    nd->data[1] = l;
    return me;
  }
  /* ContributeBinBuffer (:833-887) */
  static _Thread_local size_t bins[2][3][BINS];
  memset(bins, 0, sizeof(bins));
  float inv[3];
  for (int k = 0; k < 3; k++) {
    const float size = bmax[k] - bmin[k];
    inv[k] = size > eps ? (float)BINS / size : 0.0f;
  }
  for (uint32_t i = l; i < r; i++) {
    float slo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, shi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (int j = 0; j < S->nv; j++) { /* GetBoundingBoxOfSolid: std::min / std::max */
      const size_t pj = sah_vert(S, S->sidx[i], j);
      for (int k = 0; k < 3; k++) {
        const float x = s_f(S, pj, k);
        if (x < slo[k]) slo[k] = x;
        if (shi[k] < x) shi[k] = x;
      }
    }
    for (int k = 0; k < 3; k++) {
      size_t a = (size_t)(unsigned int)floorf((slo[k] - bmin[k]) * inv[k]);
      size_t b = (size_t)(unsigned int)floorf((shi[k] - bmin[k]) * inv[k]);
      if (a >= BINS) a = BINS - 1;
      if (b >= BINS) b = BINS - 1;
      bins[0][k][a]++;
      bins[1][k][b]++;
    }
  }
  /* FindCutFromBinBuffer (:916-988) and SAH (:890-899) */
  const float taabb = 0.2f, ttri = (float)(1.0 - (double)taabb);
  float bstep[3], cut[3], best[3];
  for (int k = 0; k < 3; k++) bstep[k] = (bmax[k] - bmin[k]) * (float)(1.0 / BINS);
  const float sa = sah_area(bmin, bmax);
  const float inv_sa = sa > eps ? (float)(1.0 / (double)sa) : 0.0f;
  for (int k = 0; k < 3; k++) {
    float best_pos = bmin[k] + 0.5f * bstep[k];
    best[k] = FLT_MAX;
    size_t left = 0, right = n;
    float llo[3], lhi[3], rlo[3], rhi[3];
    for (int q = 0; q < 3; q++) {
      llo[q] = rlo[q] = bmin[q];
      lhi[q] = rhi[q] = bmax[q];
    }
    for (int i = 0; i < BINS - 1; i++) {
      left += bins[0][k][i];
      right -= bins[1][k][i];
      const float pos = bmin[k] + ((float)i + 0.5f) * bstep[k];
      lhi[k] = pos;
      rlo[k] = pos;
      const float sl = sah_area(llo, lhi), sr = sah_area(rlo, rhi);
      const float t1 = ((sl * inv_sa) * (float)left) * ttri;
      const float t2 = ((sr * inv_sa) * (float)right) * ttri;
      const float cost = (2.0f * taabb + t1) + t2;
      if (cost < best[k]) {
        best[k] = cost;
        best_pos = pos;
      }
    }
    cut[k] = best_pos;
  }
  int ax = 0;
  float c = best[0];
  if (c > best[1]) {
    ax = 1;
    c = best[1];
  }
  if (c > best[2]) ax = 2;
  uint32_t mid = l;
  int axis = ax;
  for (int t = 0; t < 3; t++) {
    axis = (ax + t) % 3;
    mid = sah_partition(S, l, r, axis, cut[axis]);
    if (mid == l || mid == r) mid = l + (n >> 1);
    else break;
  }
  const size_t lc = sah_build(S, l, mid, depth + 1);
  const size_t rc = sah_build(S, mid, r, depth + 1);
  nd = &S->nodes[me]; /* the node array may have moved */
  nd->flag = 0;
  nd->axis = axis;
  nd->data[0] = (uint32_t)lc;
  nd->data[1] = (uint32_t)rc;
  return me;
}

static so_solids *solid_build(int nv, const float *v, const double *dv, const uint32_t *ix,
                              size_t n, int sah) {
  so_solids *S = (so_solids *)calloc(1, sizeof(so_solids));
  S->nv = nv;
  S->v = v;
  S->dv = dv;
  S->ix = ix;
  S->n = n;
  S->sidx = (uint32_t *)malloc((n + 1) * 4);
  S->code = (uint32_t *)malloc((n + 1) * 4);
  S->child = (uint32_t *)malloc((n + 1) * 4);
  S->lt = (uint8_t *)malloc(n + 1);
  S->rt = (uint8_t *)malloc(n + 1);
  if (sah || n < 1024) { /* Build; Build32 runs it below 1024 solids */
    for (size_t i = 0; i < n; i++) S->sidx[i] = (uint32_t)i;
    if (n > 0) sah_build(S, 0, (uint32_t)n, 0);
    return S;
  }
  /* scene box: every vertex -+ FLT_EPSILON * 16 (ComputeBoundingBoxOMP, :1171-1262) */
  float lo[3], hi[3];
  for (int k = 0; k < 3; k++) {
    lo[k] = s_lo(S, ix[0], k);
    hi[k] = s_hi(S, ix[0], k);
  }
  for (size_t i = 0; i < n * (size_t)nv; i++)
    for (int k = 0; k < 3; k++) {
      lo[k] = fmin_ref(lo[k], s_lo(S, ix[i], k));
      hi[k] = fmax_ref(hi[k], s_hi(S, ix[i], k));
    }
  /* CalculateMortonCodesSolidFloat30 (render/render_prefix_tree_util.cc:347-382) */
  float inv[3];
  morton_inv(lo, hi, inv);
  const float invdiv = 1.0f / (float)nv;
  for (size_t i = 0; i < n; i++) {
    float c[3] = {0.0f, 0.0f, 0.0f};
    for (int j = 0; j < nv; j++)
      for (int k = 0; k < 3; k++) c[k] = c[k] + s_f(S, ix[(size_t)nv * i + j], k);
    for (int k = 0; k < 3; k++) c[k] *= invdiv;
    S->code[i] = morton_of(c, lo, inv);
    S->sidx[i] = (uint32_t)i;
  }
  so_sort_pairs(S->code, S->sidx, n);
  so_karras(S->code, n, S->child, S->lt, S->rt);
  solid_push(S); /* the root, filled below */
  float lb0[3], lb1[3], rb0[3], rb1[3];
  const uint32_t mid = S->child[0];
  const size_t left = solid_emit(S, mid, 0, mid, S->lt[0], 0, lb0, lb1);
  const size_t right = solid_emit(S, mid + 1, mid + 1, (uint32_t)n - 1, S->rt[0], 0, rb0, rb1);
  so_solid_node *rt = &S->nodes[0];
  for (int k = 0; k < 3; k++) {
    rt->bmin[k] = (rb0[k] < lb0[k]) ? rb0[k] : lb0[k];
    rt->bmax[k] = (lb1[k] < rb1[k]) ? rb1[k] : lb1[k];
  }
  rt->axis = solid_axis(S->code[0]);
  rt->data[0] = (uint32_t)left;
  rt->data[1] = (uint32_t)right;
  return S;
}

SO_API so_solids *so_solid_build(int nv, const float *v, const uint32_t *ix, size_t n) {
  return solid_build(nv, v, NULL, ix, n, 0);
}

/* Double-precision positions (Solid::dvertices, isDoublePrecisionPos). */
SO_API so_solids *so_solid_build_d(int nv, const double *dv, const uint32_t *ix, size_t n) {
  return solid_build(nv, NULL, dv, ix, n, 0);
}

/* SolidAccel::Build (binned SAH) at every size, float or double positions. */
SO_API so_solids *so_solid_build_sah(int nv, const float *v, const double *dv,
                                     const uint32_t *ix, size_t n) {
  return solid_build(nv, v, dv, ix, n, 1);
}

SO_API void so_solid_free(so_solids *S) {
  if (!S) return;
  free(S->nodes);
  free(S->sidx);
  free(S->code);
  free(S->child);
  free(S->lt);
  free(S->rt);
  free(S);
}

SO_API size_t so_solid_num_nodes(const so_solids *S) { return S->nnodes; }

SO_API void so_solid_export(const so_solids *S, so_solid_node *nodes, uint32_t *idx) {
  if (nodes) memcpy(nodes, S->nodes, S->nnodes * sizeof(so_solid_node));
  if (idx) memcpy(idx, S->sidx, S->n * 4);
}

/* --- the Pluecker tests in double ---------------------------------------- */
typedef struct {
  float pos[3], nrm[3];
  float t;
} so_sisect;

static inline d3 dsub(d3 a, d3 b) { return (d3){a.x - b.x, a.y - b.y, a.z - b.z}; }
static inline d3 dcross(d3 a, d3 b) {
  return (d3){a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
static inline double ddot(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline d3 dscale(d3 a, double f) { return (d3){a.x * f, a.y * f, a.z * f}; }
static inline d3 dadd(d3 a, d3 b) { return (d3){a.x + b.x, a.y + b.y, a.z + b.z}; }

/* normalize (:85): a / |a| in double, then to float. */
static inline void s_unit(d3 a, float out[3]) {
  const double len = sqrt(a.x * a.x + a.y * a.y + a.z * a.z);
  out[0] = (float)(a.x / len);
  out[1] = (float)(a.y / len);
  out[2] = (float)(a.z / len);
}

/* SetCrossPoint_Sq (double, :438-444): the crossing point of a quad face. */
static inline void s_quad_point(float out[3], d3 v0, d3 v1, d3 v2, double ws0, double ws1,
                                double ws2, double ws3, d3 e2, d3 e3, d3 dir) {
  const double w = ws2 + ws3 + ddot(dcross(e2, e3), dir);
  const d3 p = dadd(dadd(dscale(v2, ws0), dscale(v0, ws1)), dscale(v1, w));
  const double den = ws0 + ws1 + w;
  out[0] = (float)(p.x / den);
  out[1] = (float)(p.y / den);
  out[2] = (float)(p.z / den);
}

/* The crossing point of a triangle face: toreal3(a*wa + b*wb + c*wc) / (float)(wa + wb + wc),
 * the weighted sum in double, the division in float. */
static inline void s_tri_point(float out[3], d3 a, double wa, d3 b, double wb, d3 c, double wc,
                               double den) {
  const d3 p = dadd(dadd(dscale(a, wa), dscale(b, wb)), dscale(c, wc));
  const float f = (float)den;
  out[0] = (float)p.x / f;
  out[1] = (float)p.y / f;
  out[2] = (float)p.z / f;
}

static inline void s_weights(int ne, const d3 *e, const d3 *vv, int mod, d3 dir, d3 org,
                             double *ws, int cw[2][12]) {
  const d3 rpc = dcross(dir, org);
  for (int i = 0; i < ne; i++) {
    const d3 epc = dcross(e[i], vv[i % mod]);
    ws[i] = ddot(dir, epc) + ddot(e[i], rpc);
    cw[0][i] = ws[i] >= 0;
    cw[1][i] = ws[i] <= 0;
  }
}

/* t of both points along the last axis with |dir| > 0.1 (:500-504). */
static inline void s_params(so_sisect is[2], d3 org, d3 dir) {
  const double o[3] = {org.x, org.y, org.z}, d[3] = {dir.x, dir.y, dir.z};
  for (int j = 0; j < 3; j++)
    if (d[j] > 0.1 || d[j] < -0.1) {
      is[0].t = (float)(((double)is[0].pos[j] - o[j]) / d[j]);
      is[1].t = (float)(((double)is[1].pos[j] - o[j]) / d[j]);
    }
  for (int k = 0; k < 3; k++) is[1].nrm[k] = -1.0f * is[1].nrm[k];
}

/* IntersectPyramidD (:455-505). */
static int s_pyramid(d3 org, d3 dir, const d3 *v, so_sisect is[2]) {
  d3 e[8] = {dsub(v[1], v[0]), dsub(v[2], v[1]), dsub(v[3], v[2]), dsub(v[0], v[3]),
             dsub(v[4], v[0]), dsub(v[4], v[1]), dsub(v[4], v[2]), dsub(v[4], v[3])};
  double ws[12];
  int cw[2][12];
  s_weights(8, e, v, 4, dir, org, ws, cw);
  for (int i = 1, n = 0; n < 2; i--, n++) {
    if (cw[i][0] && cw[i][1] && cw[i][2] && cw[i][3]) {
      s_quad_point(is[n].pos, v[0], v[1], v[2], ws[0], ws[1], ws[2], ws[3], e[2], e[3], dir);
      s_unit(dcross(e[1], e[0]), is[n].nrm);
    } else if (cw[n][0] && cw[i][4] && cw[n][5]) {
      s_tri_point(is[n].pos, v[4], -ws[0], v[1], ws[4], v[0], -ws[5], -ws[0] + ws[4] - ws[5]);
      s_unit(dcross(e[4], e[0]), is[n].nrm);
    } else if (cw[n][1] && cw[i][5] && cw[n][6]) {
      s_tri_point(is[n].pos, v[4], -ws[1], v[2], ws[5], v[1], -ws[6], -ws[1] + ws[5] - ws[6]);
      s_unit(dcross(e[5], e[1]), is[n].nrm);
    } else if (cw[n][2] && cw[i][6] && cw[n][7]) {
      s_tri_point(is[n].pos, v[4], -ws[2], v[3], ws[6], v[2], -ws[7], -ws[2] + ws[6] - ws[7]);
      s_unit(dcross(e[6], e[2]), is[n].nrm);
    } else if (cw[n][3] && cw[i][7] && cw[n][4]) {
      s_tri_point(is[n].pos, v[4], -ws[3], v[0], ws[7], v[3], -ws[4], -ws[3] + ws[7] - ws[4]);
      s_unit(dcross(e[7], e[3]), is[n].nrm);
    } else {
      return 0;
    }
  }
  s_params(is, org, dir);
  return 1;
}

/* IntersectPrismD (:559-611). */
static int s_prism(d3 org, d3 dir, const d3 *v, so_sisect is[2]) {
  d3 e[9] = {dsub(v[1], v[0]), dsub(v[2], v[1]), dsub(v[0], v[2]),
             dsub(v[4], v[3]), dsub(v[5], v[4]), dsub(v[3], v[5]),
             dsub(v[3], v[0]), dsub(v[4], v[1]), dsub(v[5], v[2])};
  double ws[12];
  int cw[2][12];
  s_weights(9, e, v, 6, dir, org, ws, cw);
  for (int i = 0, n = 1; i < 2; i++, n--) {
    if (cw[n][0] && cw[n][1] && cw[n][2]) {
      s_tri_point(is[i].pos, v[2], ws[0], v[0], ws[1], v[1], ws[2], ws[0] + ws[1] + ws[2]);
      s_unit(dcross(e[0], e[1]), is[i].nrm);
    } else if (cw[i][3] && cw[i][4] && cw[i][5]) {
      s_tri_point(is[i].pos, v[5], ws[3], v[3], ws[4], v[4], ws[5], ws[3] + ws[4] + ws[5]);
      s_unit(dcross(e[3], e[4]), is[i].nrm);
    } else if (cw[i][2] && cw[i][6] && cw[n][5] && cw[n][8]) {
      s_quad_point(is[i].pos, v[2], v[0], v[3], ws[2], ws[6], -ws[5], -ws[8], e[5], e[8], dir);
      s_unit(dcross(e[2], e[6]), is[i].nrm);
    } else if (cw[i][0] && cw[i][7] && cw[n][3] && cw[n][6]) {
      s_quad_point(is[i].pos, v[0], v[1], v[4], ws[0], ws[7], -ws[3], -ws[6], e[3], e[6], dir);
      s_unit(dcross(e[0], e[7]), is[i].nrm);
    } else if (cw[i][1] && cw[i][8] && cw[n][4] && cw[n][7]) {
      s_quad_point(is[i].pos, v[1], v[2], v[5], ws[1], ws[8], -ws[4], -ws[7], e[4], e[7], dir);
      s_unit(dcross(e[1], e[8]), is[i].nrm);
    } else {
      return 0;
    }
  }
  s_params(is, org, dir);
  return 1;
}

/* IntersectHexaD (:664-716). */
static int s_hexa(d3 org, d3 dir, const d3 *v, so_sisect is[2]) {
  d3 e[12] = {dsub(v[1], v[0]), dsub(v[2], v[1]), dsub(v[3], v[2]), dsub(v[0], v[3]),
              dsub(v[5], v[4]), dsub(v[6], v[5]), dsub(v[7], v[6]), dsub(v[4], v[7]),
              dsub(v[4], v[0]), dsub(v[5], v[1]), dsub(v[6], v[2]), dsub(v[7], v[3])};
  double ws[12];
  int cw[2][12];
  s_weights(12, e, v, 8, dir, org, ws, cw);
  for (int i = 0, n = 1; i < 2; i++, n--) {
    if (cw[n][0] && cw[n][1] && cw[n][2] && cw[n][3]) {
      s_quad_point(is[i].pos, v[0], v[1], v[2], ws[0], ws[1], ws[2], ws[3], e[2], e[3], dir);
      s_unit(dcross(e[0], e[1]), is[i].nrm);
    } else if (cw[i][4] && cw[i][5] && cw[i][6] && cw[i][7]) {
      s_quad_point(is[i].pos, v[4], v[5], v[6], ws[4], ws[5], ws[6], ws[7], e[6], e[7], dir);
      s_unit(dcross(e[4], e[5]), is[i].nrm);
    } else if (cw[i][0] && cw[i][9] && cw[n][4] && cw[n][8]) {
      s_quad_point(is[i].pos, v[0], v[1], v[5], ws[0], ws[9], -ws[4], -ws[8], e[4], e[8], dir);
      s_unit(dcross(e[0], e[9]), is[i].nrm);
    } else if (cw[i][1] && cw[i][10] && cw[n][5] && cw[n][9]) {
      s_quad_point(is[i].pos, v[1], v[2], v[6], ws[1], ws[10], -ws[5], -ws[9], e[5], e[9], dir);
      s_unit(dcross(e[1], e[10]), is[i].nrm);
    } else if (cw[i][2] && cw[i][11] && cw[n][6] && cw[n][10]) {
      s_quad_point(is[i].pos, v[2], v[3], v[7], ws[2], ws[11], -ws[6], -ws[10], e[6], e[10], dir);
      s_unit(dcross(e[2], e[11]), is[i].nrm);
    } else if (cw[i][3] && cw[i][8] && cw[n][7] && cw[n][11]) {
      s_quad_point(is[i].pos, v[3], v[0], v[4], ws[3], ws[8], -ws[7], -ws[11], e[7], e[11], dir);
      s_unit(dcross(e[3], e[8]), is[i].nrm);
    } else {
      return 0;
    }
  }
  s_params(is, org, dir);
  return 1;
}

/* SolidAccel::Traverse + TestLeafNode (:2206-2334): hits (t, u = v = 0: the
 * reference leaves them unset), the hit's normal and position. */
static void solid_trace_one(const so_solids *S, const so_ray *ray, so_hit *hit, float *nrm,
                            float *pos) {
  const float big = FLT_MAX;
  float t = big, bn[3] = {0, 0, 0}, bp[3] = {0, 0, 0};
  uint32_t prim = 0xffffffffu;
  int sign[3];
  float inv[3];
  for (int k = 0; k < 3; k++) {
    sign[k] = ray->dir[k] < 0.0f ? 1 : 0;
    inv[k] = (float)(1.0 / (double)ray->dir[k]);
  }
  const d3 org = {ray->org[0], ray->org[1], ray->org[2]};
  const d3 dir = {ray->dir[0], ray->dir[1], ray->dir[2]};
  int stack[520], sp = 0;
  stack[0] = 0;
  while (S->nnodes && sp >= 0) {
    const so_solid_node *nd = &S->nodes[stack[sp--]];
    const int boxhit = line_box_hit((const so_line_node *)nd, ray->org, inv, sign, big);
    if (nd->flag == 0) {
      if (boxhit) {
        const int nearc = sign[nd->axis];
        stack[++sp] = (int)nd->data[1 - nearc];
        stack[++sp] = (int)nd->data[nearc];
      }
    } else if (boxhit) {
      for (uint32_t j = 0; j < nd->data[0]; j++) {
        const uint32_t p = S->sidx[nd->data[1] + j];
        if (p == ray->prev_prim) continue;
        d3 vv[8];
        for (int q = 0; q < S->nv; q++) {
          const size_t f = S->ix[(size_t)S->nv * p + q];
          vv[q] = (d3){s_d(S, f, 0), s_d(S, f, 1), s_d(S, f, 2)};
        }
        so_sisect is[2];
        memset(is, 0, sizeof(is));
        int h = S->nv == 5 ? s_pyramid(org, dir, vv, is)
                           : (S->nv == 6 ? s_prism(org, dir, vv, is) : s_hexa(org, dir, vv, is));
        if (!h) continue;
        for (int s = 0; s < 2; s++)
          if (is[s].t >= 0.0f && is[s].t < t) {
            t = is[s].t;
            prim = p;
            memcpy(bn, is[s].nrm, 12);
            memcpy(bp, is[s].pos, 12);
          }
      }
    }
  }
  hit->t = t;
  hit->u = hit->v = 0.0f;
  hit->prim = t < big ? prim : 0xffffffffu;
  if (t >= big) {
    memset(bn, 0, 12);
    memset(bp, 0, 12);
  }
  if (nrm) memcpy(nrm, bn, 12);
  if (pos) memcpy(pos, bp, 12);
}

SO_API void so_solid_trace(const so_solids *S, const so_ray *rays, size_t n, so_hit *hits,
                           float *normals, float *positions, int nthreads) {
#ifdef _OPENMP
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 256) num_threads(nthreads)
#endif
  for (long long i = 0; i < (long long)n; i++)
    solid_trace_one(S, &rays[i], &hits[i], normals ? &normals[3 * i] : NULL,
                    positions ? &positions[3 * i] : NULL);
}

static void scene_other_trace(int kind, const void *obj, const so_ray *lr, so_hit *h) {
  if (kind == 3)
    line_trace_one((const so_lines *)obj, lr, h, NULL);
  else
    solid_trace_one((const so_solids *)obj, lr, h, NULL, NULL);
}
