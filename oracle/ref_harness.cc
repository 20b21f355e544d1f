// ref_harness.cc -- C entry points over the reference's own render/ classes.
//
// TEST INFRASTRUCTURE ONLY.  Compiled together with the unmodified reference
// sources (render/render_prefix_tree_util.cc, render_accel_triangle.cc,
// render_accel_tetra.cc, render_accel_particle.cc, render_texture.cc,
// tinymt64.cpp) by oracle/Makefile into oracle/_ref/libsurface_ref.so.  It pins
// the C restatement (surface_oracle.c) and serves as the timed CPU baseline
// ("cpu_baseline.kind = reference").  Nothing here re-implements an
// algorithm: each function only marshals plain arrays into the reference's
// own types and calls its public API:
//   TriangleAccel/TetraAccel/ParticleAccel::Build32, ::Traverse, ::Dump,
//   ::BoundingBox          (render/render_accel_*.h)
//   CalculateMortonCodes*, RadixSort30OMP, ConstructBinaryRadixTree30
//                          (render/render_prefix_tree_util.h)
//   FilterTexture3DFloat   (render/render_texture.h)
//   Camera::buildFrame     (render/render_camera.h)
//   BVHTree                (render/render_bvh_tree.h, RenderGraph's top level)
//   tinymt64_*             (render/tinymt64.h)
#include <fcntl.h>
#include <omp.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>
#include <unistd.h>

#include <limits>
#include <vector>

#include "render_accel_line.h"
#include "render_accel_particle.h"
#include "render_accel_solid.h"
#include "render_accel_tetra.h"
#include "render_accel_triangle.h"
#include "render_accel_volume.h"
#include "render_bvh_tree.h"
#include "render_camera.h"
#include "render_matrix.h"
#include "render_prefix_tree_util.h"
#include "render_texture.h"
#include "tinymt64.h"

using namespace lsgl::render;

#define REF_API extern "C" __attribute__((visibility("default")))

namespace {

// Build32 prints per-phase timings on stdout; keep stdout clean for the
// callers (bench.py prints exactly one JSON line).
struct QuietStdout {
  int saved = -1;
  QuietStdout() {
    fflush(stdout);
    int devnull = open("/dev/null", O_WRONLY);
    if (devnull >= 0) {
      saved = dup(1);
      dup2(devnull, 1);
      close(devnull);
    }
  }
  ~QuietStdout() {
    fflush(stdout);
    if (saved >= 0) {
      dup2(saved, 1);
      close(saved);
    }
  }
};

struct TriHandle {
  Mesh mesh;
  TriangleAccel accel;
  ~TriHandle() {
    // the arrays are borrowed from the caller; Mesh::~Mesh would free them
    mesh.vertices = nullptr;
    mesh.faces = nullptr;
    mesh.normals = nullptr;
    mesh.dvertices = nullptr;
  }
};

struct TetHandle {
  Tetrahedron tets;
  TetraAccel accel;
};

struct SphereHandle {
  Particles parts;
  ParticleAccel accel;
};

// Ray record shared with the oracle and the product ABI (32 bytes).
struct RayRec {
  float org[3];
  uint32_t prev_prim;
  float dir[3];
  float prev_t;
};

struct HitRec {
  float t, u, v;
  uint32_t prim;
};

inline Ray make_ray(const RayRec &r, const float *prevN) {
  real3 o(r.org[0], r.org[1], r.org[2]);
  real3 d(r.dir[0], r.dir[1], r.dir[2]);
  Ray ray(o, d);
  ray.double_sided = 1;
  ray.prev_prim_id = r.prev_prim;
  ray.prev_hit_t = r.prev_t;
  if (prevN) {
    ray.prev_hit_normal = real3(prevN[0], prevN[1], prevN[2]);
  } else {
    ray.prev_hit_normal = real3(0.0f, 0.0f, 0.0f);
  }
  ray.prev_node = nullptr;
  return ray;
}

}  // namespace

// ---------------------------------------------------------------- triangles
REF_API void *ref_tri_build(const float *verts, size_t nverts,
                            const uint32_t *faces, size_t nfaces) {
  TriHandle *h = new TriHandle();
  h->mesh.nvertices = nverts;
  h->mesh.vertices = verts;
  h->mesh.nfaces = nfaces;
  h->mesh.faces = const_cast<uint32_t *>(faces);
  h->mesh.isDoublePrecisionPos = false;
  TriangleBuildOptions opt;
  {
    QuietStdout q;
    h->accel.Build32(&h->mesh, opt);
  }
  return h;
}

REF_API void ref_tri_free(void *p) { delete static_cast<TriHandle *>(p); }

REF_API int ref_tri_dump(void *p, const char *path) {
  return static_cast<TriHandle *>(p)->accel.Dump(path) ? 0 : 1;
}

REF_API void ref_tri_bbox(void *p, double bmin[3], double bmax[3]) {
  static_cast<TriHandle *>(p)->accel.BoundingBox(bmin, bmax);
}

REF_API void ref_tri_trace(void *p, const RayRec *rays, size_t n, HitRec *hits,
                           int nthreads, int chunk) {
  const TriangleAccel &acc = static_cast<TriHandle *>(p)->accel;
  if (nthreads <= 0) nthreads = omp_get_max_threads();
  if (chunk <= 0) chunk = 64;
#pragma omp parallel for schedule(dynamic, chunk) num_threads(nthreads)
  for (long long i = 0; i < (long long)n; i++) {
    Ray ray = make_ray(rays[i], nullptr);
    Intersection isect;
    bool hit = acc.Traverse(isect, ray);
    hits[i].t = isect.t;
    hits[i].u = isect.u;
    hits[i].v = isect.v;
    hits[i].prim = hit ? isect.prim_id : 0xffffffffu;
  }
}

// ---------------------------------------------------------------- tetrahedra
REF_API void *ref_tet_build(const float *verts, const uint32_t *faces,
                            size_t ntets) {
  TetHandle *h = new TetHandle();
  memset(&h->tets, 0, sizeof(h->tets));
  h->tets.numTetrahedrons = ntets;
  h->tets.vertices = verts;
  h->tets.dvertices = nullptr;
  h->tets.isDoublePrecisionPos = false;
  h->tets.faces = const_cast<uint32_t *>(faces);
  TetraBuildOptions opt;
  {
    QuietStdout q;
    h->accel.Build32(&h->tets, opt);
  }
  return h;
}

// The same with double-precision positions (Tetrahedron::dvertices).
REF_API void *ref_tet_build_d(const double *dverts, const uint32_t *faces, size_t ntets) {
  TetHandle *h = new TetHandle();
  memset(&h->tets, 0, sizeof(h->tets));
  h->tets.numTetrahedrons = ntets;
  h->tets.vertices = nullptr;
  h->tets.dvertices = dverts;
  h->tets.isDoublePrecisionPos = true;
  h->tets.faces = const_cast<uint32_t *>(faces);
  TetraBuildOptions opt;
  {
    QuietStdout q;
    h->accel.Build32(&h->tets, opt);
  }
  return h;
}

REF_API void ref_tet_free(void *p) { delete static_cast<TetHandle *>(p); }

REF_API int ref_tet_dump(void *p, const char *path) {
  return static_cast<TetHandle *>(p)->accel.Dump(path) ? 0 : 1;
}

REF_API void ref_tet_bbox(void *p, double bmin[3], double bmax[3]) {
  static_cast<TetHandle *>(p)->accel.BoundingBox(bmin, bmax);
}

REF_API void ref_tet_trace(void *p, const RayRec *rays, size_t n, HitRec *hits,
                           uint32_t *subface, int nthreads, int chunk) {
  const TetraAccel &acc = static_cast<TetHandle *>(p)->accel;
  if (nthreads <= 0) nthreads = omp_get_max_threads();
  if (chunk <= 0) chunk = 64;
#pragma omp parallel for schedule(dynamic, chunk) num_threads(nthreads)
  for (long long i = 0; i < (long long)n; i++) {
    Ray ray = make_ray(rays[i], nullptr);
    Intersection isect;
    isect.subface_id = 0;
    bool hit = acc.Traverse(isect, ray);
    hits[i].t = isect.t;
    hits[i].u = isect.u;
    hits[i].v = isect.v;
    hits[i].prim = hit ? isect.prim_id : 0xffffffffu;
    if (subface) subface[i] = hit ? isect.subface_id : 0u;
  }
}

// ---------------------------------------------------------------- spheres
REF_API void *ref_sphere_build(const float *pos, const float *radius,
                               float const_radius, size_t n) {
  SphereHandle *h = new SphereHandle();
  memset(&h->parts, 0, sizeof(h->parts));
  h->parts.numParticles = n;
  h->parts.positions = pos;
  h->parts.dpositions = nullptr;
  h->parts.isDoublePrecisionPos = false;
  h->parts.radius = const_cast<float *>(radius);
  h->parts.materialIDs = nullptr;
  h->parts.constantRadius = const_radius;
  ParticleBuildOptions opt;
  {
    QuietStdout q;
    h->accel.Build32(&h->parts, opt);
  }
  return h;
}

REF_API void ref_sphere_free(void *p) { delete static_cast<SphereHandle *>(p); }

REF_API int ref_sphere_dump(void *p, const char *path) {
  return static_cast<SphereHandle *>(p)->accel.Dump(path) ? 0 : 1;
}

REF_API void ref_sphere_bbox(void *p, double bmin[3], double bmax[3]) {
  static_cast<SphereHandle *>(p)->accel.BoundingBox(bmin, bmax);
}

REF_API void ref_sphere_trace(void *p, const RayRec *rays, size_t n,
                              const float *prev_normals, HitRec *hits,
                              int nthreads, int chunk) {
  const ParticleAccel &acc = static_cast<SphereHandle *>(p)->accel;
  if (nthreads <= 0) nthreads = omp_get_max_threads();
  if (chunk <= 0) chunk = 64;
#pragma omp parallel for schedule(dynamic, chunk) num_threads(nthreads)
  for (long long i = 0; i < (long long)n; i++) {
    Ray ray = make_ray(rays[i], prev_normals ? &prev_normals[3 * i] : nullptr);
    Intersection isect;
    bool hit = acc.Traverse(isect, ray);
    hits[i].t = isect.t;
    hits[i].u = hit ? isect.u : 0.0f;  // BuildIntersection's spherical (u, v)
    hits[i].v = hit ? isect.v : 0.0f;
    hits[i].prim = hit ? isect.prim_id : 0xffffffffu;
  }
}

// ---------------------------------------------------------------- shading
// Every Intersection field the reference's Traverse fills (through
// BuildIntersection) for each ray: t/u/v/prim in hits, subface_id, and the
// 80-byte record {position, f0, normal, f1, tangent, f2, binormal, f3,
// d0..d3} (the product's srt_isect; zero on a miss).  Geometric and shading
// normals are equal in all three accels; normal here is Intersection::normal.
struct IsectRec {
  float position[3];
  uint32_t f0;
  float normal[3];
  uint32_t f1;
  float tangent[3];
  uint32_t f2;
  float binormal[3];
  uint32_t f3;
  float d[4];
};

namespace {
template <typename Accel>
void trace_isect(const Accel &acc, int kind, const RayRec *rays, size_t n,
                 const float *prev_normals, HitRec *hits, uint32_t *subface,
                 IsectRec *rec, int nthreads) {
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads)
  for (long long i = 0; i < (long long)n; i++) {
    Ray ray = make_ray(rays[i], prev_normals ? &prev_normals[3 * i] : nullptr);
    Intersection isect;
    memset(&isect, 0, sizeof(isect));
    bool hit = acc.Traverse(isect, ray);
    hits[i].t = hit ? isect.t : std::numeric_limits<float>::max();
    hits[i].u = hit ? isect.u : 0.0f;
    hits[i].v = hit ? isect.v : 0.0f;
    hits[i].prim = hit ? isect.prim_id : 0xffffffffu;
    if (subface) subface[i] = hit ? isect.subface_id : 0u;
    IsectRec &r = rec[i];
    memset(&r, 0, sizeof(r));
    if (!hit) continue;
    for (int k = 0; k < 3; k++) {
      r.position[k] = isect.position[k];
      r.normal[k] = isect.normal[k];
      if (kind == 2) {
        r.tangent[k] = isect.tangent[k];
        r.binormal[k] = isect.binormal[k];
      }
    }
    r.f0 = isect.f0;
    r.f1 = isect.f1;
    r.f2 = isect.f2;
    if (kind == 1) {
      r.f3 = isect.f3;
      r.d[0] = isect.d0;
      r.d[1] = isect.d1;
      r.d[2] = isect.d2;
      r.d[3] = isect.d3;
    }
  }
}
}  // namespace

REF_API void ref_tri_trace_isect(void *p, const RayRec *rays, size_t n, HitRec *hits,
                                 IsectRec *rec, int nthreads) {
  trace_isect(static_cast<TriHandle *>(p)->accel, 0, rays, n, nullptr, hits, nullptr, rec,
              nthreads);
}
REF_API void ref_tet_trace_isect(void *p, const RayRec *rays, size_t n, HitRec *hits,
                                 uint32_t *subface, IsectRec *rec, int nthreads) {
  trace_isect(static_cast<TetHandle *>(p)->accel, 1, rays, n, nullptr, hits, subface, rec,
              nthreads);
}
REF_API void ref_sphere_trace_isect(void *p, const RayRec *rays, size_t n,
                                    const float *prev_normals, HitRec *hits, IsectRec *rec,
                                    int nthreads) {
  trace_isect(static_cast<SphereHandle *>(p)->accel, 2, rays, n, prev_normals, hits, nullptr,
              rec, nthreads);
}

// Node record sizes of the reference's Dump() format.
REF_API void ref_node_sizes(size_t out[3]) {
  out[0] = sizeof(TriangleNode);
  out[1] = sizeof(TetraNode);
  out[2] = sizeof(ParticleNode);
}

// ---------------------------------------------------------------- stages
REF_API void ref_morton_points(const float *pts, size_t n, const float bmin[3],
                               const float bmax[3], uint32_t *codes, int simd) {
  real3 mn(bmin[0], bmin[1], bmin[2]), mx(bmax[0], bmax[1], bmax[2]);
  if (simd)
    CalculateMortonCodes30SIMD(codes, pts, mn, mx, 0, (int64_t)n);
  else
    CalculateMortonCodes30(codes, pts, mn, mx, 0, (int64_t)n);
}

REF_API void ref_morton_tris(const float *v, const uint32_t *f, size_t n,
                             const float bmin[3], const float bmax[3],
                             uint32_t *codes) {
  real3 mn(bmin[0], bmin[1], bmin[2]), mx(bmax[0], bmax[1], bmax[2]);
  CalculateMortonCodesTriangleFloat30(codes, v, f, mn, mx, 0, (int64_t)n);
}

REF_API void ref_morton_tets(const float *v, const uint32_t *f, size_t n,
                             const float bmin[3], const float bmax[3],
                             uint32_t *codes) {
  real3 mn(bmin[0], bmin[1], bmin[2]), mx(bmax[0], bmax[1], bmax[2]);
  CalculateMortonCodesTetraFloat30(codes, v, f, mn, mx, 0, (int64_t)n);
}

REF_API uint32_t ref_morton_code(const float p[3], const float bmin[3],
                                 float inv) {
  real3 pp(p[0], p[1], p[2]), mn(bmin[0], bmin[1], bmin[2]);
  return MortionCode30(pp, mn, inv, inv, inv);
}

// RadixSort30OMP on (code, index) pairs (n >= 1024 to stay on the radix path).
REF_API void ref_radix_sort(uint32_t *code, uint32_t *index, size_t n) {
  std::vector<IndexKey30> keys(n);
  for (size_t i = 0; i < n; i++) {
    keys[i].index = index[i];
    keys[i].code = code[i];
  }
  RadixSort30OMP(keys.data(), keys.data() + n);
  for (size_t i = 0; i < n; i++) {
    index[i] = keys[i].index;
    code[i] = keys[i].code;
  }
}

REF_API void ref_karras(const uint32_t *code, size_t n, uint32_t *child,
                        uint8_t *ltype, uint8_t *rtype) {
  std::vector<IndexKey30> keys(n);
  for (size_t i = 0; i < n; i++) {
    keys[i].index = (uint32_t)i;
    keys[i].code = code[i];
  }
  for (long long i = 0; i < (long long)n - 1; i++) {
    NodeInfo32 info = ConstructBinaryRadixTree30(keys.data(), (int)i, (uint32_t)n);
    child[i] = info.childIndex;
    ltype[i] = info.leftType == NODE_TYPE_LEAF ? 1 : 0;
    rtype[i] = info.rightType == NODE_TYPE_LEAF ? 1 : 0;
  }
}

REF_API void ref_tex3d(const float *img, int w, int h, int d, int comps,
                       const float *uvw, size_t m, int clamp_s, int clamp_t,
                       int clamp_r, float *rgba) {
  Texture3D tex;
  memset(&tex, 0, sizeof(tex));
  tex.image = reinterpret_cast<unsigned char *>(const_cast<float *>(img));
  tex.width = w;
  tex.height = h;
  tex.depth = d;
  tex.components = comps;
  tex.data_type = LSGL_RENDER_TEXTURE3D_FORMAT_FLOAT;
  for (size_t i = 0; i < m; i++)
    FilterTexture3DFloat(&rgba[4 * i], &tex, uvw[3 * i], uvw[3 * i + 1],
                         uvw[3 * i + 2], clamp_s != 0, clamp_t != 0,
                         clamp_r != 0);
}

// The reference tests' fixture draws (test/cctest/test-prefix-tree.cc:10-23).
REF_API void ref_tinymt64_doubles(uint64_t seed, uint32_t mat1, uint32_t mat2,
                                  uint64_t tmat, size_t n, double *out) {
  tinymt64_t rng;
  rng.mat1 = mat1;
  rng.mat2 = mat2;
  rng.tmat = tmat;
  tinymt64_init(&rng, seed);
  for (size_t i = 0; i < n; i++) out[i] = tinymt64_generate_double(&rng);
}

// Camera::buildFrame (render/render_camera.cc:17-63): out = corner, u, v.
REF_API void ref_camera_frame(const float eye[3], const float lookat[3], const float up[3],
                              float fov, int ortho, int width, int height, float out[9]) {
  Camera cam(real3(eye[0], eye[1], eye[2]), real3(lookat[0], lookat[1], lookat[2]),
             real3(up[0], up[1], up[2]), fov, ortho != 0);
  real3 corner, u, v;
  cam.buildFrame(corner, u, v, width, height);
  for (int k = 0; k < 3; k++) {
    out[k] = corner[k];
    out[3 + k] = u[k];
    out[6 + k] = v[k];
  }
}

// Camera::generateStereoEnvRay (render/render_camera.cc:65-118) of the
// stereo camera (render/render_camera.h:44-60): out = org[3], dir[3].
REF_API void ref_stereo_env_ray(const float eye[3], const float lookat[3], const float up[3],
                                float zero_parallax, float eye_separation, float image_u,
                                float image_v, int width, int height, float out[6]) {
  Camera cam(real3(eye[0], eye[1], eye[2]), real3(lookat[0], lookat[1], lookat[2]),
             real3(up[0], up[1], up[2]), zero_parallax, eye_separation);
  real3 org, dir;
  cam.generateStereoEnvRay(org, dir, image_u, image_v, width, height);
  for (int k = 0; k < 3; k++) {
    out[k] = org[k];
    out[3 + k] = dir[k];
  }
}

// BVHTree (render/render_bvh_tree.cc), the top-level tree of RenderGraph.
REF_API void *ref_bvh_build(const double *bmin, const double *bmax, const uint32_t *ids,
                            size_t n) {
  BVHTree *t = new BVHTree();
  for (size_t i = 0; i < n; i++) {
    BVHData d;
    for (int k = 0; k < 3; k++) {
      d.bmin[k] = bmin[3 * i + k];
      d.bmax[k] = bmax[3 * i + k];
    }
    d.nodeID = ids[i];
    t->AddNode(d);
  }
  t->BuildTree();
  return t;
}

REF_API void ref_bvh_free(void *p) { delete static_cast<BVHTree *>(p); }

// Node array: per node bmin[3], bmax[3] (doubles) and child0, child1, axis,
// isLeaf, nodeID (ints).  Returns the node count (arrays sized by the caller).
REF_API size_t ref_bvh_nodes(void *p, double *boxes, int32_t *ints, size_t cap) {
  const std::vector<BVHNode> &nt = static_cast<BVHTree *>(p)->GetNodesTree();
  for (size_t i = 0; i < nt.size() && i < cap; i++) {
    for (int k = 0; k < 3; k++) {
      boxes[6 * i + k] = nt[i].bmin[k];
      boxes[6 * i + 3 + k] = nt[i].bmax[k];
    }
    ints[5 * i + 0] = nt[i].child[0];
    ints[5 * i + 1] = nt[i].child[1];
    ints[5 * i + 2] = nt[i].axis;
    ints[5 * i + 3] = nt[i].isLeaf ? 1 : 0;
    ints[5 * i + 4] = (int32_t)nt[i].nodeID;
  }
  return nt.size();
}

// Sorted candidate list of one ray: (tMin, tMax) pairs and node ids.
REF_API size_t ref_bvh_trace(void *p, const double org[3], const double dir[3],
                             double *tminmax, uint32_t *ids, size_t cap) {
  StackVector<BVHNodeIntersection, 32> isects;
  double o[3] = {org[0], org[1], org[2]}, d[3] = {dir[0], dir[1], dir[2]};
  static_cast<BVHTree *>(p)->Trace(isects, o, d, (std::numeric_limits<double>::max)());
  size_t n = isects->size();
  for (size_t i = 0; i < n && i < cap; i++) {
    tminmax[2 * i] = isects[i].tMin;
    tminmax[2 * i + 1] = isects[i].tMax;
    ids[i] = isects[i].nodeID;
  }
  return n;
}

// Matrixd::Inverse of a row-major 4x4 (render/render_matrix.h), in place.
REF_API void ref_matrix_inverse(double *m16) {
  double m[4][4];
  for (int r = 0; r < 4; r++)
    for (int c = 0; c < 4; c++) m[r][c] = m16[4 * r + c];
  Matrixd::Inverse(m);
  for (int r = 0; r < 4; r++)
    for (int c = 0; c < 4; c++) m16[4 * r + c] = m[r][c];
}

// Texture::Fetch of a dense 3D texture (gles/gles_common.h:371-399): the
// per-axis remap of local::remap (gles/gles_common.h:264-269, written out
// here because that header needs the GL front end) and the reference's own
// FilterTexture3D{Byte,Float,Double}.  fmt: 0 byte, 1 float, 2 double.
REF_API void ref_tex_fetch(int fmt, const void *img, int w, int h, int d, int comps,
                           const int *clamp, const float *remap0, int n0, const float *remap1,
                           int n1, const float *remap2, int n2, const float *uvw, size_t m,
                           float *rgba) {
  Texture3D tex;
  memset(&tex, 0, sizeof(tex));
  tex.image = reinterpret_cast<unsigned char *>(const_cast<void *>(img));
  tex.width = w;
  tex.height = h;
  tex.depth = d;
  tex.components = comps;
  const float *tab[3] = {remap0, remap1, remap2};
  const int nt[3] = {n0, n1, n2};
  for (size_t i = 0; i < m; i++) {
    float c[3];
    for (int k = 0; k < 3; k++) {
      c[k] = uvw[3 * i + k];
      if (tab[k] && nt[k] > 0) {
        int idx = c[k] * nt[k];
        idx = (std::max)((std::min)(nt[k] - 1, idx), 0);
        c[k] = tab[k][idx];
      }
    }
    if (fmt == 0)
      FilterTexture3DByte(&rgba[4 * i], &tex, c[0], c[1], c[2], clamp[0] != 0, clamp[1] != 0,
                          clamp[2] != 0);
    else if (fmt == 1)
      FilterTexture3DFloat(&rgba[4 * i], &tex, c[0], c[1], c[2], clamp[0] != 0, clamp[1] != 0,
                           clamp[2] != 0);
    else
      FilterTexture3DDouble(&rgba[4 * i], &tex, c[0], c[1], c[2], clamp[0] != 0, clamp[1] != 0,
                            clamp[2] != 0);
  }
}

// Texture::Fetch of a sparse volume (gles/gles_common.h:344-369) through the
// reference's SparseVolumeAccel.  Blocks: offset[3], extent[3], size[3],
// level, then a 64-bit byte offset into the data pool (8 ints + 8 bytes).
REF_API void ref_sparse_fetch(const int32_t *blocks, size_t nblocks, const unsigned char *pool,
                              int fmt, int comps, const int *gdim, const float *uvw, size_t m,
                              float *rgba) {
  SparseVolume sv;
  for (size_t i = 0; i < nblocks; i++) {
    const int32_t *b = blocks + 12 * i;
    VolumeBlock vb;
    memset(&vb, 0, sizeof(vb));
    for (int k = 0; k < 3; k++) {
      vb.offset[k] = b[k];
      vb.extent[k] = b[3 + k];
      vb.size[k] = b[6 + k];
    }
    vb.level = b[9];
    vb.id = (int)i;
    uint64_t off;
    memcpy(&off, b + 10, 8);
    vb.data = pool + off;
    sv.blocks.push_back(vb);
  }
  for (int k = 0; k < 3; k++) sv.globalDim[k] = gdim[k];
  sv.components = comps;
  sv.format = fmt == 0 ? LSGL_RENDER_TEXTURE3D_FORMAT_BYTE
                       : fmt == 1 ? LSGL_RENDER_TEXTURE3D_FORMAT_FLOAT
                                  : LSGL_RENDER_TEXTURE3D_FORMAT_DOUBLE;
  sv.maxLevel = 0;
  SparseVolumeAccel acc;
  acc.Build(&sv);
  for (size_t i = 0; i < m; i++) {
    double value[4], position[3];
    for (int k = 0; k < 3; k++) position[k] = uvw[3 * i + k] * sv.globalDim[k];
    acc.Sample(value, position);
    for (int k = 0; k < 4; k++) rgba[4 * i + k] = value[k];
  }
}

// ---------------------------------------------------------------- lines
// LineAccel (render/render_accel_line.cc): spatial-median BVH over capped
// cylinders (Build), closest hit (Traverse), its Intersection's normal.
struct LineHandle {
  Lines lines;
  LineAccel accel;
};

REF_API void *ref_line_build(const float *pos, const float *radius, float const_radius,
                             const uint32_t *segments, size_t nlines, int min_leaf,
                             int max_depth, int cap) {
  LineHandle *h = new LineHandle();
  memset(&h->lines, 0, sizeof(h->lines));
  h->lines.numLines = nlines;
  h->lines.positions = pos;
  h->lines.dpositions = nullptr;
  h->lines.isDoublePrecisionPos = false;
  h->lines.radius = radius;
  h->lines.constantRadius = const_radius;
  h->lines.segments = const_cast<uint32_t *>(segments);
  LineBuildOptions opt;
  if (min_leaf > 0) opt.minLeafPrimitives = min_leaf;
  if (max_depth > 0) opt.maxTreeDepth = max_depth;
  opt.cap = cap != 0;
  {
    QuietStdout q;
    h->accel.Build(&h->lines, opt);
  }
  return h;
}

REF_API void ref_line_free(void *p) { delete static_cast<LineHandle *>(p); }

REF_API int ref_line_dump(void *p, const char *path) {
  return static_cast<LineHandle *>(p)->accel.Dump(path) ? 0 : 1;
}

REF_API void ref_line_bbox(void *p, double bmin[3], double bmax[3]) {
  static_cast<LineHandle *>(p)->accel.BoundingBox(bmin, bmax);
}

REF_API void ref_line_trace(void *p, const RayRec *rays, size_t n, HitRec *hits,
                            float *normals, int nthreads, int chunk) {
  const LineAccel &acc = static_cast<LineHandle *>(p)->accel;
  if (nthreads <= 0) nthreads = omp_get_max_threads();
  if (chunk <= 0) chunk = 64;
#pragma omp parallel for schedule(dynamic, chunk) num_threads(nthreads)
  for (long long i = 0; i < (long long)n; i++) {
    Ray ray = make_ray(rays[i], nullptr);
    Intersection isect;
    bool hit = acc.Traverse(isect, ray);
    hits[i].t = hit ? isect.t : std::numeric_limits<float>::max();
    hits[i].u = hit ? isect.u : 0.0f;
    hits[i].v = hit ? isect.v : 0.0f;
    hits[i].prim = hit ? isect.prim_id : 0xffffffffu;
    if (normals)
      for (int k = 0; k < 3; k++) normals[3 * i + k] = hit ? isect.normal[k] : 0.0f;
  }
}

// ---------------------------------------------------------------- solids
// SolidAccel (render/render_accel_solid.cc): Build32 (its SAH Build below
// 1024 solids), Traverse with its Intersection's t, position and normal
// (u and v are left unset by the reference's solid tests: reported as 0).
struct SolidHandle {
  Solid solids;
  SolidAccel accel;
};

REF_API void *ref_solid_build(int nv, const float *verts, const uint32_t *indices, size_t n) {
  SolidHandle *h = new SolidHandle();
  memset(&h->solids, 0, sizeof(h->solids));
  h->solids.numVertsPerSolid = nv;
  h->solids.numSolids = n;
  h->solids.vertices = verts;
  h->solids.dvertices = nullptr;
  h->solids.isDoublePrecisionPos = false;
  h->solids.indices = const_cast<uint32_t *>(indices);
  SolidBuildOptions opt;
  {
    QuietStdout q;
    h->accel.Build32(&h->solids, opt);
  }
  return h;
}

// SolidAccel::Build (binned SAH) at every size; dverts non-null: double
// positions.
REF_API void *ref_solid_build_sah(int nv, const float *verts, const double *dverts,
                                  const uint32_t *indices, size_t n) {
  SolidHandle *h = new SolidHandle();
  memset(&h->solids, 0, sizeof(h->solids));
  h->solids.numVertsPerSolid = nv;
  h->solids.numSolids = n;
  h->solids.vertices = verts;
  h->solids.dvertices = dverts;
  h->solids.isDoublePrecisionPos = dverts != nullptr;
  h->solids.indices = const_cast<uint32_t *>(indices);
  SolidBuildOptions opt;
  {
    QuietStdout q;
    h->accel.Build(&h->solids, opt);
  }
  return h;
}

// The same with double-precision positions (Solid::dvertices).
REF_API void *ref_solid_build_d(int nv, const double *dverts, const uint32_t *indices, size_t n) {
  SolidHandle *h = new SolidHandle();
  memset(&h->solids, 0, sizeof(h->solids));
  h->solids.numVertsPerSolid = nv;
  h->solids.numSolids = n;
  h->solids.vertices = nullptr;
  h->solids.dvertices = dverts;
  h->solids.isDoublePrecisionPos = true;
  h->solids.indices = const_cast<uint32_t *>(indices);
  SolidBuildOptions opt;
  {
    QuietStdout q;
    h->accel.Build32(&h->solids, opt);
  }
  return h;
}

REF_API void ref_solid_free(void *p) { delete static_cast<SolidHandle *>(p); }

REF_API int ref_solid_dump(void *p, const char *path) {
  return static_cast<SolidHandle *>(p)->accel.Dump(path) ? 0 : 1;
}

REF_API void ref_solid_bbox(void *p, double bmin[3], double bmax[3]) {
  static_cast<SolidHandle *>(p)->accel.BoundingBox(bmin, bmax);
}

REF_API void ref_solid_trace(void *p, const RayRec *rays, size_t n, HitRec *hits,
                             float *normals, float *positions, int nthreads, int chunk) {
  const SolidAccel &acc = static_cast<SolidHandle *>(p)->accel;
  if (nthreads <= 0) nthreads = omp_get_max_threads();
  if (chunk <= 0) chunk = 64;
#pragma omp parallel for schedule(dynamic, chunk) num_threads(nthreads)
  for (long long i = 0; i < (long long)n; i++) {
    Ray ray = make_ray(rays[i], nullptr);
    Intersection isect;
    bool hit = acc.Traverse(isect, ray);
    hits[i].t = hit ? isect.t : std::numeric_limits<float>::max();
    hits[i].u = 0.0f;
    hits[i].v = 0.0f;
    hits[i].prim = hit ? isect.prim_id : 0xffffffffu;
    for (int k = 0; k < 3; k++) {
      if (normals) normals[3 * i + k] = hit ? isect.normal[k] : 0.0f;
      if (positions) positions[3 * i + k] = hit ? isect.position[k] : 0.0f;
    }
  }
}
