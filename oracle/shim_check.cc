// shim_check.cc -- TEST INFRASTRUCTURE ONLY.  Drives the C++ drop-in accels of
// include/surface_rt_accel.hpp (GpuTriangleAccel, GpuTetraAccel,
// GpuParticleAccel) and the reference's own TriangleAccel / TetraAccel /
// ParticleAccel (from oracle/_ref/libsurface_ref.so) on the same primitives
// and rays, and writes every Intersection field each of them leaves, so the
// tests can compare the two field by field.  Built by oracle/Makefile against
// the reference's render/ headers; loaded only by tests/.
#include <stdint.h>
#include <string.h>

#include <vector>

#include "surface_rt_accel.hpp"

using namespace lsgl::render;

#define CHECK_API extern "C" __attribute__((visibility("default")))

namespace {

struct RayRec {
  float org[3];
  uint32_t prev_prim;
  float dir[3];
  float prev_t;
};

// Every Intersection field (148 bytes), including the ones a Traverse leaves
// untouched: both sides start from the same byte pattern.
struct FullRec {
  uint32_t hit;
  float t, u, v;
  uint32_t prim, subface;
  float position[3], geometric[3], normal[3], tangent[3], binormal[3];
  uint32_t f[8];
  float d[8];
};

Ray make_ray(const RayRec &r, const float *pn) {
  real3 o(r.org[0], r.org[1], r.org[2]);
  real3 d(r.dir[0], r.dir[1], r.dir[2]);
  Ray ray(o, d);
  ray.prev_prim_id = r.prev_prim;
  ray.prev_hit_t = r.prev_t;
  ray.prev_hit_normal = pn ? real3(pn[0], pn[1], pn[2]) : real3(0.0f, 0.0f, 0.0f);
  ray.prev_node = nullptr;
  return ray;
}

void blank(Intersection &is) { memset(&is, 0x5a, sizeof(is)); }

void record(const Intersection &is, bool hit, FullRec &o) {
  o.hit = hit ? 1u : 0u;
  o.t = is.t;
  o.u = is.u;
  o.v = is.v;
  o.prim = is.prim_id;
  o.subface = is.subface_id;
  for (int k = 0; k < 3; k++) {
    o.position[k] = is.position[k];
    o.geometric[k] = is.geometric[k];
    o.normal[k] = is.normal[k];
    o.tangent[k] = is.tangent[k];
    o.binormal[k] = is.binormal[k];
  }
  const unsigned int f[8] = {is.f0, is.f1, is.f2, is.f3, is.f4, is.f5, is.f6, is.f7};
  const float d[8] = {is.d0, is.d1, is.d2, is.d3, is.d4, is.d5, is.d6, is.d7};
  for (int k = 0; k < 8; k++) {
    o.f[k] = f[k];
    o.d[k] = d[k];
  }
}

// mode 0: the reference's Traverse per ray; 1: the drop-in's per-ray
// Traverse; 2: the drop-in's TraverseBatch over all rays.
template <typename Ref, typename Gpu>
int run(Ref &ref, Gpu &gpu, const RayRec *rays, const float *pn, size_t n, int mode,
        FullRec *out) {
  std::vector<Ray> rs;
  rs.reserve(n);
  for (size_t i = 0; i < n; i++) rs.push_back(make_ray(rays[i], pn ? pn + 3 * i : nullptr));
  if (mode == 2) {
    std::vector<Intersection> is(n);
    for (size_t i = 0; i < n; i++) blank(is[i]);
    std::vector<char> hit(n);
    bool *hb = reinterpret_cast<bool *>(hit.data());
    if (!gpu.TraverseBatch(is.data(), rs.data(), n, hb)) return 1;
    for (size_t i = 0; i < n; i++) record(is[i], hb[i], out[i]);
    return 0;
  }
  for (size_t i = 0; i < n; i++) {
    Intersection is;
    blank(is);
    const bool h = mode == 0 ? ref.Traverse(is, rs[i]) : gpu.Traverse(is, rs[i]);
    record(is, h, out[i]);
  }
  return 0;
}

}  // namespace

CHECK_API size_t shim_record_bytes() { return sizeof(FullRec); }

// Build both accels over the same triangles and trace; returns 0 on success.
CHECK_API int shim_check_triangles(const float *verts, size_t nverts, const uint32_t *faces,
                                   size_t nfaces, const RayRec *rays, size_t n, int mode,
                                   FullRec *out) {
  Mesh mesh;
  mesh.nvertices = nverts;
  mesh.vertices = verts;
  mesh.nfaces = nfaces;
  mesh.faces = const_cast<uint32_t *>(faces);
  mesh.isDoublePrecisionPos = false;
  TriangleBuildOptions opt;
  TriangleAccel ref;
  GpuTriangleAccel gpu;
  int rc = 0;
  if (mode == 0)
    ref.Build32(&mesh, opt);
  else if (!gpu.Build32(&mesh, opt))
    rc = 2;
  if (rc == 0) rc = run(ref, gpu, rays, nullptr, n, mode, out);
  // the arrays are the caller's; keep Mesh's destructor from freeing them
  mesh.vertices = nullptr;
  mesh.faces = nullptr;
  mesh.normals = nullptr;
  mesh.dvertices = nullptr;
  return rc;
}

CHECK_API int shim_check_tetrahedra(const float *verts, const uint32_t *tets, size_t ntets,
                                    const RayRec *rays, size_t n, int mode, FullRec *out) {
  Tetrahedron t;
  memset(&t, 0, sizeof(t));
  t.numTetrahedrons = ntets;
  t.vertices = verts;
  t.faces = const_cast<uint32_t *>(tets);
  t.isDoublePrecisionPos = false;
  TetraBuildOptions opt;
  TetraAccel ref;
  GpuTetraAccel gpu;
  if (mode == 0)
    ref.Build32(&t, opt);
  else if (!gpu.Build32(&t, opt))
    return 2;
  return run(ref, gpu, rays, nullptr, n, mode, out);
}

CHECK_API int shim_check_spheres(const float *pos, const float *radius, size_t np,
                                 const RayRec *rays, const float *prev_normals, size_t n,
                                 int mode, FullRec *out) {
  Particles p;
  memset(&p, 0, sizeof(p));
  p.numParticles = np;
  p.positions = pos;
  p.isDoublePrecisionPos = false;
  p.radius = const_cast<float *>(radius);
  p.constantRadius = 0.0f;
  ParticleBuildOptions opt;
  ParticleAccel ref;
  GpuParticleAccel gpu;
  if (mode == 0)
    ref.Build32(&p, opt);
  else if (!gpu.Build32(&p, opt))
    return 2;
  return run(ref, gpu, rays, prev_normals, n, mode, out);
}
