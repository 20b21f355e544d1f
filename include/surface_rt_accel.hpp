/*
 * surface_rt_accel.hpp -- C++ drop-ins for SURFACE's TriangleAccel, TetraAccel
 * and ParticleAccel over the C ABI of surface_rt.h.
 *
 * Header-only.  Compiled inside the SURFACE tree (it includes the reference's
 * render/ headers for Mesh, Tetrahedron, Particles, Ray and Intersection):
 *
 *   g++ -I<SURFACE>/render -I<this repo>/include ... -L<this repo>/surface_b200
 *       -lsurface_rt
 *
 * GpuTriangleAccel / GpuTetraAccel / GpuParticleAccel keep the members the
 * reference's accels expose to AccelBuilder and RenderGraph
 * (render/render_accel_triangle.h:69-105, render/render_accel_tetra.h:82-125,
 * render/render_accel_particle.h:68-110): Build32, Traverse, BoundingBox and
 * Dump, with the same meaning.  Traverse fills every Intersection field the
 * reference's Traverse fills, through its BuildIntersection: t, u, v,
 * prim_id, subface_id (tetrahedra), position, geometric, normal, tangent and
 * binormal (spheres), f0..f3 and d0..d3 (tetrahedra); other fields are left
 * as they were, as in the reference.  A miss sets t = FLT_MAX, u = v = 0,
 * prim_id = ~0 and returns false.
 *
 * Traverse handles one ray per call and serialises its callers (the
 * reference calls it from OpenMP threads); TraverseBatch traces a whole
 * array of rays in one GPU pass and is the form to use for a frame.
 * Input arrays are borrowed, as in the reference: the mesh must stay alive
 * and unchanged while the accel is used.  Double-precision positions
 * (isDoublePrecisionPos) are not supported: Build32 returns false.
 */
#ifndef SURFACE_RT_ACCEL_HPP_
#define SURFACE_RT_ACCEL_HPP_

#include <float.h>
#include <string.h>

#include <mutex>
#include <vector>

#include "render_accel_particle.h"
#include "render_accel_tetra.h"
#include "render_accel_triangle.h"
#include "surface_rt.h"

namespace lsgl {
namespace render {

namespace srt_shim {

// One context per process on device 0 (the accels share its stream).
inline srt_ctx *context() {
  static srt_ctx *ctx = [] {
    srt_ctx *c = nullptr;
    if (srt_ctx_create(0, &c) != SRT_OK) c = nullptr;
    return c;
  }();
  return ctx;
}

inline srt_ray to_srt(const Ray &ray) {
  srt_ray r;
  const real3 &o = ray.origin(), &d = ray.direction();
  r.org[0] = o[0];
  r.org[1] = o[1];
  r.org[2] = o[2];
  r.prev_prim = ray.prev_prim_id;
  r.dir[0] = d[0];
  r.dir[1] = d[1];
  r.dir[2] = d[2];
  r.prev_t = (float)ray.prev_hit_t;  // filled from a float by the reference
  return r;
}

// Copy one result into an Intersection the way the reference's Traverse and
// BuildIntersection write it; returns whether the ray hit.
inline bool fill(Intersection &is, const srt_hit &h, const srt_isect &r, uint32_t subface,
                 srt_kind kind) {
  is.t = h.t;
  is.u = h.u;
  is.v = h.v;
  is.prim_id = h.prim;
  if (h.prim == SRT_MISS) {
    is.t = FLT_MAX;
    is.u = 0.0f;
    is.v = 0.0f;
    return false;
  }
  if (kind == SRT_TETRAHEDRA) is.subface_id = subface;
  is.position = real3(r.position[0], r.position[1], r.position[2]);
  is.normal = real3(r.normal[0], r.normal[1], r.normal[2]);
  is.geometric = is.normal;
  if (kind == SRT_SPHERES) {
    is.tangent = real3(r.tangent[0], r.tangent[1], r.tangent[2]);
    is.binormal = real3(r.binormal[0], r.binormal[1], r.binormal[2]);
  }
  is.f0 = r.f0;
  is.f1 = r.f1;
  is.f2 = r.f2;
  if (kind == SRT_TETRAHEDRA) {
    is.f3 = r.f3;
    is.d0 = r.d[0];
    is.d1 = r.d[1];
    is.d2 = r.d[2];
    is.d3 = r.d[3];
  }
  return true;
}

// Shared part of the three accels: one srt_accel plus the trace calls.
class Base {
 public:
  explicit Base(srt_kind kind) : kind_(kind) {
    if (context()) srt_accel_create(context(), kind, &acc_);
  }
  ~Base() {
    if (acc_) srt_accel_destroy(acc_);
  }
  Base(const Base &) = delete;
  Base &operator=(const Base &) = delete;

  /// Closest hits of n rays in one GPU pass; hit[i] (optional) = whether ray
  /// i hit.  Returns false when the library reports an error.
  bool TraverseBatch(Intersection *isects, const Ray *rays, size_t n,
                     bool *hit = nullptr) const {
    if (!acc_) return false;
    std::vector<srt_ray> r(n);
    std::vector<float> pn(kind_ == SRT_SPHERES ? 3 * n : 0);
    for (size_t i = 0; i < n; i++) {
      r[i] = to_srt(rays[i]);
      if (kind_ == SRT_SPHERES)
        for (int k = 0; k < 3; k++) pn[3 * i + k] = rays[i].prev_hit_normal[k];
    }
    std::vector<srt_hit> h(n);
    std::vector<srt_isect> rec(n);
    std::vector<uint32_t> sub(kind_ == SRT_TETRAHEDRA ? n : 0);
    srt_trace_opts o;
    memset(&o, 0, sizeof(o));
    o.prev_normals = kind_ == SRT_SPHERES ? pn.data() : nullptr;
    o.subface = kind_ == SRT_TETRAHEDRA ? sub.data() : nullptr;
    o.isect = rec.data();
    if (srt_trace_closest(acc_, r.data(), n, h.data(), &o) != SRT_OK) return false;
    for (size_t i = 0; i < n; i++) {
      const bool ok = fill(isects[i], h[i], rec[i], kind_ == SRT_TETRAHEDRA ? sub[i] : 0u,
                           kind_);
      if (hit) hit[i] = ok;
    }
    return true;
  }

  /// One ray (the reference's call shape); serialised across threads.
  bool Traverse(Intersection &isect, Ray &ray) const {
    std::lock_guard<std::mutex> lock(mu_);
    bool h = false;
    if (!TraverseBatch(&isect, &ray, 1, &h)) return false;
    return h;
  }

  void BoundingBox(double bmin[3], double bmax[3]) const {
    if (acc_) srt_accel_bbox(acc_, bmin, bmax);
  }

  bool Dump(const char *filename) { return acc_ && srt_accel_dump(acc_, filename) == SRT_OK; }

  srt_accel *handle() const { return acc_; }

 protected:
  srt_kind kind_;
  srt_accel *acc_ = nullptr;
  mutable std::mutex mu_;
};

}  // namespace srt_shim

/// TriangleAccel (render/render_accel_triangle.h:69-105) on the GPU.
class GpuTriangleAccel : public srt_shim::Base {
 public:
  GpuTriangleAccel() : Base(SRT_TRIANGLES) {}
  bool Build32(const Mesh *mesh, const TriangleBuildOptions &) {
    if (!acc_ || !mesh || mesh->isDoublePrecisionPos) return false;
    mesh_ = mesh;  // borrowed, as the reference's mesh_
    return srt_accel_build_triangles(acc_, mesh->vertices, mesh->nvertices, mesh->faces,
                                     mesh->nfaces) == SRT_OK &&
           srt_ctx_synchronize(srt_shim::context()) == SRT_OK;
  }

 private:
  const Mesh *mesh_ = nullptr;
};

/// TetraAccel (render/render_accel_tetra.h:82-125) on the GPU.
class GpuTetraAccel : public srt_shim::Base {
 public:
  GpuTetraAccel() : Base(SRT_TETRAHEDRA) {}
  bool Build32(const Tetrahedron *tets, const TetraBuildOptions &) {
    if (!acc_ || !tets) return false;
    // the vertex count is not stored in Tetrahedron: one past the largest id
    size_t nv = 0;
    for (size_t i = 0; i < 4 * (size_t)tets->numTetrahedrons; i++)
      if (tets->faces[i] + 1 > nv) nv = tets->faces[i] + 1;
    tets_ = tets;
    // double-precision positions (dvertices) keep their precision
    const srt_status s =
        tets->isDoublePrecisionPos
            ? srt_accel_build_tetrahedra_double(acc_, tets->dvertices, nv, tets->faces,
                                                tets->numTetrahedrons)
            : srt_accel_build_tetrahedra(acc_, tets->vertices, nv, tets->faces,
                                         tets->numTetrahedrons);
    return s == SRT_OK && srt_ctx_synchronize(srt_shim::context()) == SRT_OK;
  }

 private:
  const Tetrahedron *tets_ = nullptr;
};

/// ParticleAccel (render/render_accel_particle.h:68-110) on the GPU.
class GpuParticleAccel : public srt_shim::Base {
 public:
  GpuParticleAccel() : Base(SRT_SPHERES) {}
  bool Build32(const Particles *parts, const ParticleBuildOptions &) {
    if (!acc_ || !parts || parts->isDoublePrecisionPos) return false;
    parts_ = parts;
    return srt_accel_build_spheres(acc_, parts->positions, parts->radius,
                                   (float)parts->constantRadius, parts->numParticles) == SRT_OK &&
           srt_ctx_synchronize(srt_shim::context()) == SRT_OK;
  }

 private:
  const Particles *parts_ = nullptr;
};

}  // namespace render
}  // namespace lsgl

#endif  // SURFACE_RT_ACCEL_HPP_
