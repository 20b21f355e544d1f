/*
 * surface_rt.h -- C ABI of the B200 ray-tracing core (libsurface_rt.so).
 *
 * A drop-in for SURFACE's render/ accel classes and the ray-dispatch calls the
 * GLES layer makes into them.  Plain pointers and sizes only.  Every entry
 * point returns srt_status (SRT_OK = 0).
 *
 * Pointers passed as primitive data, rays or hits may be host or device
 * memory; the library inspects each one (cudaPointerGetAttributes) and copies
 * host data through its own device buffers.  Device pointers are used in
 * place and must stay valid until the call's work has completed on the
 * context's stream (srt_ctx_synchronize).
 *
 * Reference interface each group replaces (paths relative to the SURFACE tree):
 *   srt_build_*            XxxAccel::Build32          render/render_accel_triangle.h:79,
 *                                                     render/render_accel_tetra.h:88,
 *                                                     render/render_accel_particle.h:86
 *                          called from AccelBuilder   gles/gles_accel_builder.cc:572,673,867
 *   srt_trace_closest      XxxAccel::Traverse         render/render_accel_triangle.h:88,
 *                                                     render/render_accel_tetra.h:97,
 *                                                     render/render_accel_particle.h:95
 *                          called per ray from        gles/gles_render_graph.cc:224-264
 *   srt_accel_bbox         XxxAccel::BoundingBox      render/render_accel_triangle.h:91
 *                          called from                gles/gles_primitive.cc:174,215,271
 *   srt_accel_dump         XxxAccel::Dump             render/render_accel_triangle.cc:1692-1719
 *   srt_volume_march_*     the shader ray march       examples/nonuniform_volume_render/input.frag:99-141
 *                          + Texture::Fetch           gles/gles_common.h:344-403
 *                          -> FilterTexture3DFloat    render/render_texture.cc:946
 *   srt_stage_*            the build's inner steps    render/render_prefix_tree_util.h:143,296,
 *                                                     render/render_prefix_tree_util.cc:230,267,562
 */
#ifndef SURFACE_RT_H_
#define SURFACE_RT_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define SRT_API __attribute__((visibility("default")))
#else
#define SRT_API
#endif

typedef enum {
  SRT_OK = 0,
  SRT_ERR_INVALID = 1,     /* bad argument (NULL, size out of range, kind) */
  SRT_ERR_CUDA = 2,        /* CUDA runtime error (see srt_last_error) */
  SRT_ERR_NO_MEMORY = 3,   /* device allocation failed */
  SRT_ERR_LIMIT = 4,       /* a kernel hit a hard limit (stack depth,
                              iteration cap) and stopped that ray */
  SRT_ERR_UNSUPPORTED = 5  /* valid request this build does not handle */
} srt_status;

typedef enum {
  SRT_TRIANGLES = 0,  /* TriangleAccel */
  SRT_TETRAHEDRA = 1, /* TetraAccel */
  SRT_SPHERES = 2     /* ParticleAccel */
} srt_kind;

#define SRT_MISS 0xFFFFFFFFu

/* One ray (32 bytes, 16-byte aligned arrays give vector loads).  prev_prim /
 * prev_t mirror Ray::prev_prim_id / prev_hit_t (render/render_ray.h:121-125):
 * a primary ray has prev_prim = SRT_MISS.  prev_t is the previous hit's
 * distance; the reference stores it as double but fills it from a float
 * (gles/gles_raytrace_engine.cc:482), so float loses nothing. */
typedef struct srt_ray {
  float org[3];
  uint32_t prev_prim;
  float dir[3];
  float prev_t;
} srt_ray;

/* Closest hit (16 bytes): Intersection::t/u/v/prim_id
 * (render/render_intersection.h:18-24).  prim = SRT_MISS on a miss (t then
 * holds FLT_MAX, u = v = 0). */
typedef struct srt_hit {
  float t;
  float u;
  float v;
  uint32_t prim;
} srt_hit;

/* Shading record of a hit (80 bytes): the Intersection fields that the
 * reference's Traverse fills through BuildIntersection besides t/u/v/prim_id
 * and subface_id (render/render_intersection.h:18-62), i.e. what the GLSL
 * fragment stage interpolates varyings from (gles/gles_common.cc:1007-1141).
 *   triangles (render/render_accel_triangle.cc:2439-2507): position =
 *     org + t * dir, normal = normalised (p1 - p0) x (p2 - p0), f0..f2 = the
 *     face's vertex ids; tangent, binormal, f3 and d are 0.
 *   tetrahedra (render/render_accel_tetra.cc:2124-2196): position, normal of
 *     the entering face (face_table of subface_id), f0..f3 = the tet's vertex
 *     ids, d[0..3] = InterpolateTetra's weights (:148-241).
 *   spheres (render/render_accel_particle.cc:2966-3049): position, normal =
 *     vnormalize(position - centre), tangent and binormal of the spherical
 *     parameterisation, f0 = f1 = f2 = prim id; the spherical (u, v) go to
 *     srt_hit.u / .v (as in every sphere trace).
 * Intersection::geometric equals normal for all three.  A miss writes an
 * all-zero record (the reference leaves the fields unset). */
typedef struct srt_isect {
  float position[3];
  uint32_t f0;
  float normal[3];
  uint32_t f1;
  float tangent[3];
  uint32_t f2;
  float binormal[3];
  uint32_t f3;
  float d[4];
} srt_isect;

/* Optional per-call inputs/outputs of srt_trace_closest.  Any field may be
 * NULL / 0. */
typedef struct srt_trace_opts {
  /* spheres: Ray::prev_hit_normal, 3 floats per ray, for the self-hit rule
   * of SphereIsect (render/render_accel_particle.cc:2470-2489) */
  const float *prev_normals;
  /* tetrahedra: Intersection::subface_id per ray (entering face 0..3) */
  uint32_t *subface;
  /* tetrahedra: per-vertex scalar; with scalar_out, the scalar interpolated
   * at the entering point with the entering face's barycentrics */
  const float *vertex_scalar;
  float *scalar_out;
  /* triangles and spheres: geometric normal at the hit (3 floats per ray,
   * as BuildIntersection computes it) */
  float *normal_out;
  /* work counters (device memory, 4 x uint64, accumulated): branch nodes
   * visited, leaves visited, primitive tests -- the reference's
   * TetraTraversalStatistics (render/render_accel_tetra.h:70-78) -- and
   * rays that took the reference's walk */
  unsigned long long *stats;
  /* SRT_TRACE_* bits */
  uint32_t flags;
  /* cap on the steps (nodes popped) of one ray's walk; 0 = the default,
   * 8 * primitives + 64, which a walk over a valid tree never reaches.  A
   * ray that reaches the cap stops with whatever it found so far and the
   * call (or srt_ctx_synchronize) reports SRT_ERR_LIMIT, like the
   * reference's stack-depth assert (render/render_accel_triangle.cc:2661);
   * the context stays usable. */
  uint32_t max_iter;
  /* per-ray shading record (srt_isect), written after the closest hit is
   * known: the reference's BuildIntersection */
  srt_isect *isect;
} srt_trace_opts;

/* srt_trace_opts.flags: walk the tree once in the reference's own order
 * (its Traverse loop step for step) instead of the default walk, which goes
 * front to back and replays the reference's order only to break exact
 * ties.  Both give identical hits; the default does far less work. */
#define SRT_TRACE_SINGLE_PASS 1u
/* Trace the rays in a coherent order (a Morton curve over origin and
 * direction, sorted on the GPU) instead of array order: fewer divergent warps
 * on large ray sets at the cost of the sort.  Hits are identical and are
 * written at each ray's own index. */
#define SRT_TRACE_SORT_RAYS 2u
/* Launch the first traversal pass as one thread per ray over a grid of all
 * rays instead of the default persistent warps (as many blocks as the GPU
 * holds at once, each warp taking 32 rays at a time until none are left).
 * Same hits; the default keeps every SM busy to the end of the launch. */
#define SRT_TRACE_GRID 4u

typedef struct srt_ctx srt_ctx;
typedef struct srt_accel srt_accel;

typedef struct srt_accel_info {
  int32_t kind;          /* srt_kind */
  int32_t node_bytes;    /* bytes per record in srt_accel_export's node dump */
  uint64_t num_prims;
  uint64_t num_nodes;    /* records in the device node array */
  uint64_t num_branches; /* branch nodes of the reference tree */
  uint64_t num_leaves;   /* leaf nodes of the reference tree */
  float scene_min[3];    /* scene box used for the Morton quantisation */
  float scene_max[3];
  double eps_scale;      /* triangles: max scene extent; others 16 */
} srt_accel_info;

/* ---- context ---------------------------------------------------------- */
SRT_API srt_status srt_ctx_create(int device, srt_ctx **out);
SRT_API srt_status srt_ctx_destroy(srt_ctx *ctx);
/* Use `stream` (a cudaStream_t) for all work of this context; NULL = the
 * context's own stream; (void*)1 = cudaStreamLegacy, the legacy default
 * stream (handle 0 in most frameworks). */
SRT_API srt_status srt_ctx_set_stream(srt_ctx *ctx, void *stream);
SRT_API void *srt_ctx_get_stream(srt_ctx *ctx);
/* Wait for all queued work; reports kernel-side limit hits (SRT_ERR_LIMIT)
 * and asynchronous CUDA errors since the last call. */
SRT_API srt_status srt_ctx_synchronize(srt_ctx *ctx);
/* Human-readable text of the last error on this thread. */
SRT_API const char *srt_last_error(void);
/* Number of kernels this context has launched so far. */
SRT_API uint64_t srt_ctx_launch_count(srt_ctx *ctx);

/* ---- acceleration structures ------------------------------------------ */
SRT_API srt_status srt_accel_create(srt_ctx *ctx, srt_kind kind, srt_accel **out);
SRT_API srt_status srt_accel_destroy(srt_accel *accel);

/* (Re)build from nfaces triangles (3 uint32 vertex ids each) over float
 * xyz vertices.  Reuses the accel's device buffers when they are large
 * enough.  Asynchronous on the context stream.  nfaces >= 2, < 2^30. */
SRT_API srt_status srt_accel_build_triangles(srt_accel *accel,
                                             const float *vertices,
                                             size_t nvertices,
                                             const uint32_t *faces,
                                             size_t nfaces);
/* ntets tetrahedra (4 uint32 vertex ids each). */
SRT_API srt_status srt_accel_build_tetrahedra(srt_accel *accel,
                                              const float *vertices,
                                              size_t nvertices,
                                              const uint32_t *tets,
                                              size_t ntets);
/* The same with double-precision positions (Tetrahedron::dvertices,
 * isDoublePrecisionPos; render/render_prim_tetra.h): as the reference's
 * Build32 does, the scene and node boxes pad each double coordinate in
 * double and round to float, the Morton codes use the positions rounded to
 * float, and the Pluecker tests take the doubles
 * (render/render_accel_tetra.cc:1621-1660, 2009-2060).  The shading records
 * (srt_trace_opts.isect) use the positions rounded to float, as
 * BuildIntersection's real3 does (:2135-2150). */
SRT_API srt_status srt_accel_build_tetrahedra_double(srt_accel *accel,
                                                     const double *vertices,
                                                     size_t nvertices,
                                                     const uint32_t *tets,
                                                     size_t ntets);
/* n spheres: xyz centres; radius per sphere, or NULL for constant_radius
 * (Particles::radius / constantRadius, render/render_prim_particle.h:19-27). */
SRT_API srt_status srt_accel_build_spheres(srt_accel *accel,
                                           const float *centers,
                                           const float *radius,
                                           float constant_radius, size_t n);

/* Convenience: create + build. */
SRT_API srt_status srt_build_triangles(srt_ctx *ctx, const float *vertices,
                                       size_t nvertices, const uint32_t *faces,
                                       size_t nfaces, srt_accel **out);
SRT_API srt_status srt_build_tetrahedra(srt_ctx *ctx, const float *vertices,
                                        size_t nvertices, const uint32_t *tets,
                                        size_t ntets, srt_accel **out);
SRT_API srt_status srt_build_spheres(srt_ctx *ctx, const float *centers,
                                     const float *radius, float constant_radius,
                                     size_t n, srt_accel **out);

/* Root box of the built tree (synchronises the context stream). */
SRT_API srt_status srt_accel_bbox(srt_accel *accel, double bmin[3],
                                  double bmax[3]);
SRT_API srt_status srt_accel_info_get(srt_accel *accel, srt_accel_info *info);

/* Copy the device tree to host memory (synchronises).  Any pointer may be
 * NULL.  nodes: info.num_nodes records of info.node_bytes -- triangles and
 * spheres: 64-byte two-child nodes {float lo0[3], hi0[3], lo1[3], hi1[3];
 * uint32 ref0, ref1, count0 | axis << 30, count1} where count 0 marks a
 * branch child (ref = node index) and count > 0 a leaf (ref = first sorted
 * primitive); tetrahedra: 32-byte own-box nodes {float lo[3]; uint32 meta;
 * float hi[3]; uint32 ref} with meta = 0x80000000 | count for a leaf (ref =
 * first sorted primitive) or the split axis for a branch (children at ref,
 * ref+1).  indices: sorted primitive ids
 * (TriangleAccel::indices_); codes: sorted Morton codes. */
SRT_API srt_status srt_accel_export(srt_accel *accel, void *nodes,
                                    uint32_t *indices, uint32_t *codes);
/* Write the reference's Dump() file (u64 node count, reference node records,
 * u64 index count, u32 indices). */
SRT_API srt_status srt_accel_dump(srt_accel *accel, const char *path);

/* Closest hit for n rays.  opts may be NULL.  Asynchronous when rays and
 * hits are device pointers; synchronous (results copied back) otherwise.
 * Ray and hit arrays must be 16-byte aligned. */
SRT_API srt_status srt_trace_closest(srt_accel *accel, const srt_ray *rays,
                                     size_t n, srt_hit *hits,
                                     const srt_trace_opts *opts);

/* Closest hit for n rays without allocating memory (no counterpart in the
 * reference, whose Traverse works one ray at a time on the stack).  Same
 * hits as srt_trace_closest with opts == NULL, for callers that must not
 * allocate once running: cudaFree synchronises the whole device, and a
 * cudaMalloc can fail mid-frame in a process that fixed its device-memory
 * budget at start-up.  srt_trace_closest grows the context's deferred-ray
 * scratch on demand; this call keeps that list in a fixed 4 MiB device array
 * compiled into the library instead.
 *   - n <= 262144 rays per call (SRT_ERR_LIMIT above that; split the array).
 *   - rays and hits: device memory, 16-byte aligned.  Asynchronous on the
 *     context's stream; errors of the kernels surface at srt_ctx_synchronize.
 *   - The first call on each device does a one-time set-up (it looks up the
 *     array's device address, which may load the library's device code on
 *     that device); make it once at start-up, before any stream capture.
 *   - The array is shared by all contexts on a device: calls whose kernels
 *     overlap in time (different streams, unordered threads) race on it.
 *     Order them on one stream or synchronise between them.
 *   - Nothing needs to be zeroed by the caller: each call clears the array's
 *     deferred-ray count on the stream before its first kernel.
 *   - The array's address is kept per device number for the life of the
 *     process: a cudaDeviceReset, or a caller that runs the library in a
 *     non-primary driver context, is not supported with this call. */
SRT_API srt_status srt_trace_closest_noalloc(srt_accel *accel,
                                             const srt_ray *rays, size_t n,
                                             srt_hit *hits);

/* ---- build stages (bit-exact against the reference's own stages) ------ */
/* Scene box and 30-bit Morton code per primitive, in input order. */
SRT_API srt_status srt_stage_morton(srt_ctx *ctx, srt_kind kind,
                                    const float *vertices, size_t nvertices,
                                    const uint32_t *prims, const float *radius,
                                    float constant_radius, size_t n,
                                    uint32_t *codes, float scene_box[6]);
/* Stable sort of (code, index) pairs by code, in place. */
SRT_API srt_status srt_stage_sort_pairs(srt_ctx *ctx, uint32_t *codes,
                                        uint32_t *indices, size_t n);
/* Karras radix tree over n sorted codes: per internal node i in [0,n-2] the
 * split child[i] and whether the left/right child is a single key. */
SRT_API srt_status srt_stage_karras(srt_ctx *ctx, const uint32_t *codes,
                                    size_t n, uint32_t *child, uint8_t *left_leaf,
                                    uint8_t *right_leaf);

/* ---- volume ray march --------------------------------------------------- */
/* Emission-absorption march over a scalar FP32 grid (x fastest) through the
 * cube [-1,1]^3 with the shader's camera and texel-corner trilinear fetch. */
typedef struct srt_volume_params {
  int32_t width, height;
  int32_t max_steps;     /* hard cap on samples per ray */
  int32_t reserved;
  float eye[3];
  float corner[3];       /* image-plane corner (srt_volume_camera) */
  float du[3], dv[3];    /* image-plane step per pixel */
  float step;            /* world distance between samples */
  float sigma_scale;     /* extinction = sigma_scale * tf.a */
  float alpha_max;       /* per-sample opacity clamp, < 1 */
} srt_volume_params;

/* build_cameraframe (input.frag:16-29, FP32, pi as 3.14). */
SRT_API srt_status srt_volume_camera(int32_t width, int32_t height,
                                     const float eye[3], const float lookat[3],
                                     const float up[3], float fov_deg,
                                     srt_volume_params *params);
/* image: width*height*4 floats (premultiplied RGB, A = 1 - transmittance).
 * transmittance (optional): per-pixel final transmittance, kept for the
 * backward pass.  All pointers device or host. */
SRT_API srt_status srt_volume_march_fwd(srt_ctx *ctx,
                                        const srt_volume_params *params,
                                        const float *density, const int32_t dims[3],
                                        const float *tf, int32_t tf_entries,
                                        float *image, float *transmittance);
/* Adjoint: given d(loss)/d(image), accumulate d(loss)/d(density) and
 * d(loss)/d(tf) (both zeroed by the caller).  Recomputes transmittance in
 * reverse order from the forward image and final transmittance. */
SRT_API srt_status srt_volume_march_bwd(srt_ctx *ctx,
                                        const srt_volume_params *params,
                                        const float *density, const int32_t dims[3],
                                        const float *tf, int32_t tf_entries,
                                        const float *image,
                                        const float *transmittance,
                                        const float *grad_image,
                                        float *grad_density, float *grad_tf);

/* The density texture's sampling state for the march (the texture3D fetch
 * of Texture::Fetch, gles/gles_common.h:371-399): remap[k] (remap_n[k]
 * entries, NULL or 0 for none) is the coordinate remap of a non-uniform
 * volume (lsglTexCoordRemap; the reference's nonuniform_volume_render example
 * remaps y), applied as local::remap (gles/gles_common.h:264-269); clamp[k]
 * selects clamp-to-edge, 0 the repeat wrap of FilterTexture3DFloat (GL's
 * default, under which a coordinate remapped to 1.0 wraps to 0).  Tables
 * may be device or host memory.  The entry points without _ex march with
 * clamp-to-edge on every axis and no remap. */
typedef struct srt_volume_sampling {
  const float *remap[3];
  uint32_t remap_n[3];
  int32_t clamp[3];
} srt_volume_sampling;
SRT_API srt_status srt_volume_march_fwd_ex(srt_ctx *ctx, const srt_volume_params *params,
                                           const srt_volume_sampling *sampling,
                                           const float *density, const int32_t dims[3],
                                           const float *tf, int32_t tf_entries,
                                           float *image, float *transmittance);
SRT_API srt_status srt_volume_march_bwd_ex(srt_ctx *ctx, const srt_volume_params *params,
                                           const srt_volume_sampling *sampling,
                                           const float *density, const int32_t dims[3],
                                           const float *tf, int32_t tf_entries,
                                           const float *image, const float *transmittance,
                                           const float *grad_image, float *grad_density,
                                           float *grad_tf);

/* ---- eye rays and framebuffer ------------------------------------------- */
/* RaytraceEngine::OnData's per-pixel ray generation and framebuffer write
 * (gles/gles_raytrace_engine.cc:547-879) for one sample per pixel, with the
 * camera frame of Camera::buildFrame (render/render_camera.cc:17-63). */
typedef struct srt_camera {
  float eye[3], lookat[3], up[3];
  float fov;            /* vertical field of view, degrees (perspective) */
  int32_t ortho;        /* Camera's orthographic mode */
  int32_t width, height;   /* framebuffer, 1..65535 */
  int32_t viewport[4];     /* glViewport x, y, width, height */
  int32_t region[4];       /* render region x0, y0, x1, y1 (scissor, screen tile) */
  int32_t step;            /* pixel step (lsglSetPixelStep), >= 1 */
} srt_camera;

/* Eye rays of the loop pixels (x, y) = region start + multiples of step
 * whose viewport-converted pixel lies on the framebuffer, row by row.
 * rays (16-byte aligned) and pixel (optional; per ray (y << 16) | x of its
 * loop pixel) are device arrays with room for every loop pixel of the
 * region; *count receives the number written.  Asynchronous. */
SRT_API srt_status srt_camera_rays(srt_ctx *ctx, const srt_camera *cam,
                                   srt_ray *rays, uint32_t *pixel,
                                   uint32_t *count);
/* Write the hits of n rays made by srt_camera_rays: each hit fills the
 * step x step block of its loop pixel (rows counted from the top, as the
 * reference's Y-down framebuffer) with its colour -- rgba (n x float4, or
 * NULL for the reference's hit colour (1,1,1,1)) -- as RGBA8 (format 0,
 * clamp((int)(c * 255.0))) or RGBA32F (format 1), and its depth t into
 * depth (optional, width x height floats).  Misses leave pixels as they
 * are.  Device arrays, 16-byte aligned; asynchronous. */
SRT_API srt_status srt_framebuffer_write(srt_ctx *ctx, const srt_camera *cam,
                                         const srt_hit *hits,
                                         const uint32_t *pixel,
                                         const float *rgba, uint32_t n,
                                         int32_t format, void *color,
                                         float *depth);

/* Several samples per pixel and the stereo environment camera, as OnData
 * does them with sampleCoverage and lsglSetStereoEnvCamera
 * (gles/gles_raytrace_engine.cc:549-553, 747-800, 826-877;
 * render/render_camera.cc:65-118). */
typedef struct srt_camera_samples {
  int32_t subsamples;      /* per axis (sampleCoverageValue), 1..16 */
  int32_t stereo_env;      /* 1: Camera::generateStereoEnvRay rays */
  float zero_parallax;     /* stereo camera's focal distance */
  float eye_separation;    /* stereo camera's eye separation */
  /* The sample jitter: subsample (vv, uu) lies at ((uu + ju) / S, (vv + jv)
   * / S) in its pixel, ju (uu != 0) then jv (vv != 0) drawn from the serial
   * renderer's random stream -- TinyMT64 with the parameters of
   * gles_common.cc's initialize_random, seeded jitter_seed (1234 there),
   * draws as (float) of its doubles -- in pixel order (rows, then x) over
   * the kept pixels, after jitter_offset draws (those of earlier frames). */
  uint64_t jitter_seed;
  uint64_t jitter_offset;
} srt_camera_samples;

/* srt_camera_rays with samples: per kept loop pixel (rows, then x) its
 * subsamples^2 rays, (vv, uu) row-major; pixel (optional) gets each ray's
 * loop pixel; rays/pixel need room for subsamples^2 rays per loop pixel.
 * *draws receives the jitter draws the frame consumed (the next frame's
 * jitter_offset is this one's plus it).  With stereo_env the camera's
 * fov and ortho are not used.  Device arrays; asynchronous. */
SRT_API srt_status srt_camera_rays_ex(srt_ctx *ctx, const srt_camera *cam,
                                      const srt_camera_samples *smp, srt_ray *rays,
                                      uint32_t *pixel, uint32_t *count,
                                      uint64_t *draws);
/* The write of n rays made by srt_camera_rays_ex: per loop pixel the sum of
 * its hits' colours and depths times 1 / subsamples^2 fills its block, for
 * pixels with at least one hit (other arguments as srt_framebuffer_write). */
SRT_API srt_status srt_framebuffer_write_ex(srt_ctx *ctx, const srt_camera *cam,
                                            const srt_camera_samples *smp,
                                            const srt_hit *hits, const uint32_t *pixel,
                                            const float *rgba, uint32_t n,
                                            int32_t format, void *color, float *depth);

/* ---- scenes: several accels with transforms ----------------------------- */
/* RenderGraph (gles/gles_render_graph.cc:104-314) on the GPU: built accels
 * placed in the world by 4x4 transforms, a top-level tree over their world
 * boxes (BVHTree, render/render_bvh_tree.cc), and the nearest hit over all
 * of them per ray.  Matrices are doubles in Matrixd's layout (m[row][col],
 * p' = p m + m[3]); the caller passes T, its inverse, the inverse of its
 * upper 3x3 and the world box, as RenderElement::Update computes them. */
typedef struct srt_scene srt_scene;
SRT_API srt_status srt_scene_create(srt_ctx *ctx, srt_scene **out);
SRT_API srt_status srt_scene_destroy(srt_scene *scene);
/* Add a built accel of the scene's context; *id (optional) = its element id
 * (0, 1, ... in call order).  Accels must stay built and unchanged while the
 * scene is used; rebuild the scene after rebuilding one of them. */
SRT_API srt_status srt_scene_add(srt_scene *scene, srt_accel *accel,
                                 const double T[16], const double invT[16],
                                 const double invT33[16],
                                 const double world_bmin[3],
                                 const double world_bmax[3], uint32_t *id);
/* The same, as RenderElement's constructor does it (gles/gles_primitive.cc:
 * 346, gles/gles_render_graph.cc:77-101): local box = srt_accel_bbox, world
 * box of its eight corners under T, invT and invT33 by Matrixd::Inverse's
 * cofactor rule -- bit for bit the reference's values. */
SRT_API srt_status srt_scene_add_element(srt_scene *scene, srt_accel *accel,
                                         const double T[16], uint32_t *id);
/* Matrixd::Inverse (render/render_matrix.h:40-134) of a row-major 4x4, in
 * place (host only). */
SRT_API void srt_matrix_inverse(double m[16]);
/* RenderGraph::Build: the top-level tree (BVHTree::BuildTree). */
SRT_API srt_status srt_scene_build(srt_scene *scene);
/* RenderGraph::Trace for n rays (device arrays): hits in world distance t
 * (u, v, prim of the element's own hit), element[i] (optional) = the hit
 * element or 0xFFFFFFFF.  prev_element (optional): the element each ray's
 * prev_prim belongs to (the self-hit rule applies only there), with
 * prev_normals (optional, 3 floats per ray) for spheres.  stats (optional,
 * device, 5 counters added to): top-level nodes visited, element walks,
 * branch nodes, leaves and primitives visited inside the elements.
 * Up to 64 candidate elements per ray (SRT_ERR_LIMIT beyond).  Asynchronous. */
SRT_API srt_status srt_scene_trace(srt_scene *scene, const srt_ray *rays,
                                   size_t n, const uint32_t *prev_element,
                                   const float *prev_normals, srt_hit *hits,
                                   uint32_t *element, uint64_t *stats);
/* The top-level tree: per node bmin[3], bmax[3] (boxes, 6 doubles) and
 * child0, child1, axis, leaf, element (ints, 5 int32); returns the node
 * count (arrays may be NULL or shorter: cap entries are filled). */
SRT_API size_t srt_scene_top_nodes(srt_scene *scene, double *boxes,
                                   int32_t *ints, size_t cap);

/* ---- 3D texture fetch ----------------------------------------------------
 * Texture::Fetch for 3D textures (gles/gles_common.h:344-399) over an array
 * of coordinates, bit for bit the reference's values.
 *   dense: FilterTexture3D{Byte,Float,Double} (render/render_texture.cc:
 *   832-1175) after the optional per-axis remap of non-uniform volumes
 *   (local::remap, gles/gles_common.h:264-269, set by lsglTexCoordRemap);
 *   repeat wrap unless clamp-to-edge (Texture::SetWrap*).
 *   sparse: SparseVolumeAccel::Build / Sample (render/render_accel_volume.cc:
 *   37-139) at u * globalDim, the nearest texel of the first block
 *   BVHTree::Locate reaches; (0, 0, 0, 0) outside every block.
 * format: 0 = bytes, 1 = float, 2 = double (LSGL_RENDER_TEXTURE3D_FORMAT_BYTE /
 * FLOAT / DOUBLE); texels x fastest, components interleaved (1..4 dense).
 * Data are copied to the device (the call synchronises the context stream).
 * srt_texture3d_fetch: uvw (3 floats per sample) and rgba (4 floats per
 * sample; 16-byte aligned when on the device): device arrays are used in
 * place and the call is asynchronous; host arrays are staged and the call
 * returns with the result written.  A sparse fetch whose block-tree walk
 * reaches its step cap returns SRT_ERR_LIMIT: from the call itself when it
 * staged host arrays, else from the next srt_ctx_synchronize. */
typedef struct srt_texture3d srt_texture3d;
typedef struct srt_volume_block {      /* VolumeBlock, render/render_prim_volume.h:18-26 */
  int32_t offset[3], extent[3], size[3], level;
  uint64_t data_offset;                /* byte offset of its voxels in the pool */
} srt_volume_block;
SRT_API srt_status srt_texture3d_create(srt_ctx *ctx, srt_texture3d **out);
SRT_API srt_status srt_texture3d_destroy(srt_texture3d *tex);
SRT_API srt_status srt_texture3d_set_dense(srt_texture3d *tex, int format, int width,
                                           int height, int depth, int components,
                                           const void *data);
SRT_API srt_status srt_texture3d_set_wrap(srt_texture3d *tex, int clamp_s, int clamp_t,
                                          int clamp_r);
/* axis 0..2; n = 0 removes the remap of that axis */
SRT_API srt_status srt_texture3d_set_remap(srt_texture3d *tex, int axis, const float *table,
                                           size_t n);
SRT_API srt_status srt_texture3d_set_sparse(srt_texture3d *tex, int format, int components,
                                            const int global_dim[3],
                                            const srt_volume_block *blocks, size_t nblocks,
                                            const void *pool, size_t pool_bytes);
SRT_API srt_status srt_texture3d_fetch(srt_texture3d *tex, const float *uvw, size_t n,
                                       float *rgba);

/* ---- accels across frames and runs ------------------------------------
 * srt_accel_load_*: the accel of the given primitives from a file in the
 * reference's Dump() format (XxxAccel::Dump, render/render_accel_triangle.cc:
 * 1692-1719, render/render_accel_tetra.cc:1900, render/render_accel_particle.cc:
 * 1868; srt_accel_dump writes the same), without a rebuild.  The reference
 * writes these files but reads none back.  The primitives must be the ones
 * the tree was built from; the file is checked completely first (counts and
 * size, node indices, leaf ranges covering every primitive once, split
 * axes, depth <= 28, the sorted order a permutation) and a damaged file is
 * SRT_ERR_INVALID (SRT_ERR_UNSUPPORTED for a leaf root or a deeper tree).
 * Synchronises the context stream. */
SRT_API srt_status srt_accel_load_triangles(srt_accel *accel, const char *path,
                                            const float *vertices, size_t nvertices,
                                            const uint32_t *faces, size_t nfaces);
SRT_API srt_status srt_accel_load_tetrahedra(srt_accel *accel, const char *path,
                                             const float *vertices, size_t nvertices,
                                             const uint32_t *tets, size_t ntets);
SRT_API srt_status srt_accel_load_spheres(srt_accel *accel, const char *path,
                                          const float *centers, const float *radius,
                                          float constant_radius, size_t n);

/* AccelBuilder's cache (gles/gles_accel_builder.cc:34-117, 400-456,
 * 1017-1037).  The key is what Locate compares: the element and array
 * buffers (any caller ids), the position attribute's offset, count and
 * offset; the kind is compared too.  srt_cache_build_* return the cached
 * accel of a static entry (a hit) or build one and keep it: in the static
 * list when is_static (both buffers static), else in the dynamic list,
 * which srt_cache_end_frame frees (AccelBuilder::EndFrame); dynamic entries
 * are never found again, as in Locate.  srt_cache_invalidate frees every
 * entry built from a buffer (AccelBuilder::Invalidate).  The cache owns its
 * accels: do not destroy them; they stay valid until invalidated, freed at
 * the end of the frame (dynamic) or the cache is destroyed.  bytes_used
 * counts the accels' device memory; like the reference, nothing is evicted
 * when it exceeds bytes_max. */
typedef struct srt_cache srt_cache;
typedef struct srt_cache_key {
  uint64_t elem_buffer, array_buffer, position_offset;
  uint32_t count, offset;
} srt_cache_key;
typedef struct srt_cache_info {
  uint64_t bytes_used, bytes_max, static_entries, dynamic_entries, hits, builds;
} srt_cache_info;
SRT_API srt_status srt_cache_create(srt_ctx *ctx, uint64_t max_bytes, srt_cache **out);
SRT_API srt_status srt_cache_destroy(srt_cache *cache);
SRT_API srt_status srt_cache_build_triangles(srt_cache *cache, const srt_cache_key *key,
                                             int is_static, const float *vertices,
                                             size_t nvertices, const uint32_t *faces,
                                             size_t nfaces, srt_accel **out);
SRT_API srt_status srt_cache_build_tetrahedra(srt_cache *cache, const srt_cache_key *key,
                                              int is_static, const float *vertices,
                                              size_t nvertices, const uint32_t *tets,
                                              size_t ntets, srt_accel **out);
SRT_API srt_status srt_cache_build_spheres(srt_cache *cache, const srt_cache_key *key,
                                           int is_static, const float *centers,
                                           const float *radius, float constant_radius,
                                           size_t n, srt_accel **out);
SRT_API srt_status srt_cache_invalidate(srt_cache *cache, uint64_t buffer);
/* AccelBuilder::BuildLineAccel (gles/gles_accel_builder.cc:188-256) and
 * BuildSolidAccel (:328-397): the same cache for line and solid accels
 * (srt_line_build with LineBuildOptions' defaults and the given cap;
 * srt_solid_build).  As in AccelBuilder::Locate, the line cap flag is not
 * part of the key: a static line accel built with one cap value is returned
 * for a later call with the other. */
typedef struct srt_line_accel srt_line_accel;
typedef struct srt_solid_accel srt_solid_accel;
SRT_API srt_status srt_cache_build_lines(srt_cache *cache, const srt_cache_key *key,
                                         int is_static, const float *positions, size_t nverts,
                                         const float *radius, float constant_radius,
                                         const uint32_t *segments, size_t nlines, int32_t cap,
                                         srt_line_accel **out);
SRT_API srt_status srt_cache_build_solids(srt_cache *cache, const srt_cache_key *key,
                                          int is_static, int32_t verts_per_solid,
                                          const float *vertices, size_t nverts,
                                          const uint32_t *indices, size_t nsolids,
                                          srt_solid_accel **out);
SRT_API srt_status srt_cache_end_frame(srt_cache *cache);
SRT_API srt_status srt_cache_info_get(srt_cache *cache, srt_cache_info *info);

/* ---- secondary rays ----------------------------------------------------- */
/* One secondary ray per hit ray (the particle workload's bounce; in the
 * reference a fragment shader builds it and calls back trace() with
 * prev_prim_id / prev_hit_t / prev_hit_normal set, gles/gles_glsl_runtime.cc:
 * 119-136; no render/ counterpart).  For every i with hits[i].prim != miss,
 * in order of i: origin = rays[i].org + t * rays[i].dir (float), direction
 * uniform on the hemisphere about normals[i] (unit), drawn from a
 * counter-based stream of `seed` and i; prev_prim = hit prim, prev_t = t;
 * out_normals gets the unit normal (pass it as srt_trace_opts.prev_normals).
 * All arrays are device memory (out / out_normals sized for n rays); *count
 * receives the number of rays written; synchronises the context stream. */
SRT_API srt_status srt_spawn_secondary(srt_ctx *ctx, const srt_ray *rays,
                                       const srt_hit *hits, const float *normals,
                                       size_t n, uint64_t seed, srt_ray *out,
                                       float *out_normals, uint32_t *count);

/* ---- batched build + trace ---------------------------------------------- */
/* Many triangle scenes of uneven size, built and traced in one pass (the
 * per-scene Build32 + Traverse of every scene, with identical results).
 * Scene s owns faces [face_offsets[s], face_offsets[s+1]) of `faces`
 * (vertex ids into `vertices`) and rays [ray_offsets[s], ray_offsets[s+1]);
 * hits are written per ray, prim = face index within the scene.  vertices,
 * faces, rays and hits are device pointers; the nscenes+1 offsets are host
 * arrays.  1 <= nscenes <= 256, each scene >= 2 faces.
 * The first call autotunes the traversal launch shape; the second call with
 * the same arguments captures build + trace in a CUDA graph (on the
 * context's own stream) and later identical calls replay it. */
typedef struct srt_batch srt_batch;
SRT_API srt_status srt_batch_create(srt_ctx *ctx, srt_batch **out);
SRT_API srt_status srt_batch_destroy(srt_batch *b);
SRT_API srt_status srt_batch_build_trace(srt_batch *b, int32_t nscenes,
                                         const float *vertices,
                                         const uint32_t *faces,
                                         const uint64_t *face_offsets,
                                         const srt_ray *rays,
                                         const uint64_t *ray_offsets,
                                         srt_hit *hits);
/* Launch shape picked by the autotuner, whether a graph is captured, and
 * the kernels one call runs. */
SRT_API srt_status srt_batch_config(srt_batch *b, int32_t *block,
                                    int32_t *rays_per_thread,
                                    int32_t *graph_captured,
                                    uint64_t *kernels_per_call);
/* The traversal point the autotuner picked on the batch's first call: block
 * size, grabs of 32 rays per warp, traversal stack depth (24, 32 or 48
 * entries) and ray order (0: array order; 12 or 22: sorted within each
 * scene by that many top bits of a Morton code over origin and direction). */
SRT_API srt_status srt_batch_tuning(srt_batch *b, int32_t *block,
                                    int32_t *rays_per_grab, int32_t *stack_depth,
                                    int32_t *sort_bits);
/* Pin the traversal point instead of autotuning it (block 64, 128 or 256;
 * 1..8 grabs; depth 24, 32 or 48; sort bits 0, 12 or 22).  Drops a captured
 * graph.  Hits do not depend on the point, except that a depth the trees
 * overflow ends the call with SRT_ERR_LIMIT. */
SRT_API srt_status srt_batch_set_tuning(srt_batch *b, int32_t block,
                                        int32_t rays_per_grab, int32_t stack_depth,
                                        int32_t sort_bits);

/* ---------------------------------------------------------------- lines
 * LineAccel (render/render_accel_line.{h,cc}): capped cylinders between the
 * end points of line segments (Lines, render/render_prim_line.h).
 * srt_line_build replaces LineAccel::Build (render_accel_line.cc:298): the
 * same spatial-median tree and line order (positions: nverts xyz floats;
 * radius: per vertex or NULL for constant_radius; segments: 2 vertex indices
 * per line; min_leaf, max_depth and cap as LineBuildOptions, 0 for its
 * defaults 4 and 512), built on the GPU level by level; a segment naming a
 * vertex beyond nverts, or a NaN position or radius, is SRT_ERR_INVALID.
 * srt_line_trace replaces LineAccel::Traverse (:704):
 * closest hit per ray (t, u, v, line index; u = distance from the axis on a
 * cap, v = 0 / 1 on a cap or the position along the axis), normals (3 floats
 * per ray, BuildIntersection's, may be NULL); stats (device memory, NULL
 * or 3 uint64 accumulated: branches popped, leaves popped, lines tested).
 * Inputs may be host or device
 * memory.  srt_line_bbox replaces LineAccel::BoundingBox (:776),
 * srt_line_dump LineAccel::Dump (:343, the same file format); srt_line_export
 * copies the tree in the Dump record layout (40 bytes per node) and the line
 * order. */
SRT_API srt_status srt_line_create(srt_ctx *ctx, srt_line_accel **out);
SRT_API srt_status srt_line_destroy(srt_line_accel *accel);
SRT_API srt_status srt_line_build(srt_line_accel *accel, const float *positions,
                                  size_t nverts, const float *radius, float constant_radius,
                                  const uint32_t *segments, size_t nlines, int32_t min_leaf,
                                  int32_t max_depth, int32_t cap);
SRT_API srt_status srt_line_trace(srt_line_accel *accel, const srt_ray *rays, size_t n,
                                  srt_hit *hits, float *normals, uint64_t *stats);
SRT_API srt_status srt_line_bbox(srt_line_accel *accel, double bmin[3], double bmax[3]);
SRT_API srt_status srt_line_info(srt_line_accel *accel, uint64_t *nlines, uint64_t *nnodes,
                                 int32_t *depth);
SRT_API srt_status srt_line_export(srt_line_accel *accel, void *nodes, uint32_t *indices);
SRT_API srt_status srt_line_dump(srt_line_accel *accel, const char *path);

/* ---------------------------------------------------------------- solids
 * SolidAccel (render/render_accel_solid.{h,cc}) over Solid
 * (render/render_prim_solid.h): pyramids (verts_per_solid 5), prisms (6),
 * hexahedra (8).  srt_solid_build replaces SolidAccel::Build32
 * (render_accel_solid.cc:1795; the same tree and solid order for 2 to
 * 2^28 - 1 solids: the LBVH on the GPU from 1024 solids on, and below 1024,
 * as the reference does, its binned-SAH SolidAccel::Build (:1612-1793) on
 * the host);
 * srt_solid_trace replaces SolidAccel::Traverse (:2345): per ray the
 * nearest entry or exit point (t, solid in hits[i].prim; u = v = 0, which
 * the reference leaves unset), skipping the solid named by prev_prim, and
 * optionally the point's normal and position (3 floats per ray each, NULL
 * to skip).  Inputs may be host or device memory.  srt_solid_bbox replaces
 * SolidAccel::BoundingBox, srt_solid_dump SolidAccel::Dump (:2126, the same
 * file format); srt_solid_export copies the tree in the Dump record layout
 * (40 bytes per node) and the solid order. */
SRT_API srt_status srt_solid_create(srt_ctx *ctx, srt_solid_accel **out);
SRT_API srt_status srt_solid_destroy(srt_solid_accel *accel);
SRT_API srt_status srt_solid_build(srt_solid_accel *accel, int32_t verts_per_solid,
                                   const float *vertices, size_t nverts,
                                   const uint32_t *indices, size_t nsolids);
/* The same with double-precision positions: Solid::dvertices with
 * isDoublePrecisionPos (render/render_prim_solid.h).  As the reference does,
 * the scene box and node boxes pad each double coordinate in double and
 * round to float, the Morton codes and SAH bins use the positions rounded
 * to float, SAHPredD sums in double, and the Pluecker tests take the
 * doubles (render_accel_solid.cc:1628-1640, 1836-1880, 2243-2250). */
SRT_API srt_status srt_solid_build_double(srt_solid_accel *accel, int32_t verts_per_solid,
                                          const double *vertices, size_t nverts,
                                          const uint32_t *indices, size_t nsolids);
/* SolidAccel::Build, the binned-SAH build (render_accel_solid.cc:1754), at
 * every size: the build the reference's GLES accel builder runs
 * (gles/gles_accel_builder.cc:967; srt_cache_build_solids uses it).  A host
 * build uploaded to the GPU; traversal as above. */
SRT_API srt_status srt_solid_build_sah(srt_solid_accel *accel, int32_t verts_per_solid,
                                       const float *vertices, size_t nverts,
                                       const uint32_t *indices, size_t nsolids);
SRT_API srt_status srt_solid_build_sah_double(srt_solid_accel *accel, int32_t verts_per_solid,
                                              const double *vertices, size_t nverts,
                                              const uint32_t *indices, size_t nsolids);
SRT_API srt_status srt_solid_trace(srt_solid_accel *accel, const srt_ray *rays, size_t n,
                                   srt_hit *hits, float *normals, float *positions);
SRT_API srt_status srt_solid_bbox(srt_solid_accel *accel, double bmin[3], double bmax[3]);
SRT_API srt_status srt_solid_info(srt_solid_accel *accel, uint64_t *nsolids, uint64_t *nnodes);
SRT_API srt_status srt_solid_export(srt_solid_accel *accel, void *nodes, uint32_t *indices);
SRT_API srt_status srt_solid_dump(srt_solid_accel *accel, const char *path);

/* Line and solid accels as scene elements: RenderGraph::Trace's
 * PRIMITIVE_LINES and PRIMITIVE_PYRAMIDS / PRISMS / HEXAHEDRONS cases
 * (gles/gles_render_graph.cc:239-260), added as srt_scene_add_element adds
 * an srt_accel (local box = srt_line_bbox / srt_solid_bbox, RenderElement's
 * world box and inverse matrices).  A hit on a line element carries the
 * line's (u, v); on a solid element u = v = 0, and the previous solid is
 * skipped inside the element the ray left (prev_element). */
SRT_API srt_status srt_scene_add_lines(srt_scene *scene, srt_line_accel *accel,
                                       const double T[16], uint32_t *id);
SRT_API srt_status srt_scene_add_solids(srt_scene *scene, srt_solid_accel *accel,
                                        const double T[16], uint32_t *id);

#ifdef __cplusplus
}
#endif
#endif /* SURFACE_RT_H_ */
