// srt_cache.cu -- accels kept across frames and runs.
//
// * srt_accel_load_*: an accel from a file in the reference's Dump() format
//   (render/render_accel_triangle.cc:1692-1719, render_accel_tetra.cc:1900,
//   render_accel_particle.cc:1868; the format srt_accel_dump writes) and the
//   primitives it was built from, without a rebuild.  The reference writes
//   these files but has no reader; the file is checked completely before
//   anything reaches the GPU (sizes, node indices, leaf ranges, axes, depth,
//   the sorted order being a permutation), so a damaged file is an error,
//   never an out-of-bounds walk.
// * srt_cache_*: AccelBuilder's cache (gles/gles_accel_builder.cc:34-117,
//   400-456, 1017-1037): accels keyed by the buffers they were built from,
//   static entries found again by Locate, dynamic ones freed at the end of
//   the frame, Invalidate(buffer) dropping every entry built from a buffer.
#include <cstdio>
#include <cstring>
#include <vector>

#include "srt_internal.cuh"

using namespace srt;

namespace {

// Reference record sizes: TriangleNode 64 B (bmin[2][3], bmax[2][3], int
// flag, int axis, uint data[2]), TetraNode 40 B (bmin[3], bmax[3], int flag,
// int axis, uint data[2]), ParticleNode 60 B (bmin[2][3], bmax[2][3],
// uint data[2], short flag, short axis).
size_t record_bytes(srt_kind k) {
  return k == SRT_TRIANGLES ? 64 : k == SRT_TETRAHEDRA ? 40 : 60;
}

struct Rec {
  float lo[2][3], hi[2][3];
  int32_t leaf, axis;
  uint32_t d0, d1;  // branch: children; leaf: count, first sorted primitive
};

Rec parse_rec(srt_kind k, const unsigned char *p) {
  Rec r;
  memset(&r, 0, sizeof(r));
  if (k == SRT_TETRAHEDRA) {
    memcpy(r.lo[0], p, 12);
    memcpy(r.hi[0], p + 12, 12);
    memcpy(&r.leaf, p + 24, 4);
    memcpy(&r.axis, p + 28, 4);
    memcpy(&r.d0, p + 32, 4);
    memcpy(&r.d1, p + 36, 4);
  } else {
    memcpy(r.lo, p, 24);
    memcpy(r.hi, p + 24, 24);
    if (k == SRT_TRIANGLES) {
      memcpy(&r.leaf, p + 48, 4);
      memcpy(&r.axis, p + 52, 4);
      memcpy(&r.d0, p + 56, 4);
      memcpy(&r.d1, p + 60, 4);
    } else {
      int16_t fl, ax;
      memcpy(&r.d0, p + 48, 4);
      memcpy(&r.d1, p + 52, 4);
      memcpy(&fl, p + 56, 2);
      memcpy(&ax, p + 58, 2);
      r.leaf = fl;
      r.axis = ax;
    }
  }
  return r;
}

float bits_f(uint32_t u) {
  float f;
  memcpy(&f, &u, 4);
  return f;
}

srt_status fail(srt_status s, const std::string &m) {
  set_error(m);
  return s;
}

// Reads and checks a dump for n primitives; converts it to the device
// layout.  Tree rules checked: root at record 0 is a branch, every record is
// reached exactly once, children are later records, leaves hold 1..2^30-1
// primitives and together cover [0, n) once, axes are 0..2, depth <= 28
// (the traversal stack holds 32 entries).
srt_status read_dump(srt_kind kind, const char *path, size_t n, std::vector<unsigned char> &dev,
                     size_t &nnodes, uint32_t &nbranches, std::vector<uint32_t> &idx) {
  FILE *fp = fopen(path, "rb");
  if (!fp) return fail(SRT_ERR_INVALID, std::string("cannot read ") + path);
  std::vector<unsigned char> buf;
  unsigned char chunk[1 << 16];
  size_t got;
  while ((got = fread(chunk, 1, sizeof(chunk), fp)) > 0) buf.insert(buf.end(), chunk, chunk + got);
  fclose(fp);
  const size_t rb = record_bytes(kind);
  unsigned long long nn = 0, ni = 0;
  if (buf.size() < 16) return fail(SRT_ERR_INVALID, "dump too short");
  memcpy(&nn, buf.data(), 8);
  if (nn == 0 || nn > (buf.size() - 16) / rb) return fail(SRT_ERR_INVALID, "dump node count");
  const size_t off_i = 8 + (size_t)nn * rb;
  memcpy(&ni, buf.data() + off_i, 8);
  if (ni != n) return fail(SRT_ERR_INVALID, "dump holds a tree for another primitive count");
  if (buf.size() != off_i + 8 + (size_t)ni * 4)
    return fail(SRT_ERR_INVALID, "dump size does not match its counts (wrong accel kind?)");
  idx.resize(n);
  memcpy(idx.data(), buf.data() + off_i + 8, n * 4);
  std::vector<unsigned char> seen(n, 0);
  for (size_t j = 0; j < n; j++) {
    if (idx[j] >= n || seen[idx[j]]) return fail(SRT_ERR_INVALID, "dump order is not a permutation");
    seen[idx[j]] = 1;
  }
  std::vector<Rec> rec(nn);
  for (size_t i = 0; i < nn; i++) rec[i] = parse_rec(kind, buf.data() + 8 + i * rb);
  if (rec[0].leaf) return fail(SRT_ERR_UNSUPPORTED, "dump root is a leaf");
  // walk from the root: every record once, leaves covering [0, n) once
  std::vector<unsigned char> reached(nn, 0);
  std::vector<unsigned char> covered(n, 0);
  struct Item {
    uint32_t r;
    int depth;
  };
  std::vector<Item> stk{{0u, 0}};
  reached[0] = 1;
  size_t branches = 0, leaves = 0;
  while (!stk.empty()) {
    const Item it = stk.back();
    stk.pop_back();
    const Rec &x = rec[it.r];
    if (it.depth > 28) return fail(SRT_ERR_UNSUPPORTED, "dump tree deeper than 28 levels");
    if (x.leaf != 0 && x.leaf != 1) return fail(SRT_ERR_INVALID, "dump leaf flag");
    if (x.leaf) {
      if (x.d0 == 0 || x.d0 > kCountMask || (uint64_t)x.d1 + x.d0 > n)
        return fail(SRT_ERR_INVALID, "dump leaf range");
      for (uint32_t j = x.d1; j < x.d1 + x.d0; j++) {
        if (covered[j]) return fail(SRT_ERR_INVALID, "dump leaves overlap");
        covered[j] = 1;
      }
      leaves++;
      continue;
    }
    if (x.axis < 0 || x.axis > 2) return fail(SRT_ERR_INVALID, "dump split axis");
    for (uint32_t c : {x.d0, x.d1}) {
      if (c <= it.r || c >= nn || reached[c]) return fail(SRT_ERR_INVALID, "dump child index");
      reached[c] = 1;
      stk.push_back({c, it.depth + 1});
    }
    branches++;
  }
  for (size_t i = 0; i < nn; i++)
    if (!reached[i]) return fail(SRT_ERR_INVALID, "dump holds unreachable nodes");
  for (size_t j = 0; j < n; j++)
    if (!covered[j]) return fail(SRT_ERR_INVALID, "dump leaves miss primitives");
  (void)leaves;
  nbranches = (uint32_t)branches;
  if (kind == SRT_TETRAHEDRA) {
    // own-box nodes, the two children of a branch in adjacent slots
    nnodes = 2 * branches + 1;
    std::vector<NodeT> out(nnodes);
    std::vector<std::pair<uint32_t, uint32_t>> q{{0u, 0u}};  // (record, slot)
    uint32_t next = 1;
    for (size_t h = 0; h < q.size(); h++) {
      const Rec &x = rec[q[h].first];
      NodeT &d = out[q[h].second];
      uint32_t meta, ref;
      if (x.leaf) {
        meta = kLeafBit | x.d0;
        ref = x.d1;
      } else {
        meta = (uint32_t)x.axis;
        ref = next;
        q.push_back({x.d0, next});
        q.push_back({x.d1, next + 1});
        next += 2;
      }
      d.a = make_float4(x.lo[0][0], x.lo[0][1], x.lo[0][2], bits_f(meta));
      d.b = make_float4(x.hi[0][0], x.hi[0][1], x.hi[0][2], bits_f(ref));
    }
    dev.resize(nnodes * sizeof(NodeT));
    memcpy(dev.data(), out.data(), dev.size());
  } else {
    // two-child nodes in depth-first order; leaves fold into their parent
    nnodes = branches;
    std::vector<uint32_t> slot(nn, 0);
    uint32_t k = 0;
    std::vector<uint32_t> order{0u};
    std::vector<uint32_t> pre;
    while (!order.empty()) {
      const uint32_t r = order.back();
      order.pop_back();
      if (rec[r].leaf) continue;
      slot[r] = k++;
      pre.push_back(r);
      order.push_back(rec[r].d1);
      order.push_back(rec[r].d0);
    }
    std::vector<Node2> out(nnodes);
    for (uint32_t r : pre) {
      const Rec &x = rec[r];
      uint32_t ref[2], cnt[2];
      const uint32_t ch[2] = {x.d0, x.d1};
      for (int c = 0; c < 2; c++) {
        const Rec &y = rec[ch[c]];
        ref[c] = y.leaf ? y.d1 : slot[ch[c]];
        cnt[c] = y.leaf ? y.d0 : 0u;
      }
      Node2 &d = out[slot[r]];
      d.a = make_float4(x.lo[0][0], x.lo[0][1], x.lo[0][2], x.hi[0][0]);
      d.b = make_float4(x.hi[0][1], x.hi[0][2], x.lo[1][0], x.lo[1][1]);
      d.c = make_float4(x.lo[1][2], x.hi[1][0], x.hi[1][1], x.hi[1][2]);
      d.d = make_uint4(ref[0], ref[1], cnt[0] | ((uint32_t)x.axis << 30), cnt[1]);
    }
    dev.resize(nnodes * sizeof(Node2));
    memcpy(dev.data(), out.data(), dev.size());
  }
  return SRT_OK;
}

srt_status load_common(srt_accel *a, srt_kind kind, const char *path, const float *verts,
                       size_t nverts, const uint32_t *prims, size_t nprims, int per_prim,
                       const float *radius, float constr) {
  if (!a || !path || !verts) return fail(SRT_ERR_INVALID, "NULL argument");
  if (a->kind != kind) return fail(SRT_ERR_INVALID, "accel kind does not match the loader");
  if (nprims < 2 || nprims >= (1u << 30))
    return fail(SRT_ERR_INVALID, "primitive count must be in [2, 2^30)");
  if (per_prim > 0 && (!prims || nverts == 0))
    return fail(SRT_ERR_INVALID, "NULL primitive index array");
  std::vector<unsigned char> nodes;
  std::vector<uint32_t> idx;
  size_t nnodes = 0;
  uint32_t nbranches = 0;
  srt_status s = read_dump(kind, path, nprims, nodes, nnodes, nbranches, idx);
  if (s != SRT_OK) return s;
  srt_ctx *ctx = a->ctx;
  if (cudaSetDevice(ctx->device) != cudaSuccess) return cuda_status(cudaGetLastError(), "device");
  // the primitives as the build takes them: device arrays in place, host
  // arrays copied into the accel's staging
  const void *dv = nullptr, *df = nullptr, *dr = nullptr;
  auto view = [&](const void *p, size_t bytes, DevBuf &stage, const void **out) -> srt_status {
    if (!p || bytes == 0 || is_device_ptr(p)) {
      *out = p;
      return SRT_OK;
    }
    cudaError_t e = stage.ensure(bytes);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(stage.p, p, bytes, cudaMemcpyHostToDevice, ctx->stream);
    if (e != cudaSuccess) return cuda_status(e, "load staging");
    *out = stage.p;
    return SRT_OK;
  };
  s = view(verts, (per_prim > 0 ? nverts : nprims) * 3 * sizeof(float), a->in_verts, &dv);
  if (s == SRT_OK && per_prim > 0)
    s = view(prims, nprims * per_prim * sizeof(uint32_t), a->in_faces, &df);
  if (s == SRT_OK && radius) s = view(radius, nprims * sizeof(float), a->in_radius, &dr);
  if (s != SRT_OK) return s;
  a->built = false;
  a->n = nprims;
  a->src_verts = static_cast<const float *>(dv);
  a->src_faces = static_cast<const uint32_t *>(df);
  s = load_accel(a, static_cast<const float *>(dv), static_cast<const uint32_t *>(df),
                 static_cast<const float *>(dr), constr, nprims, nodes.data(), nnodes,
                 nbranches, idx.data());
  a->built = (s == SRT_OK);
  return s;
}

}  // namespace

// ------------------------------------------------------------------ cache
struct srt_cache {
  srt_ctx *ctx = nullptr;
  uint64_t max_bytes = 0, used = 0, hits = 0, builds = 0;
  // kind: an srt_kind, or kLines / kSolids; obj: srt_accel, srt_line_accel
  // or srt_solid_accel
  struct Entry {
    srt_cache_key key;
    int kind;
    void *obj;
    uint64_t bytes, hit_count;
  };
  std::vector<Entry> static_list, dynamic_list;
};

namespace {

bool same_key(const srt_cache_key &a, const srt_cache_key &b) {
  return a.elem_buffer == b.elem_buffer && a.array_buffer == b.array_buffer &&
         a.position_offset == b.position_offset && a.count == b.count && a.offset == b.offset;
}

// Device bytes an accel holds (tree, order, codes, primitive cache, staging).
uint64_t accel_bytes(const srt_accel *a) {
  return a->nodes.cap + a->indices.cap + a->codes.cap + a->prims.cap + a->scene.cap +
         a->in_verts.cap + a->in_faces.cap + a->in_radius.cap;
}

constexpr int kLines = 3, kSolids = 4;  // cache kinds beyond srt_kind

void destroy_obj(int kind, void *obj) {
  if (kind == kLines)
    srt_line_destroy(static_cast<srt_line_accel *>(obj));
  else if (kind == kSolids)
    srt_solid_destroy(static_cast<srt_solid_accel *>(obj));
  else
    srt_accel_destroy(static_cast<srt_accel *>(obj));
}

uint64_t obj_bytes(int kind, void *obj) {
  if (kind == kLines) return line_accel_bytes(static_cast<srt_line_accel *>(obj));
  if (kind == kSolids) return solid_accel_bytes(static_cast<srt_solid_accel *>(obj));
  return accel_bytes(static_cast<srt_accel *>(obj));
}

void drop(srt_cache *c, srt_cache::Entry &e) {
  c->used -= e.bytes;
  destroy_obj(e.kind, e.obj);
  e.obj = nullptr;
}

// AccelBuilder's Build*Accel: Locate a static entry (the key and kind), else
// create (create(&obj)), build (build(obj)) and keep a new one.
template <typename T, typename Create, typename Build>
srt_status cache_get(srt_cache *c, int kind, const srt_cache_key *key, int is_static, T **out,
                     Create create, Build build) {
  if (!c || !key || !out) return fail(SRT_ERR_INVALID, "NULL argument");
  *out = nullptr;
  // Locate: the static entries only (a dynamic entry lives one frame)
  for (srt_cache::Entry &e : c->static_list)
    if (e.kind == kind && same_key(e.key, *key)) {
      e.hit_count++;
      c->hits++;
      *out = static_cast<T *>(e.obj);
      return SRT_OK;
    }
  T *a = nullptr;
  srt_status s = create(&a);
  if (s != SRT_OK) return s;
  s = build(a);
  if (s != SRT_OK) {
    destroy_obj(kind, a);
    return s;
  }
  srt_cache::Entry e{*key, kind, a, obj_bytes(kind, a), 1};
  c->used += e.bytes;
  c->builds++;
  (is_static ? c->static_list : c->dynamic_list).push_back(e);
  *out = a;
  return SRT_OK;
}

template <typename Build>
srt_status cache_get_accel(srt_cache *c, srt_kind kind, const srt_cache_key *key, int is_static,
                           srt_accel **out, Build build) {
  return cache_get<srt_accel>(
      c, kind, key, is_static, out,
      [&](srt_accel **a) { return srt_accel_create(c->ctx, kind, a); }, build);
}

}  // namespace

extern "C" {

SRT_API srt_status srt_accel_load_triangles(srt_accel *a, const char *path, const float *vertices,
                                            size_t nvertices, const uint32_t *faces,
                                            size_t nfaces) {
  return load_common(a, SRT_TRIANGLES, path, vertices, nvertices, faces, nfaces, 3, nullptr,
                     0.0f);
}

SRT_API srt_status srt_accel_load_tetrahedra(srt_accel *a, const char *path, const float *vertices,
                                             size_t nvertices, const uint32_t *tets,
                                             size_t ntets) {
  return load_common(a, SRT_TETRAHEDRA, path, vertices, nvertices, tets, ntets, 4, nullptr,
                     0.0f);
}

SRT_API srt_status srt_accel_load_spheres(srt_accel *a, const char *path, const float *centers,
                                          const float *radius, float constant_radius, size_t n) {
  return load_common(a, SRT_SPHERES, path, centers, n, nullptr, n, 0, radius, constant_radius);
}

SRT_API srt_status srt_cache_create(srt_ctx *ctx, uint64_t max_bytes, srt_cache **out) {
  if (!ctx || !out) return SRT_ERR_INVALID;
  srt_cache *c = new (std::nothrow) srt_cache();
  if (!c) return SRT_ERR_NO_MEMORY;
  c->ctx = ctx;
  c->max_bytes = max_bytes;
  *out = c;
  return SRT_OK;
}

SRT_API srt_status srt_cache_destroy(srt_cache *c) {
  if (!c) return SRT_OK;
  for (auto &e : c->static_list) drop(c, e);
  for (auto &e : c->dynamic_list) drop(c, e);
  delete c;
  return SRT_OK;
}

SRT_API srt_status srt_cache_build_triangles(srt_cache *c, const srt_cache_key *key,
                                             int is_static, const float *vertices,
                                             size_t nvertices, const uint32_t *faces,
                                             size_t nfaces, srt_accel **out) {
  return cache_get_accel(c, SRT_TRIANGLES, key, is_static, out, [&](srt_accel *a) {
    return srt_accel_build_triangles(a, vertices, nvertices, faces, nfaces);
  });
}

SRT_API srt_status srt_cache_build_tetrahedra(srt_cache *c, const srt_cache_key *key,
                                              int is_static, const float *vertices,
                                              size_t nvertices, const uint32_t *tets,
                                              size_t ntets, srt_accel **out) {
  return cache_get_accel(c, SRT_TETRAHEDRA, key, is_static, out, [&](srt_accel *a) {
    return srt_accel_build_tetrahedra(a, vertices, nvertices, tets, ntets);
  });
}

SRT_API srt_status srt_cache_build_spheres(srt_cache *c, const srt_cache_key *key,
                                           int is_static, const float *centers,
                                           const float *radius, float constant_radius,
                                           size_t n, srt_accel **out) {
  return cache_get_accel(c, SRT_SPHERES, key, is_static, out, [&](srt_accel *a) {
    return srt_accel_build_spheres(a, centers, radius, constant_radius, n);
  });
}

SRT_API srt_status srt_cache_build_lines(srt_cache *c, const srt_cache_key *key, int is_static,
                                        const float *positions, size_t nverts,
                                        const float *radius, float constant_radius,
                                        const uint32_t *segments, size_t nlines, int32_t cap,
                                        srt_line_accel **out) {
  return cache_get<srt_line_accel>(
      c, kLines, key, is_static, out,
      [&](srt_line_accel **a) { return srt_line_create(c->ctx, a); },
      [&](srt_line_accel *a) {
        return srt_line_build(a, positions, nverts, radius, constant_radius, segments, nlines,
                              0, 0, cap);
      });
}

SRT_API srt_status srt_cache_build_solids(srt_cache *c, const srt_cache_key *key, int is_static,
                                         int32_t verts_per_solid, const float *vertices,
                                         size_t nverts, const uint32_t *indices, size_t nsolids,
                                         srt_solid_accel **out) {
  return cache_get<srt_solid_accel>(
      c, kSolids, key, is_static, out,
      [&](srt_solid_accel **a) { return srt_solid_create(c->ctx, a); },
      [&](srt_solid_accel *a) {
        // AccelBuilder::BuildSolidAccel builds with SolidAccel::Build, the
        // binned-SAH build, at every size (gles/gles_accel_builder.cc:967)
        return srt_solid_build_sah(a, verts_per_solid, vertices, nverts, indices, nsolids);
      });
}

SRT_API srt_status srt_cache_invalidate(srt_cache *c, uint64_t buffer) {
  if (!c) return SRT_ERR_INVALID;
  for (auto *list : {&c->static_list, &c->dynamic_list}) {
    std::vector<srt_cache::Entry> keep;
    for (auto &e : *list) {
      if (e.key.elem_buffer == buffer || e.key.array_buffer == buffer)
        drop(c, e);
      else
        keep.push_back(e);
    }
    list->swap(keep);
  }
  return SRT_OK;
}

SRT_API srt_status srt_cache_end_frame(srt_cache *c) {
  if (!c) return SRT_ERR_INVALID;
  for (auto &e : c->dynamic_list) drop(c, e);
  c->dynamic_list.clear();
  return SRT_OK;
}

SRT_API srt_status srt_cache_info_get(srt_cache *c, srt_cache_info *info) {
  if (!c || !info) return SRT_ERR_INVALID;
  memset(info, 0, sizeof(*info));
  info->bytes_used = c->used;
  info->bytes_max = c->max_bytes;
  info->static_entries = c->static_list.size();
  info->dynamic_entries = c->dynamic_list.size();
  info->hits = c->hits;
  info->builds = c->builds;
  return SRT_OK;
}

}  // extern "C"
