// srt_scene.cu -- several accels with transforms traced as one scene: the
// GPU side of RenderGraph (gles/gles_render_graph.cc:104-314).
//
// The caller adds each element (a built accel, its transform T, inverse
// transform invT, inverse of T's upper 3x3 invT33 and world bounding box --
// what RenderElement::Update computes on the host,
// gles/gles_render_graph.cc:77-101) and builds the scene: the top-level
// tree over the world boxes is built here on the host exactly as
// BVHTree::BuildTree / ConstructTree do (render/render_bvh_tree.cc:319-500:
// spatial median on the longest axis with PartitionNodes' in-place order,
// axis retries, object median fallback, child boxes widened by 1e-6 of
// their extent) and uploaded with the element table.  srt_scene_trace then
// runs RenderGraph::Trace for a ray array in one kernel (srt_trace.cu).
#include <vector>

#include "srt_internal.cuh"

using namespace srt;

struct srt_scene {
  srt_ctx *ctx = nullptr;
  struct Elem {
    srt_accel *acc = nullptr;  // or one of:
    srt_line_accel *lines = nullptr;
    srt_solid_accel *solids = nullptr;
    double T[16], invT[16], invT33[16], bmin[3], bmax[3];
  };
  std::vector<Elem> elems;
  std::vector<TopNode> top;
  DevBuf d_top, d_elems, d_rank, scratch;
  bool built = false;
  uint32_t max_iter = 64;
  uint32_t kinds = 0;          // bit k: the scene holds elements of kind k
  uint32_t rank_start[4] = {};  // first rank of triangles, tetrahedra, spheres, lines + solids
  bool deep_lines = false;      // a line element deeper than the loop's short stack
  SceneStreams ss;
  ~srt_scene() {
    for (cudaStream_t &q : ss.side)
      if (q) cudaStreamDestroy(q);
    for (cudaEvent_t &v : ss.fork)
      if (v) cudaEventDestroy(v);
    for (cudaEvent_t &v : ss.join)
      if (v) cudaEventDestroy(v);
  }
};

namespace {

struct TopData {
  double bmin[3], bmax[3];
  uint32_t id;
};

// PartitionNodes (render/render_bvh_tree.cc:83-130): elements whose box
// ends before the split position move to the front, in the reference's
// swap order; returns the split index.
size_t partition(std::vector<TopData> &d, size_t l, size_t r, double pos, int axis) {
  const TopData leftmost = d[l];
  size_t pivot = l;
  for (size_t i = l + 1; i < r; i++) {
    if (d[i].bmax[axis] < pos) {
      pivot++;
      std::swap(d[pivot], d[i]);
    }
  }
  d[l] = d[pivot];
  d[pivot] = leftmost;
  size_t split = l;
  for (size_t i = l; i < r; i++)
    if (d[i].bmax[axis] < pos) split++;
  return split;
}

// CalculateBoundingBox (render/render_bvh_tree.cc:133-152), std::min/max.
void range_box(const std::vector<TopData> &d, size_t s, size_t e, double bmin[3],
               double bmax[3]) {
  for (int k = 0; k < 3; k++) {
    bmin[k] = d[s].bmin[k];
    bmax[k] = d[s].bmax[k];
  }
  for (size_t i = s + 1; i < e; i++)
    for (int k = 0; k < 3; k++) {
      bmin[k] = (d[i].bmin[k] < bmin[k]) ? d[i].bmin[k] : bmin[k];
      bmax[k] = (bmax[k] < d[i].bmax[k]) ? d[i].bmax[k] : bmax[k];
    }
}

TopNode make_node(const double bmin[3], const double bmax[3]) {
  TopNode n{};
  for (int k = 0; k < 3; k++) {
    n.bmin[k] = bmin[k];
    n.bmax[k] = bmax[k];
  }
  return n;
}

void construct(std::vector<TopNode> &nt, std::vector<TopData> &d, size_t root, size_t l,
               size_t r) {
  static const int axis_list[3][3] = {{0, 1, 2}, {1, 2, 0}, {2, 0, 1}};
  const size_t n = r - l;
  if (n == 1) {
    nt[root].leaf = 1;
    nt[root].child[0] = nt[root].child[1] = 0;
    nt[root].id = d[l].id;
    return;
  }
  double bsize[3], bmin[3];
  for (int k = 0; k < 3; k++) {
    bsize[k] = nt[root].bmax[k] - nt[root].bmin[k];
    bmin[k] = nt[root].bmin[k];
  }
  double maxlen = bsize[0];
  int axis_try = 0;
  if (maxlen < bsize[1]) {
    maxlen = bsize[1];
    axis_try = 1;
  }
  if (maxlen < bsize[2]) {
    maxlen = bsize[2];
    axis_try = 2;
  }
  size_t split = l, nleft = 0, nright = n;
  int axis = 0;
  for (int i = 0; i < 3; i++) {
    axis = axis_list[axis_try][i];
    const double pos = bmin[axis] + bsize[axis] * 0.5;
    split = partition(d, l, r, pos, axis);
    if (split != l && split != r) {
      nleft = split - l;
      nright = n - nleft;
      break;
    }
  }
  if (split == l || split == r) {  // no spatial split: object median
    nleft = n / 2;
    nright = n - nleft;
    split = l + (r - l) / 2;
  }
  nt[root].axis = axis;
  nt[root].leaf = 0;
  const double eps = 1.0e-6;
  for (int side = 0; side < 2; side++) {
    const size_t cnt = side == 0 ? nleft : nright;
    if (cnt == 0) {
      nt[root].child[side] = 0;
      continue;
    }
    const size_t s = side == 0 ? l : split, e = side == 0 ? split : r;
    double cb[3], ce[3];
    range_box(d, s, e, cb, ce);
    for (int k = 0; k < 3; k++) {  // widened by 1e-6 of the extent
      const double ext = ce[k] - cb[k];
      cb[k] = cb[k] - ext * eps;
      ce[k] = ce[k] + ext * eps;
    }
    const size_t child = nt.size();
    nt[root].child[side] = (int32_t)child;
    nt.push_back(make_node(cb, ce));
    construct(nt, d, child, s, e);
  }
}

// Matrixd::Inverse (render/render_matrix.h:40-134): the cofactor inverse
// (Cramer's rule) of Intel's SSE note "Inverse of 4x4 Matrix", with the
// products and sums in that routine's order so that the doubles round the
// same way.  s = m transposed; each entry is (three pair products) minus
// (three pair products), the pairs taken from the lower half of s for rows
// 0-1 and from the upper half for rows 2-3.  The reference's term for m[3][3]
// reads s[0] where the note has s[10]; it is kept (MultV never reads m[3][3]).
void inverse4(double m[16]) {
  double s[16];
  for (int r = 0; r < 4; r++)
    for (int c = 0; c < 4; c++) s[4 * c + r] = m[4 * r + c];
  static const unsigned char pair_lo[12][2] = {{10, 15}, {11, 14}, {9, 15}, {11, 13},
                                               {9, 14},  {10, 13}, {8, 15}, {11, 12},
                                               {8, 14},  {10, 12}, {8, 13}, {9, 12}};
  // per entry: 3 (pair, s) products added, then 3 subtracted
  static const unsigned char terms[16][6][2] = {
      {{0, 5}, {3, 6}, {4, 7}, {1, 5}, {2, 6}, {5, 7}},
      {{1, 4}, {6, 6}, {9, 7}, {0, 4}, {7, 6}, {8, 7}},
      {{2, 4}, {7, 5}, {10, 7}, {3, 4}, {6, 5}, {11, 7}},
      {{5, 4}, {8, 5}, {11, 6}, {4, 4}, {9, 5}, {10, 6}},
      {{1, 1}, {2, 2}, {5, 3}, {0, 1}, {3, 2}, {4, 3}},
      {{0, 0}, {7, 2}, {8, 3}, {1, 0}, {6, 2}, {9, 3}},
      {{3, 0}, {6, 1}, {11, 3}, {2, 0}, {7, 1}, {10, 3}},
      {{4, 0}, {9, 1}, {10, 2}, {5, 0}, {8, 1}, {11, 2}},
      {{0, 13}, {3, 14}, {4, 15}, {1, 13}, {2, 14}, {5, 15}},
      {{1, 12}, {6, 14}, {9, 15}, {0, 12}, {7, 14}, {8, 15}},
      {{2, 12}, {7, 13}, {10, 15}, {3, 12}, {6, 13}, {11, 15}},
      {{5, 12}, {8, 13}, {11, 14}, {4, 12}, {9, 13}, {10, 14}},
      {{2, 10}, {5, 11}, {1, 9}, {4, 11}, {0, 9}, {3, 10}},
      {{8, 11}, {0, 8}, {7, 10}, {6, 10}, {9, 11}, {1, 8}},
      {{6, 9}, {11, 11}, {3, 8}, {10, 11}, {2, 8}, {7, 9}},
      {{10, 10}, {4, 8}, {9, 9}, {8, 9}, {11, 0}, {5, 8}}};
  double pr[12];
  for (int half = 0; half < 2; half++) {
    const int off = half ? -8 : 0;  // upper pairs: the same pattern 8 lower in s
    for (int k = 0; k < 12; k++)
      pr[k] = s[pair_lo[k][0] + off] * s[pair_lo[k][1] + off];
    for (int e = 8 * half; e < 8 * half + 8; e++) {
      const unsigned char(*t)[2] = terms[e];
      const double add = pr[t[0][0]] * s[t[0][1]] + pr[t[1][0]] * s[t[1][1]] +
                         pr[t[2][0]] * s[t[2][1]];
      const double sub = pr[t[3][0]] * s[t[3][1]] + pr[t[4][0]] * s[t[4][1]] +
                         pr[t[5][0]] * s[t[5][1]];
      m[e] = add - sub;
    }
  }
  const double det = s[0] * m[0] + s[1] * m[1] + s[2] * m[2] + s[3] * m[3];
  const double rdet = 1.0 / det;
  for (int e = 0; e < 16; e++) m[e] *= rdet;
}

// RenderElement::Update (gles/gles_render_graph.cc:17-101): the world box of
// the local box's eight corners under T (TransformBoundingBox, std::min /
// std::max with the corner first), invT = T^-1 and invT33 = the inverse of T
// with its translation row cleared.
void element_update(const double T[16], const double lbmin[3], const double lbmax[3],
                    double invT[16], double invT33[16], double wbmin[3], double wbmax[3]) {
  for (int c = 0; c < 8; c++) {
    const double v[3] = {(c & 1) ? lbmax[0] : lbmin[0], (c & 2) ? lbmax[1] : lbmin[1],
                         (c & 4) ? lbmax[2] : lbmin[2]};
    double x[3];
    for (int k = 0; k < 3; k++) x[k] = T[k] * v[0] + T[4 + k] * v[1] + T[8 + k] * v[2] + T[12 + k];
    for (int k = 0; k < 3; k++) {
      if (c == 0) {
        wbmin[k] = wbmax[k] = x[k];
      } else {
        wbmin[k] = (wbmin[k] < x[k]) ? wbmin[k] : x[k];
        wbmax[k] = (x[k] < wbmax[k]) ? wbmax[k] : x[k];
      }
    }
  }
  for (int k = 0; k < 16; k++) invT[k] = invT33[k] = T[k];
  inverse4(invT);
  invT33[12] = invT33[13] = invT33[14] = 0.0;
  inverse4(invT33);
}

}  // namespace

namespace srt {
// BVHTree::BuildTree over n boxes (element or block ids 0..n-1).
void build_top_tree(const double *bmin, const double *bmax, size_t n,
                    std::vector<TopNode> &out) {
  std::vector<TopData> d(n);
  for (size_t i = 0; i < n; i++) {
    for (int k = 0; k < 3; k++) {
      d[i].bmin[k] = bmin[3 * i + k];
      d[i].bmax[k] = bmax[3 * i + k];
    }
    d[i].id = (uint32_t)i;
  }
  double lo[3], hi[3];
  range_box(d, 0, n, lo, hi);  // CalcSceneBBox (render/render_bvh_tree.cc:155-170)
  out.clear();
  out.push_back(make_node(lo, hi));
  construct(out, d, 0, 0, n);
}
}  // namespace srt

extern "C" {

SRT_API void srt_matrix_inverse(double m[16]) { inverse4(m); }

SRT_API srt_status srt_scene_create(srt_ctx *ctx, srt_scene **out) {
  if (!ctx || !out) return SRT_ERR_INVALID;
  srt_scene *s = new (std::nothrow) srt_scene();
  if (!s) return SRT_ERR_NO_MEMORY;
  s->ctx = ctx;
  cudaError_t e = cudaSetDevice(ctx->device);
  for (int k = 0; k < 4 && e == cudaSuccess; k++)
    e = cudaStreamCreateWithFlags(&s->ss.side[k], cudaStreamNonBlocking);
  for (int k = 0; k < 3 && e == cudaSuccess; k++)
    e = cudaEventCreateWithFlags(&s->ss.fork[k], cudaEventDisableTiming);
  for (int k = 0; k < 4 && e == cudaSuccess; k++)
    e = cudaEventCreateWithFlags(&s->ss.join[k], cudaEventDisableTiming);
  if (e != cudaSuccess) {
    delete s;
    return cuda_status(e, "scene streams");
  }
  *out = s;
  return SRT_OK;
}

SRT_API srt_status srt_scene_destroy(srt_scene *s) {
  if (!s) return SRT_OK;
  cudaSetDevice(s->ctx->device);
  cudaStreamSynchronize(s->ctx->stream);
  for (cudaStream_t q : s->ss.side)
    if (q) cudaStreamSynchronize(q);
  delete s;
  return SRT_OK;
}

}  // extern "C"

namespace {

// Appends element e (its accel pointer set) with the caller's matrices and
// world box.
srt_status scene_push(srt_scene *s, srt_scene::Elem e, const double T[16], const double invT[16],
                      const double invT33[16], const double world_bmin[3],
                      const double world_bmax[3], uint32_t *id) {
  for (int k = 0; k < 16; k++) {
    e.T[k] = T[k];
    e.invT[k] = invT[k];
    e.invT33[k] = invT33[k];
  }
  for (int k = 0; k < 3; k++) {
    e.bmin[k] = world_bmin[k];
    e.bmax[k] = world_bmax[k];
  }
  if (id) *id = (uint32_t)s->elems.size();
  s->elems.push_back(e);
  s->built = false;
  return SRT_OK;
}

// RenderElement's constructor for an element with local box lbmin / lbmax.
srt_status scene_push_update(srt_scene *s, const srt_scene::Elem &e, const double T[16],
                             const double lbmin[3], const double lbmax[3], uint32_t *id) {
  double invT[16], invT33[16], wbmin[3], wbmax[3];
  element_update(T, lbmin, lbmax, invT, invT33, wbmin, wbmax);
  return scene_push(s, e, T, invT, invT33, wbmin, wbmax, id);
}

}  // namespace

extern "C" {

SRT_API srt_status srt_scene_add(srt_scene *s, srt_accel *acc, const double T[16],
                                 const double invT[16], const double invT33[16],
                                 const double world_bmin[3], const double world_bmax[3],
                                 uint32_t *id) {
  if (!s || !acc || !T || !invT || !invT33 || !world_bmin || !world_bmax) {
    set_error("NULL argument");
    return SRT_ERR_INVALID;
  }
  if (!acc->built || acc->ctx != s->ctx) {
    set_error("scene elements must be built accels of the scene's context");
    return SRT_ERR_INVALID;
  }
  srt_scene::Elem e;
  e.acc = acc;
  return scene_push(s, e, T, invT, invT33, world_bmin, world_bmax, id);
}

SRT_API srt_status srt_scene_add_element(srt_scene *s, srt_accel *acc, const double T[16],
                                         uint32_t *id) {
  if (!s || !acc || !T) {
    set_error("NULL argument");
    return SRT_ERR_INVALID;
  }
  if (!acc->built || acc->ctx != s->ctx) {
    set_error("scene elements must be built accels of the scene's context");
    return SRT_ERR_INVALID;
  }
  double lbmin[3], lbmax[3];
  srt_status st = srt_accel_bbox(acc, lbmin, lbmax);
  if (st != SRT_OK) return st;
  srt_scene::Elem e;
  e.acc = acc;
  return scene_push_update(s, e, T, lbmin, lbmax, id);
}

SRT_API srt_status srt_scene_add_lines(srt_scene *s, srt_line_accel *acc, const double T[16],
                                       uint32_t *id) {
  if (!s || !acc || !T) {
    set_error("NULL argument");
    return SRT_ERR_INVALID;
  }
  srt_ctx *c = nullptr;
  SceneElem v{};
  int depth = 0;
  if (!line_scene_view(acc, &c, v, depth) || c != s->ctx) {
    set_error("scene elements must be built accels of the scene's context");
    return SRT_ERR_INVALID;
  }
  double lbmin[3], lbmax[3];
  srt_status st = srt_line_bbox(acc, lbmin, lbmax);
  if (st != SRT_OK) return st;
  srt_scene::Elem e;
  e.lines = acc;
  return scene_push_update(s, e, T, lbmin, lbmax, id);
}

SRT_API srt_status srt_scene_add_solids(srt_scene *s, srt_solid_accel *acc, const double T[16],
                                        uint32_t *id) {
  if (!s || !acc || !T) {
    set_error("NULL argument");
    return SRT_ERR_INVALID;
  }
  srt_ctx *c = nullptr;
  SceneElem v{};
  bool deep = false;
  if (!solid_scene_view(acc, &c, v, deep) || c != s->ctx) {
    set_error("scene elements must be built accels of the scene's context");
    return SRT_ERR_INVALID;
  }
  double lbmin[3], lbmax[3];
  srt_status st = srt_solid_bbox(acc, lbmin, lbmax);
  if (st != SRT_OK) return st;
  srt_scene::Elem e;
  e.solids = acc;
  return scene_push_update(s, e, T, lbmin, lbmax, id);
}

SRT_API srt_status srt_scene_build(srt_scene *s) {
  if (!s) return SRT_ERR_INVALID;
  if (s->elems.empty()) {
    set_error("empty scene");
    return SRT_ERR_INVALID;
  }
  std::vector<double> lo(3 * s->elems.size()), hi(3 * s->elems.size());
  for (size_t i = 0; i < s->elems.size(); i++)
    for (int k = 0; k < 3; k++) {
      lo[3 * i + k] = s->elems[i].bmin[k];
      hi[3 * i + k] = s->elems[i].bmax[k];
    }
  build_top_tree(lo.data(), hi.data(), s->elems.size(), s->top);
  std::vector<SceneElem> el(s->elems.size());
  size_t total = 0;
  uint32_t kinds = 0;
  bool deep = false;
  for (size_t i = 0; i < el.size(); i++) {
    const srt_scene::Elem &se = s->elems[i];
    srt_ctx *c = nullptr;
    bool ok;
    if (se.lines) {
      int depth = 0;
      ok = line_scene_view(se.lines, &c, el[i], depth);
      deep = deep || depth + 2 > 64;
    } else if (se.solids) {
      bool sdeep = false;
      ok = solid_scene_view(se.solids, &c, el[i], sdeep);
      deep = deep || sdeep;
    } else {
      const srt_accel *a = se.acc;
      ok = a->built;
      el[i].kind = a->kind;
      el[i].nprims = (uint32_t)a->n;
      el[i].aux = a->dbl ? kTetAuxDouble : 0;
      el[i].nodes = a->nodes.p;
      el[i].prims = a->prims.as<float4>();
      el[i].sidx = a->indices.as<uint32_t>();
      el[i].scene = a->scene.as<SceneInfo>();
    }
    if (!ok) {
      set_error("scene element not built");
      return SRT_ERR_INVALID;
    }
    for (int k = 0; k < 16; k++) {
      el[i].T[k] = s->elems[i].T[k];
      el[i].invT[k] = s->elems[i].invT[k];
      el[i].invT33[k] = s->elems[i].invT33[k];
    }
    total += el[i].nprims;
    kinds |= 1u << el[i].kind;
  }
  cudaSetDevice(s->ctx->device);
  cudaError_t e;
  // element ranks: ids grouped by kind (triangles, tetrahedra, spheres,
  // then lines and solids), each group in id order -- the trace sorts its
  // items by rank, so each kind's items form one range; lines and solids
  // (ranks from rank_start[3] on) are walked by the per-ray loop only
  std::vector<uint32_t> rank(el.size());
  uint32_t r = 0;
  for (int k = 0; k < 5; k++) {
    if (k < 4) s->rank_start[k] = r;
    for (size_t i = 0; i < el.size(); i++)
      if (el[i].kind == k) rank[i] = r++;
  }
  if (r != el.size()) {
    set_error("scene element of unknown kind");
    return SRT_ERR_INVALID;
  }
  if ((e = s->d_top.ensure(s->top.size() * sizeof(TopNode))) != cudaSuccess ||
      (e = s->d_elems.ensure(el.size() * sizeof(SceneElem))) != cudaSuccess ||
      (e = s->d_rank.ensure(rank.size() * sizeof(uint32_t))) != cudaSuccess)
    return cuda_status(e, "scene tables");
  cudaStream_t st = s->ctx->stream;
  e = cudaMemcpyAsync(s->d_top.p, s->top.data(), s->top.size() * sizeof(TopNode),
                      cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(s->d_elems.p, el.data(), el.size() * sizeof(SceneElem),
                        cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(s->d_rank.p, rank.data(), rank.size() * sizeof(uint32_t),
                        cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);  // host tables go out of scope
  if (e != cudaSuccess) return cuda_status(e, "scene upload");
  s->max_iter = (uint32_t)std::min<size_t>(8 * total + 64 + 8 * s->top.size(), 0xfffffff0u);
  s->kinds = kinds;
  s->deep_lines = deep;
  s->built = true;
  return SRT_OK;
}

SRT_API size_t srt_scene_top_nodes(srt_scene *s, double *boxes, int32_t *ints, size_t cap) {
  if (!s || !s->built) return 0;
  for (size_t i = 0; i < s->top.size() && i < cap; i++) {
    for (int k = 0; k < 3; k++) {
      if (boxes) {
        boxes[6 * i + k] = s->top[i].bmin[k];
        boxes[6 * i + 3 + k] = s->top[i].bmax[k];
      }
    }
    if (ints) {
      ints[5 * i + 0] = s->top[i].child[0];
      ints[5 * i + 1] = s->top[i].child[1];
      ints[5 * i + 2] = s->top[i].axis;
      ints[5 * i + 3] = s->top[i].leaf;
      ints[5 * i + 4] = (int32_t)s->top[i].id;
    }
  }
  return s->top.size();
}

SRT_API srt_status srt_scene_trace(srt_scene *s, const srt_ray *rays, size_t n,
                                   const uint32_t *prev_element, const float *prev_normals,
                                   srt_hit *hits, uint32_t *element, uint64_t *stats) {
  if (!s || (n && (!rays || !hits))) {
    set_error("NULL argument");
    return SRT_ERR_INVALID;
  }
  if (!s->built) {
    set_error("scene not built");
    return SRT_ERR_INVALID;
  }
  if (n == 0) return SRT_OK;
  srt_ctx *ctx = s->ctx;
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_status(e, "set device");
  if (!is_device_ptr(rays) || !is_device_ptr(hits) ||
      (prev_element && !is_device_ptr(prev_element)) ||
      (prev_normals && !is_device_ptr(prev_normals)) || (element && !is_device_ptr(element)) ||
      (stats && !is_device_ptr(stats))) {
    set_error("srt_scene_trace: all arrays must be device memory");
    return SRT_ERR_INVALID;
  }
  if ((reinterpret_cast<uintptr_t>(rays) | reinterpret_cast<uintptr_t>(hits)) & 15u) {
    set_error("ray and hit arrays must be 16-byte aligned");
    return SRT_ERR_INVALID;
  }
  if (n >= (1ull << 29)) {  // the phase-1 items n * 7 are 32-bit indices
    set_error("srt_scene_trace: at most 2^29 - 1 rays per call");
    return SRT_ERR_LIMIT;
  }
  // scratch sections (each 256-byte aligned): candidates, nearest distance,
  // candidate counts, sort keys and values of both phases, phase-1 results,
  // overflow list, counters, kind bounds
  auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
  const size_t ne = s->elems.size();
  const size_t nk = n * kRoundCand, n1 = n * (kRoundCand - 1);
  const size_t b_ct = al(nk * sizeof(double)), b_ce = al(nk * 4), b_tn = al(n * 4),
               b_nc = al(n), b_k0 = al(n * 4), b_k1 = al(n1 * 4),
               b_res = al(nk * sizeof(float4)), b_dl = al(n1 * sizeof(Deferred)),
               b_ovf = al(n * 4), b_cnt = al(kSceneCounters * 4), b_bd = al(8 * 4);
  e = s->scratch.ensure(b_ct + b_ce + b_tn + b_nc + 2 * b_k0 + 2 * b_k1 + b_res + b_dl + b_ovf +
                        b_cnt + b_bd);
  if (e != cudaSuccess) return cuda_status(e, "scene trace scratch");
  char *p = s->scratch.as<char>();
  auto take = [&p](size_t bytes) {
    char *q = p;
    p += bytes;
    return q;
  };
  SceneWork W;
  W.elems = s->d_elems.as<SceneElem>();
  W.elem_rank = s->d_rank.as<uint32_t>();
  W.nelem = (uint32_t)ne;
  for (int k = 0; k < 4; k++) W.rank_start[k] = s->rank_start[k];
  W.rays = rays;
  W.prev_element = prev_element;
  W.prev_normals = prev_normals;
  W.hits = hits;
  W.element = element;
  W.cand_t = reinterpret_cast<double *>(take(b_ct));
  W.cand_e = reinterpret_cast<uint32_t *>(take(b_ce));
  W.tnear = reinterpret_cast<float *>(take(b_tn));
  W.ncand = reinterpret_cast<uint8_t *>(take(b_nc));
  W.keys0 = reinterpret_cast<uint32_t *>(take(b_k0));
  W.vals0 = reinterpret_cast<uint32_t *>(take(b_k0));
  W.keys1 = reinterpret_cast<uint32_t *>(take(b_k1));
  W.vals1 = reinterpret_cast<uint32_t *>(take(b_k1));
  W.res = reinterpret_cast<float4 *>(take(b_res));
  W.dlist = reinterpret_cast<Deferred *>(take(b_dl));
  W.ovf = reinterpret_cast<uint32_t *>(take(b_ovf));
  W.counters = reinterpret_cast<uint32_t *>(take(b_cnt));
  W.bounds = reinterpret_cast<uint32_t *>(take(b_bd));
  W.n = n;
  W.max_iter = s->max_iter;
  W.stats = reinterpret_cast<unsigned long long *>(stats);
  W.err = ctx->d_err;
  return launch_scene_trace(ctx, s->d_top.as<TopNode>(), W, s->kinds, s->deep_lines, s->ss);
}

}  // extern "C"
