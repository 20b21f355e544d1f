// srt_volume.cu -- emission-absorption volume march and its adjoint.
//
// Geometry follows the reference shader (examples/nonuniform_volume_render/
// input.frag): build_cameraframe with pi written as 3.14 (:16-29), a ray
// through each fragment centre (:101-108), the IntersectP slab test against
// [-1,1]^3 with +-10000 initial bounds (:59-97), the half-open inside() test
// (:50-57) and texture3D(tex0, 0.5*p + 0.5) fetched with FilterTexture3DFloat's
// texel-corner trilinear weights (render/render_texture.cc:946-1058, vox =
// u*(dim-1)).  Compositing is front-to-back emission-absorption, samples at
// t0 + (s + 1/2) * step for s < floor((t1 - t0) / step):
//   rgba = lerp of the transfer function at rho*(entries-1)
//   alpha = min(1 - exp(-sigma_scale * rgba.a * step), alpha_max)
//   C += T * alpha * rgba.rgb;  T *= 1 - alpha;  output (C, 1 - T)
// The adjoint walks the samples in reverse and rebuilds transmittance as
// T_k = T_{k+1} / (1 - alpha_k) from the stored final T (no per-sample
// state); alpha_max < 1 keeps the division bounded.
#include <cmath>
#include <cstring>

#include "srt_internal.cuh"

namespace srt {
namespace {

struct VolConst {
  srt_volume_params p;
  int dim[3];
  int tfn;
  // sampling state of the density texture: per-axis coordinate remap of a
  // non-uniform volume and clamp-to-edge (else repeat) per axis
  const float *remap[3];
  int nremap[3];
  int clamp[3];
};

// The fetch coordinate of axis k: local::remap (gles/gles_common.h:264-269)
// then the repeat wrap of FilterTexture3DFloat unless clamp-to-edge.
__device__ __forceinline__ float tex_coord(const VolConst &K, int k, float u) {
  if (K.nremap[k]) {
    const int nk = K.nremap[k];
    int idx = f2i_x86(u * (float)nk);
    idx = max(min(nk - 1, idx), 0);
    u = __ldg(&K.remap[k][idx]);
  }
  if (!K.clamp[k]) u = u - (float)floor_ref(u);
  return u;
}

// Lower texel corner (clamped) and trilinear fractions of a fetch.
struct Cell {
  int vx, vy, vz;
  float dx, dy, dz;
};

// Pixel of thread index `idx`: each warp covers an 8x4 tile (blocks of 128
// threads a 16x8 tile) so the rays of a warp sample neighbouring voxels.
__device__ __forceinline__ bool tile_pixel(int idx, int W, int H, int &px, int &py) {
  const int lane = idx & 31, warp = idx >> 5;
  const int tiles_x = (W + 7) >> 3;
  const int tx = warp % tiles_x, ty = warp / tiles_x;
  px = tx * 8 + (lane & 7);
  py = ty * 4 + (lane >> 3);
  return px < W && py < H;
}

__device__ __forceinline__ float lerpf(float t, float a, float b) {
  return (1.f - t) * a + t * b;
}

__device__ __forceinline__ void pixel_ray(const srt_volume_params &P, int px, int py,
                                          float o[3], float d[3]) {
  const float fx = (float)px + 0.5f, fy = (float)py + 0.5f;
  float v[3];
#pragma unroll
  for (int k = 0; k < 3; k++) v[k] = (P.corner[k] + fx * P.du[k] + fy * P.dv[k]) - P.eye[k];
  const float l = sqrtf(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
#pragma unroll
  for (int k = 0; k < 3; k++) {
    d[k] = v[k] / l;
    o[k] = P.eye[k];
  }
}

__device__ __forceinline__ bool slab(const float o[3], const float d[3], float &t0,
                                     float &t1) {
  t0 = -10000.0f;
  t1 = 10000.0f;
#pragma unroll
  for (int k = 0; k < 3; k++) {
    float tn = (-1.0f - o[k]) / d[k];
    float tf = (1.0f - o[k]) / d[k];
    if (tn > tf) {
      float x = tn;
      tn = tf;
      tf = x;
    }
    t0 = tn > t0 ? tn : t0;
    t1 = tf < t1 ? tf : t1;
  }
  return t0 <= t1;
}

__device__ __forceinline__ bool inside(const float p[3]) {
  return p[0] >= -1.0f && p[0] < 1.0f && p[1] >= -1.0f && p[1] < 1.0f && p[2] >= -1.0f &&
         p[2] < 1.0f;
}

// FilterTexture3DFloat, clamp-to-edge, one component.  Voxel indices are
// 32-bit: make_const rejects volumes of 2^31 voxels or more.
__device__ __forceinline__ float fetch(const float *__restrict__ img, const int dim[3],
                                       float u, float v, float r, Cell *cell) {
  const float vox0 = u * (dim[0] - 1.0f);
  const float vox1 = v * (dim[1] - 1.0f);
  const float vox2 = r * (dim[2] - 1.0f);
  const int vx = min(max((int)vox0, 0), dim[0] - 1);
  const int vy = min(max((int)vox1, 0), dim[1] - 1);
  const int vz = min(max((int)vox2, 0), dim[2] - 1);
  const int sy = dim[0], sz = dim[0] * dim[1];
  const int ox = vx + 1 < dim[0] ? 1 : 0;
  const int oy = vy + 1 < dim[1] ? sy : 0;
  const int oz = vz + 1 < dim[2] ? sz : 0;
  const float dx = vox0 - vx, dy = vox1 - vy, dz = vox2 - vz;
  const float *q = img + (vz * sz + vy * sy + vx);
  const float D000 = __ldg(q);
  const float D100 = __ldg(q + ox);
  const float D010 = __ldg(q + oy);
  const float D110 = __ldg(q + oy + ox);
  const float D001 = __ldg(q + oz);
  const float D101 = __ldg(q + oz + ox);
  const float D011 = __ldg(q + oz + oy);
  const float D111 = __ldg(q + oz + oy + ox);
  const float d00 = lerpf(dx, D000, D100);
  const float d10 = lerpf(dx, D010, D110);
  const float d01 = lerpf(dx, D001, D101);
  const float d11 = lerpf(dx, D011, D111);
  const float d0 = lerpf(dy, d00, d10);
  const float d1 = lerpf(dy, d01, d11);
  const float val = lerpf(dz, d0, d1);
  if (cell) {
    cell->vx = vx;
    cell->vy = vy;
    cell->vz = vz;
    cell->dx = dx;
    cell->dy = dy;
    cell->dz = dz;
  }
  return val;
}

// Transfer-function lookup: returns rgba, sets i0/i1/f and whether rho was
// inside the table's range (clamped samples have no density gradient).
// (SHARED: the table is a shared-memory copy, else global memory.)
template <bool SHARED = false>
__device__ __forceinline__ void tf_lookup_ab(const float4 *__restrict__ tf, int tfn,
                                             float rho, float4 &c, int &i0, int &i1,
                                             float &f, bool &inrange, float4 &a, float4 &b) {
  const float top = (float)(tfn - 1);
  float x = rho * top;
  inrange = (x > 0.0f) && (x < top);
  x = x < 0.0f ? 0.0f : (x > top ? top : x);
  i0 = (int)x;
  i1 = min(i0 + 1, tfn - 1);
  f = x - (float)i0;
  a = SHARED ? tf[i0] : __ldg(&tf[i0]);
  b = SHARED ? tf[i1] : __ldg(&tf[i1]);
  c = make_float4(lerpf(f, a.x, b.x), lerpf(f, a.y, b.y), lerpf(f, a.z, b.z),
                  lerpf(f, a.w, b.w));
}

__device__ __forceinline__ void tf_lookup(const float4 *__restrict__ tf, int tfn,
                                          float rho, float4 &c, int &i0, int &i1,
                                          float &f, bool &inrange) {
  float4 a, b;
  tf_lookup_ab(tf, tfn, rho, c, i0, i1, f, inrange, a, b);
}

__global__ void __launch_bounds__(128)
vol_fwd_kernel(const VolConst K, const float *__restrict__ dens,
               const float4 *__restrict__ tf, float4 *__restrict__ image,
               float *__restrict__ trans) {
  const int W = K.p.width, H = K.p.height;
  int px, py;
  if (!tile_pixel(blockIdx.x * blockDim.x + threadIdx.x, W, H, px, py)) return;
  const int pix = py * W + px;
  float o[3], d[3], t0, t1;
  pixel_ray(K.p, px, py, o, d);
  float C0 = 0.f, C1 = 0.f, C2 = 0.f, T = 1.0f;
  if (slab(o, d, t0, t1)) {
    int ns = (int)((t1 - t0) / K.p.step);
    if (ns > K.p.max_steps) ns = K.p.max_steps;
    for (int s = 0; s < ns; s++) {
      const float t = t0 + ((float)s + 0.5f) * K.p.step;
      const float p[3] = {o[0] + t * d[0], o[1] + t * d[1], o[2] + t * d[2]};
      if (!inside(p)) continue;
      const float rho = fetch(dens, K.dim, tex_coord(K, 0, 0.5f * p[0] + 0.5f),
                              tex_coord(K, 1, 0.5f * p[1] + 0.5f),
                              tex_coord(K, 2, 0.5f * p[2] + 0.5f), nullptr);
      float4 c;
      int i0, i1;
      float f;
      bool inr;
      tf_lookup(tf, K.tfn, rho, c, i0, i1, f, inr);
      const float sig = K.p.sigma_scale * c.w;
      float al = 1.0f - expf(-sig * K.p.step);
      if (al > K.p.alpha_max) al = K.p.alpha_max;
      const float w = T * al;
      C0 += w * c.x;
      C1 += w * c.y;
      C2 += w * c.z;
      T = T * (1.0f - al);
    }
  }
  image[pix] = make_float4(C0, C1, C2, 1.0f - T);
  if (trans) trans[pix] = T;
}

constexpr int kTfCopies = 4;  // copies of the block-local TF gradient

// Scale of the block's fixed-point accumulators.  An entry's colour
// gradient is the sum over the block's rays of g.c times the ray's weight
// on the entry; a ray's weights are compositing weights, which sum to at
// most 1 - T <= 1, so every partial sum is bounded by bound = the sum over
// the rays of max_c |g.c|.  The scale 2^29 / bound (a power of two: scaling
// and the final division are exact) leaves 2x headroom for the rounding of
// the reconstructed weights and the per-term rounding below 2^31; the
// resolution is bound * 2^-29.  Shared-memory integer adds are native, float
// adds are not, and the block's sums in integers are exact.
__device__ __forceinline__ float colour_scale(float bound) {
  int e;
  frexpf(bound, &e);  // bound in [2^(e-1), 2^e)
  return ldexpf(1.0f, 29 - max(e, -90));
}

// The opacity part of an entry's gradient sums the samples' gc3 = ga * sstep
// * e (0 where alpha is clamped) times their interpolation weights.  With
// G = sum_c |g.c|, cm the table's largest |colour| component and
// iom * e = 1 (e = 1 - alpha unclamped), |ga| <= Tk G cm + iom (G cm + |g.w|)
// gives |gc3| <= sstep (2 G cm + |g.w|) per sample (Tk e <= 1), so the
// ray's sum is bounded by ns sstep (2 G cm + |g.w|) and the block's by the
// sum of that over its rays: the opacity accumulators' bound, scaled as the
// colour ones.

// |x|, or infinity when x is not finite (NaN included).
__device__ __forceinline__ float abs_or_inf(float x) {
  const float a = fabsf(x);
  return a <= FLT_MAX ? a : __int_as_float(0x7f800000);
}

// Transfer-function gradient of one table entry added to the block's
// shared copy: the colour part is the ray's image gradient g (constant along
// the ray) times the run's summed weight a.x, in fixed point at scale
// cscale, the opacity part a.y in fixed point at scale oscale (float adds
// where a scale is 0: a block whose bound is not finite, or zero).
__device__ __forceinline__ void flush_entry(float *g, int i, float2 &a, const float4 &gi,
                                            float cscale, float oscale) {
  if (a.x != 0.0f) {
    if (cscale != 0.0f) {
      int *q = reinterpret_cast<int *>(g) + 4 * i;
      const float w = a.x * cscale;
      if (gi.x != 0.0f) atomicAdd(q, __float2int_rn(w * gi.x));
      if (gi.y != 0.0f) atomicAdd(q + 1, __float2int_rn(w * gi.y));
      if (gi.z != 0.0f) atomicAdd(q + 2, __float2int_rn(w * gi.z));
    } else {
      if (gi.x != 0.0f) atomicAdd(&g[4 * i], a.x * gi.x);
      if (gi.y != 0.0f) atomicAdd(&g[4 * i + 1], a.x * gi.y);
      if (gi.z != 0.0f) atomicAdd(&g[4 * i + 2], a.x * gi.z);
    }
  }
  if (a.y != 0.0f) {
    if (oscale != 0.0f)
      atomicAdd(reinterpret_cast<int *>(g) + 4 * i + 3, __float2int_rn(a.y * oscale));
    else
      atomicAdd(&g[4 * i + 3], a.y);
  }
  a = make_float2(0.0f, 0.0f);
}

// Add the eight corner sums of one texel cell to the density gradient: its
// lower corner's index `key` and, in `edge`, whether the cell sits on the
// last texel of x (bit 0), y (bit 1), z (bit 2), where the fetch clamps the
// upper corner onto the lower one.
__device__ __forceinline__ void flush_dens(float *__restrict__ g, const int dim[3], int key,
                                           int edge, float (&a)[8]) {
  const int ox = (edge & 1) ? 0 : 1;
  const int oy = (edge & 2) ? 0 : dim[0];
  const int oz = (edge & 4) ? 0 : dim[0] * dim[1];
  float *q = g + key;
#pragma unroll
  for (int k = 0; k < 8; k++) {
    const int off = ((k & 1) ? ox : 0) + ((k & 2) ? oy : 0) + ((k & 4) ? oz : 0);
    atomicAdd(q + off, a[k]);
    a[k] = 0.0f;
  }
}
constexpr int kTfMax = 1024;  // kTfCopies * (4 * kTfMax + 1) floats of shared memory

__global__ void __launch_bounds__(128, 8)
vol_bwd_kernel(const VolConst K, const float *__restrict__ dens,
               const float4 *__restrict__ tf, const float *__restrict__ trans,
               const float4 *__restrict__ gimg, float *__restrict__ gdens,
               float *__restrict__ gtf) {
  // Block-local transfer-function gradient in kTfCopies copies, lane-hashed
  // so that lanes accumulating into the same entry hit different copies;
  // copies are padded by one word to fall on different banks.
  extern __shared__ float s_gtf[];
  __shared__ float s_bound[4][4];
  const int tstride = 4 * K.tfn + 1;
  for (int i = threadIdx.x; i < kTfCopies * tstride; i += blockDim.x) s_gtf[i] = 0.0f;
  // the transfer function itself, after the copies (16-byte aligned), and
  // its largest |colour| component
  float4 *s_tf = reinterpret_cast<float4 *>(s_gtf + ((kTfCopies * tstride + 3) & ~3));
  float cm = 0.0f;
  for (int i = threadIdx.x; i < K.tfn; i += blockDim.x) {
    const float4 v = __ldg(&tf[i]);
    s_tf[i] = v;
    cm = fmaxf(cm, fmaxf(abs_or_inf(v.x), fmaxf(abs_or_inf(v.y), abs_or_inf(v.z))));
  }
  float *my_gtf = s_gtf + (threadIdx.x & (kTfCopies - 1)) * tstride;
  const int W = K.p.width, H = K.p.height;
  int px, py;
  const bool pixel = tile_pixel(blockIdx.x * blockDim.x + threadIdx.x, W, H, px, py);
  const int pix = pixel ? py * W + px : 0;
  const float4 g = pixel ? gimg[pix] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  float o[3], d[3], t0 = 0.0f, t1 = 0.0f;
  int ns = 0;
  if (pixel) {
    pixel_ray(K.p, px, py, o, d);
    if (slab(o, d, t0, t1)) {
      ns = (int)((t1 - t0) / K.p.step);
      if (ns > K.p.max_steps) ns = K.p.max_steps;
    }
  }
  const float sstep = K.p.sigma_scale * K.p.step;
  // the block's bounds: colour = sum of max_c |g.c|; opacity = sstep
  // (cm * sum of 2 ns G + sum of ns |g.w|)
  const float ax = abs_or_inf(g.x), ay = abs_or_inf(g.y), az = abs_or_inf(g.z);
  float b[4] = {fmaxf(ax, fmaxf(ay, az)), 2.0f * (float)ns * (ax + ay + az),
                (float)ns * abs_or_inf(g.w), cm};
#pragma unroll
  for (int sh = 16; sh > 0; sh >>= 1) {
#pragma unroll
    for (int k = 0; k < 3; k++) b[k] += __shfl_xor_sync(0xffffffffu, b[k], sh);
    b[3] = fmaxf(b[3], __shfl_xor_sync(0xffffffffu, b[3], sh));
  }
  if ((threadIdx.x & 31) == 0)
    for (int k = 0; k < 4; k++) s_bound[threadIdx.x >> 5][k] = b[k];
  __syncthreads();
  float bc = 0.0f, b1 = 0.0f, b2 = 0.0f, bm = 0.0f;
  for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
    bc += s_bound[w][0];
    b1 += s_bound[w][1];
    b2 += s_bound[w][2];
    bm = fmaxf(bm, s_bound[w][3]);
  }
  const float bo = fabsf(sstep) * (b1 * bm + b2);
  // 0: float adds (a block whose bound is not finite, or zero)
  const float cscale = (bc > 0.0f && bc <= FLT_MAX) ? colour_scale(bc) : 0.0f;
  const float oscale = (bo > 0.0f && bo <= FLT_MAX) ? colour_scale(bo) : 0.0f;
  if (ns > 0) {
    const float Tfin = trans[pix];
    const float gwT = g.w * Tfin;
    float Tn = Tfin;
    float gCb = 0.0f;  // g . (colour composited behind the sample)
    const float top = (float)(K.tfn - 1);
    // Run-length accumulators: consecutive samples often share the
    // transfer-function bin (always in empty space) and the voxel cell
    // (the step is half a voxel); contributions are summed in registers
    // and flushed when the bin / cell changes.  A table entry's colour
    // gradient is g times a scalar weight sum, so a run keeps per entry
    // (colour weight, opacity gradient).
    int run_i0 = -1;
    float2 ta0 = make_float2(0.f, 0.f), ta1 = make_float2(0.f, 0.f);
    int run_cell = -1, run_edge = 0;
    float da[8];
#pragma unroll
    for (int cc = 0; cc < 8; cc++) da[cc] = 0.0f;
    for (int s = ns - 1; s >= 0; s--) {
      const float t = t0 + ((float)s + 0.5f) * K.p.step;
      const float p[3] = {o[0] + t * d[0], o[1] + t * d[1], o[2] + t * d[2]};
      if (!inside(p)) continue;
      Cell cl;
      const float rho = fetch(dens, K.dim, tex_coord(K, 0, 0.5f * p[0] + 0.5f),
                              tex_coord(K, 1, 0.5f * p[1] + 0.5f),
                              tex_coord(K, 2, 0.5f * p[2] + 0.5f), &cl);
      float4 c, ta, tb;
      int i0, i1;
      float f;
      bool inr;
      tf_lookup_ab<true>(s_tf, K.tfn, rho, c, i0, i1, f, inr, ta, tb);
      const float e = __expf(-(K.p.sigma_scale * c.w) * K.p.step);
      float al = 1.0f - e;
      const bool clamped = al > K.p.alpha_max;
      if (clamped) al = K.p.alpha_max;
      const float iom = __fdividef(1.0f, 1.0f - al);
      const float Tk = Tn * iom;  // transmittance in front of sample s
      const float w = Tk * al;    // the sample's weight in the image
      const float gcol = g.x * c.x + g.y * c.y + g.z * c.z;
      // d loss / d alpha: Tk g.c - (g.Cb - g.w Tfin) / (1 - al)
      const float ga = Tk * gcol - iom * (gCb - gwT);
      const float gc3 = clamped ? 0.0f : ga * sstep * e;
      // transfer-function gradient: i1 = i0 + 1 except at the top entry
      if (i0 != run_i0) {
        // The run's two table entries are run_i0 (ta0) and run_i0 + 1 (ta1).
        // A step of one bin keeps the shared entry in registers and
        // flushes only the entry that leaves.
        if (run_i0 >= 0) {
          if (i0 == run_i0 + 1) {
            flush_entry(my_gtf, run_i0, ta0, g, cscale, oscale);
            ta0 = ta1;
            ta1 = make_float2(0.0f, 0.0f);
          } else if (i0 == run_i0 - 1) {
            flush_entry(my_gtf, min(run_i0 + 1, K.tfn - 1), ta1, g, cscale, oscale);
            ta1 = ta0;
            ta0 = make_float2(0.0f, 0.0f);
          } else {
            flush_entry(my_gtf, run_i0, ta0, g, cscale, oscale);
            flush_entry(my_gtf, min(run_i0 + 1, K.tfn - 1), ta1, g, cscale, oscale);
          }
        }
        run_i0 = i0;
      }
      const float wf0 = 1.0f - f;
      ta0.x += wf0 * w;
      ta0.y += wf0 * gc3;
      ta1.x += f * w;
      ta1.y += f * gc3;
      const float drho = inr ? (w * (g.x * (tb.x - ta.x) + g.y * (tb.y - ta.y) +
                                     g.z * (tb.z - ta.z)) +
                                gc3 * (tb.w - ta.w)) * top
                             : 0.0f;
      if (drho != 0.0f) {
        const int key = (cl.vz * K.dim[1] + cl.vy) * K.dim[0] + cl.vx;
        if (key != run_cell) {
          if (run_cell >= 0) flush_dens(gdens, K.dim, run_cell, run_edge, da);
          run_cell = key;
          run_edge = (cl.vx + 1 < K.dim[0] ? 0 : 1) | (cl.vy + 1 < K.dim[1] ? 0 : 2) |
                     (cl.vz + 1 < K.dim[2] ? 0 : 4);
        }
        // corner c = x + 2y + 4z gets drho * wx * wy * wz
        const float x0 = drho * (1.0f - cl.dx), x1 = drho * cl.dx;
        const float y0z0 = (1.0f - cl.dy) * (1.0f - cl.dz), y1z0 = cl.dy * (1.0f - cl.dz);
        const float y0z1 = (1.0f - cl.dy) * cl.dz, y1z1 = cl.dy * cl.dz;
        da[0] += x0 * y0z0;
        da[1] += x1 * y0z0;
        da[2] += x0 * y1z0;
        da[3] += x1 * y1z0;
        da[4] += x0 * y0z1;
        da[5] += x1 * y0z1;
        da[6] += x0 * y1z1;
        da[7] += x1 * y1z1;
      }
      gCb += w * gcol;
      Tn = Tk;
    }
    if (run_i0 >= 0) {
      flush_entry(my_gtf, run_i0, ta0, g, cscale, oscale);
      flush_entry(my_gtf, min(run_i0 + 1, K.tfn - 1), ta1, g, cscale, oscale);
    }
    if (run_cell >= 0) flush_dens(gdens, K.dim, run_cell, run_edge, da);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 4 * K.tfn; i += blockDim.x) {
    float v = 0.0f;
    const float sc = (i & 3) == 3 ? oscale : cscale;
    if (sc != 0.0f) {  // fixed point: the copies' integer sum, unscaled
      long long q = 0;
#pragma unroll
      for (int c = 0; c < kTfCopies; c++) q += __float_as_int(s_gtf[c * tstride + i]);
      v = (float)((double)q / (double)sc);
    } else {
#pragma unroll
      for (int c = 0; c < kTfCopies; c++) v += s_gtf[c * tstride + i];
    }
    if (v != 0.0f) atomicAdd(&gtf[i], v);
  }
}

srt_status make_const(const srt_volume_params *params, const int32_t dims[3],
                      int32_t tfn, VolConst &K) {
  if (!params || !dims || params->width <= 0 || params->height <= 0 || tfn < 2 ||
      tfn > kTfMax || dims[0] < 1 || dims[1] < 1 || dims[2] < 1 ||
      !(params->alpha_max < 1.0f) || params->step <= 0.0f || params->max_steps < 0) {
    set_error("invalid volume parameters");
    return SRT_ERR_INVALID;
  }
  if ((double)dims[0] * dims[1] * dims[2] >= 2147483647.0) {
    set_error("volume larger than 2^31 voxels");
    return SRT_ERR_INVALID;
  }
  K.p = *params;
  for (int k = 0; k < 3; k++) {
    K.dim[k] = dims[k];
    K.remap[k] = nullptr;
    K.nremap[k] = 0;
    K.clamp[k] = 1;  // without a sampling state: clamp-to-edge, no remap
  }
  K.tfn = tfn;
  return SRT_OK;
}

}  // namespace

// device view helper shared with the C API (declared here to keep the
// volume entry points self-contained)
static srt_status vol_view(srt_ctx *ctx, const void *p, size_t bytes, DevBuf &stage,
                           const void **out, cudaStream_t st) {
  if (!p) {
    *out = nullptr;
    return SRT_OK;
  }
  if (is_device_ptr(p)) {
    *out = p;
    return SRT_OK;
  }
  cudaError_t e = stage.ensure(bytes);
  if (e != cudaSuccess) return cuda_status(e, "volume staging");
  e = cudaMemcpyAsync(stage.p, p, bytes, cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return cuda_status(e, "volume copy");
  *out = stage.p;
  return SRT_OK;
}

// The texture's sampling state into K; host remap tables are staged in tmp.
static srt_status apply_sampling(srt_ctx *ctx, const srt_volume_sampling *sm, VolConst &K,
                                 DevBuf (&tmp)[3], cudaStream_t st) {
  if (!sm) return SRT_OK;
  for (int k = 0; k < 3; k++) {
    K.clamp[k] = sm->clamp[k] != 0;
    if (sm->remap[k] && sm->remap_n[k]) {
      if (sm->remap_n[k] > 0x7fffffffu) {
        set_error("remap table longer than 2^31 - 1 entries");
        return SRT_ERR_INVALID;
      }
      const void *dv;
      srt_status s = vol_view(ctx, sm->remap[k], (size_t)sm->remap_n[k] * 4, tmp[k], &dv, st);
      if (s != SRT_OK) return s;
      K.remap[k] = static_cast<const float *>(dv);
      K.nremap[k] = (int)sm->remap_n[k];
    }
  }
  return SRT_OK;
}

}  // namespace srt

using namespace srt;

extern "C" {

SRT_API srt_status srt_volume_camera(int32_t W, int32_t H, const float eye[3],
                                     const float lookat[3], const float up[3],
                                     float fov_deg, srt_volume_params *P) {
  if (!eye || !lookat || !up || !P || W <= 0 || H <= 0) return SRT_ERR_INVALID;
  // build_cameraframe, FP32 (same expression order as the oracle)
  float look[3], tmp[3], du[3], dv[3];
  for (int k = 0; k < 3; k++) look[k] = lookat[k] - eye[k];
  float ll = sqrtf(look[0] * look[0] + look[1] * look[1] + look[2] * look[2]);
  for (int k = 0; k < 3; k++) look[k] = look[k] / ll;
  tmp[0] = look[1] * up[2] - look[2] * up[1];
  tmp[1] = look[2] * up[0] - look[0] * up[2];
  tmp[2] = look[0] * up[1] - look[1] * up[0];
  float lu = sqrtf(tmp[0] * tmp[0] + tmp[1] * tmp[1] + tmp[2] * tmp[2]);
  for (int k = 0; k < 3; k++) du[k] = tmp[k] / lu;
  tmp[0] = look[1] * du[2] - look[2] * du[1];
  tmp[1] = look[2] * du[0] - look[0] * du[2];
  tmp[2] = look[0] * du[1] - look[1] * du[0];
  float lv = sqrtf(tmp[0] * tmp[0] + tmp[1] * tmp[1] + tmp[2] * tmp[2]);
  for (int k = 0; k < 3; k++) dv[k] = tmp[k] / lv;
  float flen = 0.5f * (float)H / (float)tan(0.5 * ((double)fov_deg * 3.14 / 180.0));
  P->width = W;
  P->height = H;
  for (int k = 0; k < 3; k++) {
    float lk = flen * look[k] + eye[k];
    P->corner[k] = lk - 0.5f * ((float)W * du[k] + (float)H * dv[k]);
    P->eye[k] = eye[k];
    P->du[k] = du[k];
    P->dv[k] = dv[k];
  }
  return SRT_OK;
}

SRT_API srt_status srt_volume_march_fwd_ex(srt_ctx *ctx, const srt_volume_params *params,
                                           const srt_volume_sampling *sampling,
                                           const float *density, const int32_t dims[3],
                                           const float *tf, int32_t tf_entries, float *image,
                                           float *transmittance) {
  if (!ctx || !density || !tf || !image) return SRT_ERR_INVALID;
  VolConst K;
  srt_status s = make_const(params, dims, tf_entries, K);
  if (s != SRT_OK) return s;
  cudaSetDevice(ctx->device);
  cudaStream_t st = ctx->stream;
  DevBuf remap_tmp[3];
  if ((s = apply_sampling(ctx, sampling, K, remap_tmp, st)) != SRT_OK) return s;
  const size_t nvox = (size_t)dims[0] * dims[1] * dims[2];
  const size_t npix = (size_t)params->width * params->height;
  const void *dd, *dt;
  if ((s = vol_view(ctx, density, nvox * 4, ctx->s_stage_in, &dd, st)) != SRT_OK) return s;
  if ((s = vol_view(ctx, tf, (size_t)tf_entries * 16, ctx->s_stage_aux, &dt, st)) != SRT_OK)
    return s;
  const bool img_dev = is_device_ptr(image);
  const bool tr_dev = transmittance ? is_device_ptr(transmittance) : true;
  float *di = image, *dtr = transmittance;
  DevBuf tmp_tr;
  cudaError_t e;
  if (!img_dev) {
    if ((e = ctx->s_stage_out.ensure(npix * 16)) != cudaSuccess) return cuda_status(e, "img");
    di = ctx->s_stage_out.as<float>();
  }
  if (!tr_dev) {
    if ((e = tmp_tr.ensure(npix * 4)) != cudaSuccess) return cuda_status(e, "trans");
    dtr = tmp_tr.as<float>();
  }
  const size_t nthreads = (size_t)((params->width + 7) / 8) * ((params->height + 3) / 4) * 32;
  vol_fwd_kernel<<<(unsigned)((nthreads + 127) / 128), 128, 0, st>>>(
      K, static_cast<const float *>(dd), static_cast<const float4 *>(dt),
      reinterpret_cast<float4 *>(di), dtr);
  ctx->launches++;
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_status(e, "volume fwd");
  if (!img_dev) cudaMemcpyAsync(image, di, npix * 16, cudaMemcpyDeviceToHost, st);
  if (!tr_dev) cudaMemcpyAsync(transmittance, dtr, npix * 4, cudaMemcpyDeviceToHost, st);
  const bool staged = remap_tmp[0].p || remap_tmp[1].p || remap_tmp[2].p;
  if (!img_dev || !tr_dev || staged)
    return cuda_status(cudaStreamSynchronize(st), "volume fwd");
  return SRT_OK;
}

SRT_API srt_status srt_volume_march_bwd_ex(srt_ctx *ctx, const srt_volume_params *params,
                                           const srt_volume_sampling *sampling,
                                           const float *density, const int32_t dims[3],
                                           const float *tf, int32_t tf_entries,
                                           const float *image, const float *transmittance,
                                           const float *grad_image, float *grad_density,
                                           float *grad_tf) {
  (void)image;  // the colour behind each sample is accumulated during the walk
  if (!ctx || !density || !tf || !transmittance || !grad_image || !grad_density || !grad_tf)
    return SRT_ERR_INVALID;
  VolConst K;
  srt_status s = make_const(params, dims, tf_entries, K);
  if (s != SRT_OK) return s;
  cudaSetDevice(ctx->device);
  cudaStream_t st = ctx->stream;
  DevBuf remap_tmp[3];
  if ((s = apply_sampling(ctx, sampling, K, remap_tmp, st)) != SRT_OK) return s;
  const size_t nvox = (size_t)dims[0] * dims[1] * dims[2];
  const size_t npix = (size_t)params->width * params->height;
  if (!is_device_ptr(grad_density) || !is_device_ptr(grad_tf)) {
    set_error("gradient outputs must be device memory");
    return SRT_ERR_INVALID;
  }
  DevBuf s_tr, s_g;
  const void *dd, *dt, *dtr, *dg;
  if ((s = vol_view(ctx, density, nvox * 4, ctx->s_stage_in, &dd, st)) != SRT_OK) return s;
  if ((s = vol_view(ctx, tf, (size_t)tf_entries * 16, ctx->s_stage_aux, &dt, st)) != SRT_OK)
    return s;
  if ((s = vol_view(ctx, transmittance, npix * 4, s_tr, &dtr, st)) != SRT_OK) return s;
  if ((s = vol_view(ctx, grad_image, npix * 16, s_g, &dg, st)) != SRT_OK) return s;
  const size_t shmem =
      (size_t)(((kTfCopies * (4 * tf_entries + 1) + 3) & ~3) + 4 * tf_entries) * sizeof(float);
  if (shmem > 48 * 1024) {
    cudaError_t ea = cudaFuncSetAttribute(vol_bwd_kernel,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)shmem);
    if (ea != cudaSuccess) return cuda_status(ea, "volume bwd shared memory");
  }
  const size_t nthreads = (size_t)((params->width + 7) / 8) * ((params->height + 3) / 4) * 32;
  vol_bwd_kernel<<<(unsigned)((nthreads + 127) / 128), 128, shmem, st>>>(
      K, static_cast<const float *>(dd), static_cast<const float4 *>(dt),
      static_cast<const float *>(dtr), static_cast<const float4 *>(dg), grad_density,
      grad_tf);
  ctx->launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_status(e, "volume bwd");
  if (s_tr.p || s_g.p || remap_tmp[0].p || remap_tmp[1].p || remap_tmp[2].p)
    return cuda_status(cudaStreamSynchronize(st), "volume bwd");
  return SRT_OK;
}


SRT_API srt_status srt_volume_march_fwd(srt_ctx *ctx, const srt_volume_params *params,
                                        const float *density, const int32_t dims[3],
                                        const float *tf, int32_t tf_entries, float *image,
                                        float *transmittance) {
  return srt_volume_march_fwd_ex(ctx, params, nullptr, density, dims, tf, tf_entries, image,
                                 transmittance);
}

SRT_API srt_status srt_volume_march_bwd(srt_ctx *ctx, const srt_volume_params *params,
                                        const float *density, const int32_t dims[3],
                                        const float *tf, int32_t tf_entries,
                                        const float *image, const float *transmittance,
                                        const float *grad_image, float *grad_density,
                                        float *grad_tf) {
  return srt_volume_march_bwd_ex(ctx, params, nullptr, density, dims, tf, tf_entries, image,
                                 transmittance, grad_image, grad_density, grad_tf);
}

}  // extern "C"
