// srt_texture.cu -- Texture::Fetch of 3D textures on the GPU
// (gles/gles_common.h:344-399), for a whole array of coordinates.
//
// Dense textures: the per-axis coordinate remap of non-uniform volumes
// (local::remap, gles/gles_common.h:264-269, set by lsglTexCoordRemap), then
// FilterTexture3D{Byte,Float,Double} (render/render_texture.cc:832-1175):
// repeat wrap by fasterfloorf unless clamp-to-edge, vox = u * (dim - 1),
// texel-corner trilinear interpolation with the reference's Lerp (dlerp in
// double for double textures), bytes read as v / 255.5f, a single component
// replicated to rgba.
//
// Sparse volumes: position = u * globalDim, the first block that
// BVHTree::Locate reaches (render/render_bvh_tree.cc:587-655; the tree is
// built on the host like the scene's top level), then
// SparseVolumeAccel::Sample (render/render_accel_volume.cc:61-139): the
// nearest texel of the block, the local offset scaled by size/extent of x on
// all three axes as the reference does, bytes as v / 255.0f, doubles through
// float, alpha 1 below four components, (0, 0, 0, 0) outside every block.
//
// Float-to-int conversions follow x86 (NaN and out-of-range values give
// INT_MIN), so every coordinate gives the reference's texel.  Compiled without
// FMA contraction: each expression rounds as in the reference.
#include <algorithm>
#include <cstring>
#include <vector>

#include "srt_internal.cuh"

using namespace srt;

struct srt_texture3d {
  srt_ctx *ctx = nullptr;
  bool sparse = false;
  int format = 1, comps = 1;
  int dim[3] = {0, 0, 0};   // dense: width, height, depth; sparse: globalDim
  int clamp[3] = {0, 0, 0};  // clamp-to-edge per axis (else repeat)
  DevBuf data;               // dense texels or the sparse data pool
  size_t data_bytes = 0;
  DevBuf remap[3];
  uint32_t nremap[3] = {0, 0, 0};
  DevBuf tree, blocks;       // sparse: BVHTree over the blocks, block table
  uint32_t nblocks = 0, ntree = 0;
};

namespace srt {
namespace {

__device__ __forceinline__ int clampi(int v, int lo, int hi) {
  return min(max(v, lo), hi);
}

__device__ __forceinline__ float lerp_ref(float t, float a, float b) {
  return (1.f - t) * a + t * b;
}
__device__ __forceinline__ double dlerp_ref(double t, double a, double b) {
  return (1.0 - t) * a + t * b;
}

struct DenseTex {
  const void *data;
  const float *remap[3];
  uint32_t nremap[3];
  int dim[3], clamp[3], comps, format;
};

template <int FMT>
__device__ __forceinline__ float texel_f(const void *d, size_t k) {
  if (FMT == 0) return (float)static_cast<const unsigned char *>(d)[k] / 255.5f;
  return __ldg(&static_cast<const float *>(d)[k]);
}

template <int FMT>
__global__ void __launch_bounds__(256)
dense_fetch_kernel(DenseTex t, const float *__restrict__ uvw, size_t n,
                   float4 *__restrict__ rgba) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    float c[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
      c[k] = __ldg(&uvw[3 * i + k]);
      if (t.nremap[k]) {  // local::remap
        const int nk = (int)t.nremap[k];
        int idx = f2i_x86(c[k] * (float)nk);
        idx = max(min(nk - 1, idx), 0);
        c[k] = __ldg(&t.remap[k][idx]);
      }
      if (!t.clamp[k]) c[k] = c[k] - (float)floor_ref(c[k]);
    }
    float vox[3];
    int v0[3], v1[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
      vox[k] = c[k] * ((float)t.dim[k] - 1.0f);
      v0[k] = clampi(f2i_x86(vox[k]), 0, t.dim[k] - 1);
      v1[k] = min(v0[k] + 1, t.dim[k] - 1);
    }
    const size_t sx = (size_t)t.comps, sy = sx * t.dim[0], sz = sy * t.dim[1];
    const size_t b000 = v0[2] * sz + v0[1] * sy + v0[0] * sx;
    const size_t ox = (size_t)(v1[0] - v0[0]) * sx, oy = (size_t)(v1[1] - v0[1]) * sy,
                 oz = (size_t)(v1[2] - v0[2]) * sz;
    float vals[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    for (int ch = 0; ch < t.comps && ch < 4; ch++) {
      const size_t b = b000 + ch;
      if (FMT == 2) {
        const double *d = static_cast<const double *>(t.data);
        const double dx = (double)(vox[0] - (float)v0[0]), dy = (double)(vox[1] - (float)v0[1]),
                     dz = (double)(vox[2] - (float)v0[2]);
        const double d00 = dlerp_ref(dx, __ldg(&d[b]), __ldg(&d[b + ox]));
        const double d10 = dlerp_ref(dx, __ldg(&d[b + oy]), __ldg(&d[b + oy + ox]));
        const double d01 = dlerp_ref(dx, __ldg(&d[b + oz]), __ldg(&d[b + oz + ox]));
        const double d11 = dlerp_ref(dx, __ldg(&d[b + oz + oy]), __ldg(&d[b + oz + oy + ox]));
        const double d0 = dlerp_ref(dy, d00, d10), d1 = dlerp_ref(dy, d01, d11);
        vals[ch] = (float)dlerp_ref(dz, d0, d1);
      } else {
        const float dx = vox[0] - (float)v0[0], dy = vox[1] - (float)v0[1],
                    dz = vox[2] - (float)v0[2];
        const float d00 = lerp_ref(dx, texel_f<FMT>(t.data, b), texel_f<FMT>(t.data, b + ox));
        const float d10 =
            lerp_ref(dx, texel_f<FMT>(t.data, b + oy), texel_f<FMT>(t.data, b + oy + ox));
        const float d01 =
            lerp_ref(dx, texel_f<FMT>(t.data, b + oz), texel_f<FMT>(t.data, b + oz + ox));
        const float d11 = lerp_ref(dx, texel_f<FMT>(t.data, b + oz + oy),
                                   texel_f<FMT>(t.data, b + oz + oy + ox));
        const float d0 = lerp_ref(dy, d00, d10), d1 = lerp_ref(dy, d01, d11);
        vals[ch] = lerp_ref(dz, d0, d1);
      }
    }
    rgba[i] = (t.comps == 1) ? make_float4(vals[0], vals[0], vals[0], vals[0])
                             : make_float4(vals[0], vals[1], vals[2], vals[3]);
  }
}

struct SparseTex {
  const TopNode *tree;
  const srt_volume_block *blocks;
  const unsigned char *pool;
  int gdim[3], comps, format;
  uint32_t max_iter;
};

__device__ __forceinline__ bool in_box(const TopNode &t, const double p[3]) {
  return p[0] >= t.bmin[0] && p[0] <= t.bmax[0] && p[1] >= t.bmin[1] && p[1] <= t.bmax[1] &&
         p[2] >= t.bmin[2] && p[2] <= t.bmax[2];
}

// BVHTree::Locate's first leaf: depth first, the left child first.
__device__ int locate(const TopNode *__restrict__ tree, const double p[3], uint32_t max_iter,
                      uint32_t *err) {
  int stk[64];
  int sp = 0, node = 0;
  for (uint32_t g = 0; g < max_iter; g++) {
    const TopNode &t = tree[node];
    if (t.leaf) {
      if (in_box(t, p)) return (int)t.id;
      if (sp < 1) return -1;
      node = stk[--sp];
      continue;
    }
    const bool h0 = t.child[0] > 0 && in_box(tree[t.child[0]], p);
    const bool h1 = t.child[1] > 0 && in_box(tree[t.child[1]], p);
    if (!h0 && !h1) {
      if (sp < 1) return -1;
      node = stk[--sp];
    } else if (h0 && h1) {
      if (sp >= 64) {
        atomicOr(err, kErrStack);
        return -1;
      }
      stk[sp++] = t.child[1];
      node = t.child[0];
    } else {
      node = h0 ? t.child[0] : t.child[1];
    }
  }
  atomicOr(err, kErrIter);
  return -1;
}

__global__ void __launch_bounds__(256)
sparse_fetch_kernel(SparseTex t, const float *__restrict__ uvw, size_t n,
                    float4 *__restrict__ rgba, uint32_t *__restrict__ err) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    double p[3];
#pragma unroll
    for (int k = 0; k < 3; k++) p[k] = (double)(__ldg(&uvw[3 * i + k]) * (float)t.gdim[k]);
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    const int id = locate(t.tree, p, t.max_iter, err);
    if (id >= 0) {
      const srt_volume_block &bl = t.blocks[id];
      const int nc = t.comps >= 4 ? 4 : t.comps;
      v[3] = 1.0;
      const double sx = (double)bl.size[0] / (double)bl.extent[0];
      const double x = (p[0] - (double)bl.offset[0]) * sx;
      const double y = (p[1] - (double)bl.offset[1]) * sx;  // x's ratio on every axis
      const double z = (p[2] - (double)bl.offset[2]) * sx;
      const int ix = max(min(bl.size[0] - 1, d2i_x86(x)), 0);
      const int iy = max(min(bl.size[1] - 1, d2i_x86(y)), 0);
      const int iz = max(min(bl.size[2] - 1, d2i_x86(z)), 0);
      const size_t idx =
          ((size_t)iz * bl.size[1] + (size_t)iy) * (size_t)bl.size[0] + (size_t)ix;
      const unsigned char *base = t.pool + bl.data_offset;
      for (int c = 0; c < nc; c++) {
        const size_t k = (size_t)nc * idx + c;  // the stride is the clamped count
        if (t.format == 0)
          v[c] = (double)((float)base[k] / 255.0f);
        else if (t.format == 1)
          v[c] = (double)reinterpret_cast<const float *>(base)[k];
        else
          v[c] = (double)(float)reinterpret_cast<const double *>(base)[k];
      }
    }
    rgba[i] = make_float4((float)v[0], (float)v[1], (float)v[2], (float)v[3]);
  }
}

size_t format_bytes(int f) { return f == 0 ? 1 : f == 1 ? 4 : 8; }

srt_status upload(srt_ctx *ctx, DevBuf &dst, const void *src, size_t bytes) {
  cudaError_t e = dst.ensure(bytes ? bytes : 1);
  if (e == cudaSuccess && bytes)
    e = cudaMemcpyAsync(dst.p, src, bytes,
                        is_device_ptr(src) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                        ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);  // src may be freed next
  return cuda_status(e, "texture upload");
}

}  // namespace
}  // namespace srt

extern "C" {

SRT_API srt_status srt_texture3d_create(srt_ctx *ctx, srt_texture3d **out) {
  if (!ctx || !out) return SRT_ERR_INVALID;
  srt_texture3d *t = new (std::nothrow) srt_texture3d();
  if (!t) return SRT_ERR_NO_MEMORY;
  t->ctx = ctx;
  *out = t;
  return SRT_OK;
}

SRT_API srt_status srt_texture3d_destroy(srt_texture3d *t) {
  if (!t) return SRT_OK;
  cudaSetDevice(t->ctx->device);
  cudaStreamSynchronize(t->ctx->stream);
  delete t;
  return SRT_OK;
}

SRT_API srt_status srt_texture3d_set_dense(srt_texture3d *t, int format, int width, int height,
                                           int depth, int components, const void *data) {
  if (!t || !data) return SRT_ERR_INVALID;
  if (format < 0 || format > 2 || components < 1 || components > 4 || width < 1 ||
      height < 1 || depth < 1) {
    set_error("srt_texture3d_set_dense: format 0..2, 1..4 components, positive size");
    return SRT_ERR_INVALID;
  }
  cudaSetDevice(t->ctx->device);
  const size_t bytes =
      (size_t)width * height * depth * components * format_bytes(format);
  srt_status s = upload(t->ctx, t->data, data, bytes);
  if (s != SRT_OK) return s;
  t->sparse = false;
  t->format = format;
  t->comps = components;
  t->dim[0] = width;
  t->dim[1] = height;
  t->dim[2] = depth;
  t->data_bytes = bytes;
  return SRT_OK;
}

SRT_API srt_status srt_texture3d_set_wrap(srt_texture3d *t, int clamp_s, int clamp_t,
                                          int clamp_r) {
  if (!t) return SRT_ERR_INVALID;
  t->clamp[0] = clamp_s != 0;
  t->clamp[1] = clamp_t != 0;
  t->clamp[2] = clamp_r != 0;
  return SRT_OK;
}

SRT_API srt_status srt_texture3d_set_remap(srt_texture3d *t, int axis, const float *table,
                                           size_t n) {
  if (!t || axis < 0 || axis > 2 || (n && !table) || n > 0x7fffffffu) {
    set_error("srt_texture3d_set_remap: axis 0..2 and a table of n < 2^31 entries");
    return SRT_ERR_INVALID;
  }
  cudaSetDevice(t->ctx->device);
  if (n) {
    srt_status s = upload(t->ctx, t->remap[axis], table, n * sizeof(float));
    if (s != SRT_OK) return s;
  }
  t->nremap[axis] = (uint32_t)n;
  return SRT_OK;
}

SRT_API srt_status srt_texture3d_set_sparse(srt_texture3d *t, int format, int components,
                                            const int global_dim[3],
                                            const srt_volume_block *blocks, size_t nblocks,
                                            const void *pool, size_t pool_bytes) {
  if (!t || !global_dim || !blocks || !nblocks || !pool) return SRT_ERR_INVALID;
  if (format < 0 || format > 2 || components < 1 || nblocks >= (1u << 30)) {
    set_error("srt_texture3d_set_sparse: format 0..2, at least one component and block");
    return SRT_ERR_INVALID;
  }
  const int nc = components >= 4 ? 4 : components;
  std::vector<double> lo(3 * nblocks), hi(3 * nblocks);
  for (size_t i = 0; i < nblocks; i++) {
    const srt_volume_block &b = blocks[i];
    uint64_t vox = (uint64_t)nc * format_bytes(format);
    for (int k = 0; k < 3; k++) {
      if (b.size[k] < 1 || b.extent[k] < 1) {
        set_error("srt_texture3d_set_sparse: block sizes and extents must be positive");
        return SRT_ERR_INVALID;
      }
      vox *= (uint64_t)b.size[k];
      lo[3 * i + k] = (double)b.offset[k];
      hi[3 * i + k] = (double)((int64_t)b.offset[k] + b.extent[k]);
    }
    if (b.data_offset > pool_bytes || vox > pool_bytes - b.data_offset ||
        (b.data_offset % format_bytes(format)) != 0) {
      set_error("srt_texture3d_set_sparse: a block's voxels lie outside the pool or misaligned");
      return SRT_ERR_INVALID;
    }
  }
  std::vector<TopNode> tree;
  build_top_tree(lo.data(), hi.data(), nblocks, tree);
  cudaSetDevice(t->ctx->device);
  srt_status s = upload(t->ctx, t->data, pool, pool_bytes);
  if (s == SRT_OK) s = upload(t->ctx, t->tree, tree.data(), tree.size() * sizeof(TopNode));
  if (s == SRT_OK) s = upload(t->ctx, t->blocks, blocks, nblocks * sizeof(srt_volume_block));
  if (s != SRT_OK) return s;
  t->sparse = true;
  t->format = format;
  t->comps = components;
  for (int k = 0; k < 3; k++) t->dim[k] = global_dim[k];
  t->data_bytes = pool_bytes;
  t->nblocks = (uint32_t)nblocks;
  t->ntree = (uint32_t)tree.size();
  return SRT_OK;
}

SRT_API srt_status srt_texture3d_fetch(srt_texture3d *t, const float *uvw, size_t n,
                                       float *rgba) {
  if (!t || (n && (!uvw || !rgba))) return SRT_ERR_INVALID;
  if (!t->data.p) {
    set_error("srt_texture3d_fetch: no texture data set");
    return SRT_ERR_INVALID;
  }
  if (n == 0) return SRT_OK;
  srt_ctx *ctx = t->ctx;
  cudaSetDevice(ctx->device);
  if (!is_device_ptr(uvw) || !is_device_ptr(rgba) ||
      (reinterpret_cast<uintptr_t>(rgba) & 15u)) {
    set_error("srt_texture3d_fetch: device arrays, rgba 16-byte aligned");
    return SRT_ERR_INVALID;
  }
  const unsigned grid = (unsigned)std::min<size_t>((n + 255) / 256, (size_t)ctx->num_sms * 16);
  float4 *out = reinterpret_cast<float4 *>(rgba);
  if (t->sparse) {
    SparseTex st;
    st.tree = t->tree.as<TopNode>();
    st.blocks = t->blocks.as<srt_volume_block>();
    st.pool = t->data.as<unsigned char>();
    for (int k = 0; k < 3; k++) st.gdim[k] = t->dim[k];
    st.comps = t->comps;
    st.format = t->format;
    st.max_iter = 4 * t->ntree + 8;
    sparse_fetch_kernel<<<grid, 256, 0, ctx->stream>>>(st, uvw, n, out, ctx->d_err);
  } else {
    DenseTex dt;
    dt.data = t->data.p;
    for (int k = 0; k < 3; k++) {
      dt.remap[k] = t->remap[k].as<float>();
      dt.nremap[k] = t->nremap[k];
      dt.dim[k] = t->dim[k];
      dt.clamp[k] = t->clamp[k];
    }
    dt.comps = t->comps;
    dt.format = t->format;
    if (t->format == 0)
      dense_fetch_kernel<0><<<grid, 256, 0, ctx->stream>>>(dt, uvw, n, out);
    else if (t->format == 1)
      dense_fetch_kernel<1><<<grid, 256, 0, ctx->stream>>>(dt, uvw, n, out);
    else
      dense_fetch_kernel<2><<<grid, 256, 0, ctx->stream>>>(dt, uvw, n, out);
  }
  ctx->launches++;
  return cuda_status(cudaGetLastError(), "texture fetch");
}

}  // extern "C"
