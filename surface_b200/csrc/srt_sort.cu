// srt_sort.cu -- stable sort of (Morton code, index) pairs.
//
// The order is the reference's: ascending 30-bit code, ties in input order
// (RadixSort30OMP, render/render_prefix_tree_util.h:296-402, is a stable LSD
// sort whose keys start as index = i).  Here: three 10-bit LSD passes, one
// decoupled look-back kernel per pass:
//
//   os_hist_kernel   one read of the codes: the global count of every digit
//                    of the three passes (shared-memory histograms, warp-
//                    aggregated; zeroed by a memset before)
//   os_pass_kernel   per pass, tiles of 256 x ROUNDS keys in tile order
//                    (tile ids from a ticket counter, so a tile only waits on
//                    tiles that are already running): rank every key within
//                    its tile (warps own consecutive chunks, one ballot per
//                    digit bit ranks lanes in order), publish the tile's digit
//                    counts, add the counts of earlier tiles (look-back over
//                    their published aggregates / inclusive prefixes), stage
//                    the tile in shared memory in (digit, input) order and
//                    write it out in runs of equal digits.
//
// Look-back words are 64 bits: the pass's epoch (a per-context counter, so
// the status array is never cleared between passes) and a 32-bit value
// (flag in bits 30-31: aggregate or inclusive prefix; count in bits 0-29).
// Every wait is bounded: a tile that waits longer than kSpinLimit polls sets
// the context's error flag and gives up (SRT_ERR_LIMIT), it never hangs.
#include <algorithm>

#include "srt_internal.cuh"

namespace srt {
namespace {

constexpr int kOsBits = 10;
constexpr int kOsBins = 1 << kOsBits;
constexpr int kOsWarps = 8;
constexpr int kOsThreads = kOsWarps * 32;
constexpr int kOsPerThread = kOsBins / kOsThreads;  // 4 bins per thread
constexpr uint32_t kFlagAgg = 1u << 30;
constexpr uint32_t kFlagInc = 2u << 30;
constexpr uint32_t kCountMask30 = (1u << 30) - 1u;
constexpr uint32_t kSpinLimit = 1u << 22;
constexpr uint32_t kErrSort = kErrSortWait;

// Exclusive scan of kOsBins values held 4 per thread (bins 4t..4t+3), in
// place; returns the total.  Uses `tmp` (kOsWarps words) of shared memory.
__device__ __forceinline__ uint32_t block_scan4(uint32_t x[kOsPerThread], uint32_t *tmp) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  uint32_t s = 0;
#pragma unroll
  for (int q = 0; q < kOsPerThread; q++) {
    const uint32_t t = x[q];
    x[q] = s;
    s += t;
  }
  uint32_t inc = s;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += y;
  }
  if (lane == 31) tmp[w] = inc;
  __syncthreads();
  uint32_t wbase = 0, total = 0;
#pragma unroll
  for (int k = 0; k < kOsWarps; k++) {
    const uint32_t v = tmp[k];
    if (k < w) wbase += v;
    total += v;
  }
  const uint32_t base = wbase + inc - s;
#pragma unroll
  for (int q = 0; q < kOsPerThread; q++) x[q] += base;
  __syncthreads();
  return total;
}

__global__ void __launch_bounds__(kOsThreads)
os_hist_kernel(const uint32_t *__restrict__ keys, size_t n, uint32_t *__restrict__ ghist,
               unsigned long long *__restrict__ tickets) {
  __shared__ uint32_t h[3][kOsBins];
  // the passes that follow on the stream take their tile ids from these
  if (blockIdx.x == 0 && threadIdx.x < 3) tickets[threadIdx.x] = 0ull;
  for (int i = threadIdx.x; i < 3 * kOsBins; i += kOsThreads) (&h[0][0])[i] = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const size_t stride = (size_t)gridDim.x * kOsThreads;
  for (size_t base = (size_t)blockIdx.x * kOsThreads; base < n; base += stride) {
    const size_t i = base + threadIdx.x;
    const bool ok = i < n;
    const uint32_t k = ok ? __ldg(&keys[i]) : 0u;
    const unsigned act = __ballot_sync(0xffffffffu, ok);
#pragma unroll
    for (int p = 0; p < 3; p++) {
      const uint32_t d = (k >> (kOsBits * p)) & (kOsBins - 1);
      // warp-aggregated: one shared atomic per distinct digit of the warp
      const unsigned peers = __match_any_sync(0xffffffffu, d) & act;
      if (ok && lane == __ffs(peers) - 1) atomicAdd(&h[p][d], (uint32_t)__popc(peers));
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 3 * kOsBins; i += kOsThreads) {
    const uint32_t c = (&h[0][0])[i];
    if (c) atomicAdd(&ghist[i], c);
  }
}

__device__ __forceinline__ unsigned long long ld_status(const unsigned long long *p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_status(unsigned long long *p, unsigned long long v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Shared memory of one pass block (dynamic): per-warp digit counts, then the
// staged tile.
template <int ROUNDS>
struct PassSmem {
  static constexpr int kTile = kOsThreads * ROUNDS;
  uint32_t wc[kOsWarps][kOsBins];  // counts, then exclusive offsets per warp
  uint32_t tloc[kOsBins];          // tile-local start of each digit
  uint32_t gdst[kOsBins];          // global position of tile slot 0 per digit
  uint32_t tmp[kOsWarps];
  uint32_t tile;
  uint32_t key[kTile];
  uint32_t val[kTile];
};

template <int ROUNDS>
__global__ void __launch_bounds__(kOsThreads)
os_pass_kernel(const uint32_t *__restrict__ kin, const uint32_t *__restrict__ vin,
               uint32_t *__restrict__ kout, uint32_t *__restrict__ vout, uint32_t n, int shift,
               const uint32_t *__restrict__ ghist, unsigned long long *__restrict__ status,
               unsigned long long *__restrict__ ticket, uint32_t epoch,
               uint32_t *__restrict__ err) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  PassSmem<ROUNDS> &S = *reinterpret_cast<PassSmem<ROUNDS> *>(smem_raw);
  constexpr int kTile = PassSmem<ROUNDS>::kTile;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (threadIdx.x == 0) S.tile = (uint32_t)atomicAdd(ticket, 1ull);
  for (int i = threadIdx.x; i < kOsWarps * kOsBins; i += kOsThreads) (&S.wc[0][0])[i] = 0;
  __syncthreads();
  const uint32_t tile = S.tile;
  if (tile >= gridDim.x) {  // a counter left over from a failed launch
    if (threadIdx.x == 0) atomicOr(err, kErrSort);
    return;
  }
  const uint32_t base = tile * (uint32_t)kTile + (uint32_t)w * (32u * ROUNDS);

  // load, digits, in-warp ranks (peers: lanes of the round with this digit)
  uint32_t k[ROUNDS], v[ROUNDS], dg[ROUNDS], rk[ROUNDS];
  bool ok[ROUNDS];
#pragma unroll
  for (int r = 0; r < ROUNDS; r++) {
    const uint32_t idx = base + (uint32_t)r * 32u + (uint32_t)lane;
    ok[r] = idx < n;
    k[r] = ok[r] ? kin[idx] : 0u;
    v[r] = ok[r] ? (vin ? vin[idx] : idx) : 0u;
  }
  const unsigned lt = (1u << lane) - 1u;
#pragma unroll
  for (int r = 0; r < ROUNDS; r++) {
    unsigned pm = __ballot_sync(0xffffffffu, ok[r]);
    const uint32_t d = (k[r] >> shift) & (kOsBins - 1);
#pragma unroll
    for (int b = 0; b < kOsBits; b++) {
      const bool bit = (d >> b) & 1u;
      const unsigned m = __ballot_sync(0xffffffffu, bit);
      pm &= bit ? m : ~m;
    }
    dg[r] = d;
    // rank among this warp's earlier keys of the same digit
    uint32_t before = 0;
    if (ok[r]) before = S.wc[w][d];
    __syncwarp();
    rk[r] = before + (uint32_t)__popc(pm & lt);
    if (ok[r] && lane == __ffs(pm) - 1) S.wc[w][d] = before + (uint32_t)__popc(pm);
    __syncwarp();
  }
  __syncthreads();

  // tile counts; per-warp exclusive offsets within each digit
  uint32_t c[kOsPerThread];
#pragma unroll
  for (int q = 0; q < kOsPerThread; q++) {
    const int d = kOsPerThread * threadIdx.x + q;
    uint32_t run = 0;
#pragma unroll
    for (int ww = 0; ww < kOsWarps; ww++) {
      const uint32_t t = S.wc[ww][d];
      S.wc[ww][d] = run;
      run += t;
    }
    c[q] = run;
  }
  // publish this tile's counts before anything else, so later tiles can go on
  unsigned long long *st = status + (size_t)tile * kOsBins;
  const unsigned long long ep = (unsigned long long)epoch << 32;
#pragma unroll
  for (int q = 0; q < kOsPerThread; q++) {
    const int d = kOsPerThread * threadIdx.x + q;
    st_status(&st[d], ep | (tile == 0 ? kFlagInc : kFlagAgg) | c[q]);
  }
  // global digit starts (exclusive scan of this pass's histogram)
  uint32_t g[kOsPerThread];
#pragma unroll
  for (int q = 0; q < kOsPerThread; q++) g[q] = __ldg(&ghist[kOsPerThread * threadIdx.x + q]);
  block_scan4(g, S.tmp);
  // tile-local digit starts
  uint32_t tl[kOsPerThread];
#pragma unroll
  for (int q = 0; q < kOsPerThread; q++) tl[q] = c[q];
  block_scan4(tl, S.tmp);
  // look-back: keys of each digit in earlier tiles.  The thread's four bins
  // walk back together, kWin predecessor words per bin per round, all loads
  // of a round in flight at once; a window is consumed up to its nearest
  // inclusive prefix, or retried while a word in it is not yet published.
  constexpr int kWin = 4;
  bool failed = false;
  uint32_t prefix[kOsPerThread];
  int jnext[kOsPerThread];  // next predecessor to read, -1: done
#pragma unroll
  for (int q = 0; q < kOsPerThread; q++) {
    prefix[q] = 0;
    jnext[q] = (int)tile - 1;
  }
  uint32_t spins = 0;
  while (true) {
    bool pending = false;
#pragma unroll
    for (int q = 0; q < kOsPerThread; q++) pending |= jnext[q] >= 0;
    if (!pending) break;
    unsigned long long wv[kOsPerThread][kWin];
#pragma unroll
    for (int q = 0; q < kOsPerThread; q++) {
      const int d = kOsPerThread * threadIdx.x + q;
#pragma unroll
      for (int w = 0; w < kWin; w++) {
        const int j = jnext[q] - w;
        wv[q][w] = j >= 0 ? ld_status(&status[(size_t)j * kOsBins + d])
                          : (((unsigned long long)epoch << 32) | kFlagInc);  // tile -1: 0
      }
    }
    bool stalled = false;
#pragma unroll
    for (int q = 0; q < kOsPerThread; q++) {
      if (jnext[q] < 0) continue;
      uint32_t add = 0;
      int consumed = 0;
      bool fin = false, wait = false;
#pragma unroll
      for (int w = 0; w < kWin; w++) {
        if (fin || wait) continue;
        if ((uint32_t)(wv[q][w] >> 32) != epoch) {
          wait = true;
          continue;
        }
        const uint32_t x = (uint32_t)wv[q][w];
        add += x & kCountMask30;
        consumed = w + 1;
        if (x & kFlagInc) fin = true;
      }
      prefix[q] += add;
      jnext[q] = fin ? -1 : jnext[q] - consumed;
      stalled |= wait && consumed == 0;
    }
    if (stalled) {
      if (++spins > kSpinLimit) {
        failed = true;
        break;
      }
      __nanosleep(64);
    }
  }
#pragma unroll
  for (int q = 0; q < kOsPerThread; q++) {
    const int d = kOsPerThread * threadIdx.x + q;
    if (tile > 0) st_status(&st[d], ep | kFlagInc | ((prefix[q] + c[q]) & kCountMask30));
    S.tloc[d] = tl[q];
    S.gdst[d] = g[q] + prefix[q] - tl[q];
  }
  if (failed) atomicOr(err, kErrSort);
  __syncthreads();

  // stage the tile in (digit, input) order
#pragma unroll
  for (int r = 0; r < ROUNDS; r++) {
    if (!ok[r]) continue;
    const uint32_t d = dg[r];
    const uint32_t pos = S.tloc[d] + S.wc[w][d] + rk[r];
    S.key[pos] = k[r];
    S.val[pos] = v[r];
  }
  __syncthreads();
  // write out: consecutive slots of one digit go to consecutive addresses
  const uint32_t cnt = min((uint32_t)kTile, n - tile * (uint32_t)kTile);
  for (uint32_t j = threadIdx.x; j < cnt; j += kOsThreads) {
    const uint32_t kk = S.key[j];
    const uint32_t d = (kk >> shift) & (kOsBins - 1);
    const uint32_t gp = S.gdst[d] + j;
    if (gp < n) {  // holds unless a look-back gave up (error flag set)
      kout[gp] = kk;
      vout[gp] = S.val[j];
    }
  }
}

template <int ROUNDS>
srt_status os_sort(srt_ctx *ctx, uint32_t *keys, uint32_t *vals, size_t n, bool identity_vals,
                   bool hist_ready) {
  cudaStream_t st = ctx->stream;
  constexpr int kTile = PassSmem<ROUNDS>::kTile;
  const uint32_t ntiles = (uint32_t)((n + kTile - 1) / kTile);
  const size_t smem = sizeof(PassSmem<ROUNDS>);
  static bool attr_set[64] = {};
  if (ctx->device >= 0 && ctx->device < 64 && !attr_set[ctx->device]) {
    cudaError_t e = cudaFuncSetAttribute(os_pass_kernel<ROUNDS>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return cuda_status(e, "sort pass attributes");
    attr_set[ctx->device] = true;
  }
  uint32_t *ghist = nullptr;
  unsigned long long *tickets = nullptr;
  srt_status s = sort_codes30_scratch(ctx, n, &ghist, &tickets);
  if (s != SRT_OK) return s;
  unsigned long long *status = tickets + 32;  // after the 256-byte header
  if (!hist_ready) {
    cudaError_t e = cudaMemsetAsync(ghist, 0, 3 * kOsBins * 4, st);
    if (e != cudaSuccess) return cuda_status(e, "sort");
    // each block flushes up to 3 x 1024 counters: about 4096 keys per block
    const int hgrid = (int)std::min<size_t>((n + 4095) / 4096, (size_t)ctx->num_sms * 2);
    os_hist_kernel<<<hgrid, kOsThreads, 0, st>>>(keys, n, ghist, tickets);
    ctx->launches++;
  }
  // keys -> 2 -> 3 -> keys: three passes end where they started
  uint32_t *ksrc[3] = {keys, ctx->s_keys2.as<uint32_t>(), ctx->s_keys3.as<uint32_t>()};
  uint32_t *vsrc[3] = {vals, ctx->s_vals2.as<uint32_t>(), ctx->s_vals3.as<uint32_t>()};
  for (int p = 0; p < 3; p++) {
    const uint32_t epoch = ++ctx->os_epoch == 0 ? ++ctx->os_epoch : ctx->os_epoch;
    const uint32_t *vin = (p == 0 && identity_vals) ? nullptr : vsrc[p];
    os_pass_kernel<ROUNDS><<<ntiles, kOsThreads, smem, st>>>(
        ksrc[p], vin, ksrc[(p + 1) % 3], vsrc[(p + 1) % 3], (uint32_t)n, kOsBits * p,
        ghist + kOsBins * p, status, tickets + p, epoch, ctx->d_err);
    ctx->launches++;
  }
  return cuda_status(cudaGetLastError(), "sort passes");
}

}  // namespace

// Scratch of sort_codes30 for n keys: ping-pong buffers, the digit
// histograms (3 x 1024 words) and the look-back words behind a 256-byte
// header whose first three 64-bit words are the passes' tile counters.
srt_status sort_codes30_scratch(srt_ctx *ctx, size_t n, uint32_t **hist,
                                unsigned long long **tickets) {
  cudaError_t e;
  if ((e = ctx->s_keys2.ensure(n * 4)) != cudaSuccess) return cuda_status(e, "sort");
  if ((e = ctx->s_vals2.ensure(n * 4)) != cudaSuccess) return cuda_status(e, "sort");
  if ((e = ctx->s_keys3.ensure(n * 4)) != cudaSuccess) return cuda_status(e, "sort");
  if ((e = ctx->s_vals3.ensure(n * 4)) != cudaSuccess) return cuda_status(e, "sort");
  if ((e = ctx->s_hist.ensure(3 * kOsBins * 4)) != cudaSuccess) return cuda_status(e, "sort");
  const size_t ntiles = (n + kOsThreads * 4 - 1) / (kOsThreads * 4);  // the smallest tiles
  const size_t sbytes = 256 + ntiles * kOsBins * 8;
  if (sbytes > ctx->s_status.cap || !ctx->s_status.p) {
    // fresh words: epoch 0 never matches a pass
    if ((e = ctx->s_status.ensure(sbytes)) != cudaSuccess) return cuda_status(e, "sort");
    if ((e = cudaMemsetAsync(ctx->s_status.p, 0, ctx->s_status.cap, ctx->stream)) !=
        cudaSuccess)
      return cuda_status(e, "sort");
  }
  *hist = ctx->s_hist.as<uint32_t>();
  *tickets = ctx->s_status.as<unsigned long long>();
  return SRT_OK;
}

// Stable sort of (30-bit code, value) pairs by code, in place.  identity_vals:
// the values are 0..n-1 on entry (not read).  hist_ready: the digit
// histograms of the three passes are already in the scratch and the tile
// counters zeroed (the Morton kernel of a build does both).  n < 2^30.
srt_status sort_codes30(srt_ctx *ctx, uint32_t *keys, uint32_t *vals, size_t n,
                        bool identity_vals, bool hist_ready) {
  if (n == 0) return SRT_OK;
  if (n >= (1u << 30)) {
    set_error("sort: at most 2^30 - 1 keys");
    return SRT_ERR_INVALID;
  }
  // small arrays: short tiles keep every SM busy; large: long tiles amortise
  // the per-tile look-back
  if (n <= (1u << 21)) return os_sort<4>(ctx, keys, vals, n, identity_vals, hist_ready);
  return os_sort<16>(ctx, keys, vals, n, identity_vals, hist_ready);
}

}  // namespace srt
