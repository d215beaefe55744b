// prims.cu -- radix sort, merge-path merge and sorted difference of 64-bit
// keys (declarations and the scan/select templates are in prims.cuh).
#include <algorithm>

#include "prims.cuh"

namespace trc {

// ---------------------------------------------------------------------------
// Radix sort, one sweep per 8-bit digit.  (1) One pass over the keys counts
// every digit position at once (per-CTA shared histograms, then global
// atomics), (2) one CTA turns the counts into each digit value's global
// start, (3) per digit, one scatter kernel: each tile ranks its keys (warp
// __match_any_sync ranking, warps combined by a per-digit prefix in shared
// memory), publishes its per-digit counts, and finds the counts of all
// earlier tiles by decoupled look-back over a status word per (tile, digit)
// (flag in the top bits, running count below; tiles take ids in launch
// order from an atomic counter, so a tile only waits on tiles that started
// before it).  The wait is bounded: after SortWait::spin_limit polls the tile
// sets ERR_TIMEOUT in the error word and proceeds (its output is then garbage
// and the caller fails the call; every write stays inside the output, whose
// digit ranges come from the full histogram).

constexpr uint64_t OS_AGG = 1ull << 62;   // tile count published
constexpr uint64_t OS_INC = 2ull << 62;   // count of this tile and all before it
constexpr uint64_t OS_VAL = (1ull << 62) - 1;
constexpr int OS_MAXD = 8;

struct OsShifts {
  int s[OS_MAXD];
  int n;
};

__global__ void __launch_bounds__(RS_T) k_os_hist(const uint64_t *in, uint64_t n, OsShifts sh,
                                                  unsigned long long *ghist) {
  __shared__ uint32_t h[OS_MAXD][256];
  for (int i = threadIdx.x; i < OS_MAXD * 256; i += RS_T) (&h[0][0])[i] = 0;
  __syncthreads();
  const uint64_t stride = (uint64_t)gridDim.x * RS_T;
  for (uint64_t i = (uint64_t)blockIdx.x * RS_T + threadIdx.x; i < n; i += stride) {
    uint64_t k = in[i];
    for (int d = 0; d < sh.n; d++) atomicAdd(&h[d][(uint32_t)(k >> sh.s[d]) & 255u], 1u);
  }
  __syncthreads();
  for (int d = 0; d < sh.n; d++)
    if (h[d][threadIdx.x]) atomicAdd(&ghist[d * 256 + threadIdx.x], (unsigned long long)h[d][threadIdx.x]);
}

// one CTA of 256 threads: exclusive prefix of every digit position's counts
__global__ void k_os_prefix(const unsigned long long *ghist, int nd, uint64_t *goff) {
  __shared__ uint64_t ws[RS_T / 32 + 1];
  for (int d = 0; d < nd; d++) {
    uint64_t tot;
    uint64_t ex = block_excl_scan<uint64_t, RS_T>(ghist[d * 256 + threadIdx.x], ws, tot);
    goff[d * 256 + threadIdx.x] = ex;
  }
}

__global__ void __launch_bounds__(RS_T) k_os_scatter(const uint64_t *in, uint64_t *out, uint64_t n,
                                                     int shift, const uint64_t *goff,
                                                     uint64_t *status, uint32_t *tile_ctr,
                                                     uint32_t *err, uint32_t spin_limit,
                                                     uint32_t tile_base) {
  __shared__ uint32_t wh[RS_W][256];
  __shared__ uint64_t tbase[256];    // global start of digit d for this tile, minus its tile start
  __shared__ uint32_t dstart[256];   // start of digit d inside the tile (tile-sorted order)
  __shared__ uint64_t stage[RS_TILE];
  __shared__ uint32_t tile_s;
  __shared__ uint32_t ws[RS_W + 1];
  for (int i = threadIdx.x; i < RS_W * 256; i += RS_T) (&wh[0][0])[i] = 0;
  if (threadIdx.x == 0) tile_s = atomicAdd(tile_ctr, 1u) + tile_base;
  __syncthreads();
  const uint32_t tile = tile_s;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // warp w owns keys [base, base + RS_I*32) of the tile, slot-major
  const uint64_t tile0 = (uint64_t)tile * RS_TILE;
  const uint64_t base = tile0 + (uint64_t)warp * (RS_I * 32);
  uint64_t k[RS_I];
  uint32_t rank[RS_I];
  const uint32_t lt = lanemask_lt();
#pragma unroll
  for (int s = 0; s < RS_I; s++) {
    uint64_t idx = base + (uint64_t)s * 32 + lane;
    bool valid = idx < n;
    k[s] = valid ? in[idx] : 0;
    uint32_t active = __ballot_sync(0xFFFFFFFFu, valid);
    if (valid) {
      uint32_t d = (uint32_t)(k[s] >> shift) & 255u;
      uint32_t peers = __match_any_sync(active, d);
      uint32_t cnt = wh[warp][d];
      rank[s] = cnt + __popc(peers & lt);
      __syncwarp(active);
      if (lane == __ffs(peers) - 1) wh[warp][d] = cnt + __popc(peers);
      __syncwarp(active);
    }
  }
  __syncthreads();
  {
    // thread d: offsets of digit d inside the tile (per warp) and the tile's count
    const uint32_t d = threadIdx.x;
    uint32_t run = 0;
#pragma unroll
    for (int w = 0; w < RS_W; w++) {
      uint32_t c = wh[w][d];
      wh[w][d] = run;
      run += c;
    }
    // start of digit d in the tile-sorted order
    uint32_t tot;
    uint32_t ex = block_excl_scan<uint32_t, RS_T>(run, ws, tot);
    dstart[d] = ex;
    volatile uint64_t *st = status;
    uint64_t excl = 0;
    if (tile == 0) {
      st[d] = OS_INC | run;
    } else {
      st[(uint64_t)tile * 256 + d] = OS_AGG | run;
      int64_t t = (int64_t)tile - 1;
      uint32_t spins = 0;
      while (t >= 0) {
        uint64_t v = st[(uint64_t)t * 256 + d];
        uint64_t f = v & ~OS_VAL;
        if (f == 0) {
          if (++spins > spin_limit) {
            atomicOr(err, ERR_TIMEOUT);
            break;
          }
          if (spins > 64) __nanosleep(64);
          continue;
        }
        excl += v & OS_VAL;
        if (f == OS_INC) break;
        t--;
      }
      st[(uint64_t)tile * 256 + d] = OS_INC | (excl + run);
    }
    tbase[d] = goff[d] + excl - ex;  // + tile-sorted position = output position
  }
  __syncthreads();
  // stage the tile in digit order, then write it out: consecutive threads
  // write consecutive keys of one digit to consecutive output slots
#pragma unroll
  for (int s = 0; s < RS_I; s++) {
    uint64_t idx = base + (uint64_t)s * 32 + lane;
    if (idx < n) {
      uint32_t d = (uint32_t)(k[s] >> shift) & 255u;
      stage[dstart[d] + wh[warp][d] + rank[s]] = k[s];
    }
  }
  __syncthreads();
  // (a tile past the end exists only when tile ids start at 1: no keys)
  const uint32_t valid = tile0 >= n ? 0u
                         : n - tile0 < (uint64_t)RS_TILE ? (uint32_t)(n - tile0) : (uint32_t)RS_TILE;
  for (uint32_t j = threadIdx.x; j < valid; j += RS_T) {
    uint64_t x = stage[j];
    uint32_t d = (uint32_t)(x >> shift) & 255u;
    out[tbase[d] + j] = x;
  }
}

uint64_t radix_tmp_elems(uint64_t n) {
  uint64_t tiles = ceil_div(n, RS_TILE);
  // histograms + digit starts (OS_MAXD x 256 each), status ((tiles + 1) x
  // 256 per digit position -- one spare tile for SortWait::withhold_first --
  // cleared once per sort), tile counters (one word per digit position)
  return 2 * OS_MAXD * 256 + (uint64_t)OS_MAXD * (tiles + 1) * 256 + OS_MAXD + 2;
}

uint64_t *radix_sort_u64(uint64_t *keys, uint64_t *alt, uint64_t n, uint32_t vbits,
                         uint64_t *tmp, cudaStream_t s, Profiler &prof, uint32_t *err,
                         const SortWait &wait) {
  // digit shifts: dst bits [0,vbits) and src bits [32,32+vbits)
  int shifts[16];
  int ns = 0;
  for (int sh = 0; sh < (int)vbits; sh += 8) shifts[ns++] = sh;
  for (int sh = 32; sh < 32 + (int)vbits; sh += 8) shifts[ns++] = sh;
  return radix_sort_u64_shifts(keys, alt, n, shifts, ns, tmp, s, prof, err, wait);
}

uint64_t *radix_sort_u64_shifts(uint64_t *keys, uint64_t *alt, uint64_t n, const int *shifts,
                                int ns, uint64_t *tmp, cudaStream_t s, Profiler &prof,
                                uint32_t *err, const SortWait &wait) {
  if (n <= 1 || ns == 0) return keys;
  if (ns > OS_MAXD) throw_error(TRC_ERR_INVALID, "too many radix digits");
  const uint64_t ntiles = ceil_div(n, RS_TILE);
  if (ntiles > 0xFFFFFFFFull) throw_error(TRC_ERR_INVALID, "sort too large");
  unsigned long long *ghist = (unsigned long long *)tmp;
  uint64_t *goff = tmp + OS_MAXD * 256;
  uint64_t *status = goff + OS_MAXD * 256;
  const uint64_t sstride = (ntiles + 1) * 256;  // status words per digit pass
  uint32_t *ctr = (uint32_t *)(status + (uint64_t)ns * sstride);
  OsShifts sh;
  sh.n = ns;
  for (int i = 0; i < OS_MAXD; i++) sh.s[i] = i < ns ? shifts[i] : 0;
  TRC_CUDA(cudaMemsetAsync(ghist, 0, (size_t)OS_MAXD * 256 * 8, s));
  TRC_CUDA(cudaMemsetAsync(ctr, 0, (size_t)OS_MAXD * 4, s));
  TRC_CUDA(cudaMemsetAsync(status, 0, (size_t)ns * sstride * 8, s));
  const unsigned hgrid = (unsigned)std::min<uint64_t>(ceil_div(n, RS_T * 8), (uint64_t)num_sms() * 8);
  TRC_LAUNCH(prof, s, "radix_hist", hgrid, RS_T, 0, k_os_hist, keys, n, sh, ghist);
  TRC_LAUNCH(prof, s, "radix_prefix", 1, RS_T, 0, k_os_prefix, ghist, ns, goff);
  uint64_t *cur = keys, *nxt = alt;
  for (int i = 0; i < ns; i++) {
    TRC_LAUNCH(prof, s, "radix_scatter", ntiles, RS_T, 0, k_os_scatter, cur, nxt, n, shifts[i],
               goff + i * 256, status + (uint64_t)i * sstride, ctr + i, err, wait.spin_limit,
               wait.withhold_first ? 1u : 0u);
    uint64_t *t = cur;
    cur = nxt;
    nxt = t;
  }
  return cur;
}

// ---------------------------------------------------------------------------
// Bucket sort (see prims.cuh).

namespace {

constexpr uint64_t BK_INVALID = ~0ull;
constexpr uint32_t BK_MID = 256;   // 33..BK_MID keys: a warp in registers
constexpr uint32_t BK_BIG = 2048;  // BK_MID+1..BK_BIG: a CTA in static shared memory
                                   // above: a CTA in dynamic shared memory

// Bucket of a key: with split points (sp, nb + 1 non-decreasing source ids,
// sp[0] = 0, in shared memory) bucket b holds the sources [sp[b], sp[b+1]);
// without, bucket = source >> shift.  Bucket nb holds the invalid keys.
struct BucketArgs {
  uint32_t nb;
  uint32_t shift;
  const uint32_t *sp;  // (shared memory) or null
  __device__ uint32_t of(uint64_t x) const {
    if (x == BK_INVALID) return nb;
    const uint32_t src = (uint32_t)(x >> 32);
    if (!sp) return src >> shift;
    uint32_t lo = 0, hi = nb;  // the last b with sp[b] <= src
    while (hi - lo > 1) {
      const uint32_t m = (lo + hi) >> 1;
      if (sp[m] <= src) lo = m;
      else hi = m;
    }
    return lo;
  }
};

// Counting and placing go by tiles of BK_TILE keys, a CTA each, with the
// tile's bucket counts in shared memory: counts[b * nct + t] = keys of tile
// t in bucket b (bucket-major, so one exclusive scan gives every (bucket,
// tile) its output offset), then each tile places its keys at those offsets
// with shared-memory atomics.  No global atomics: the skewed sources of
// RMAT-like batches do not serialise anywhere.
constexpr uint32_t BK_TILE = 16384;
constexpr uint32_t BK_T = 1024;
constexpr uint32_t BK_MAXB = BUCKET_SPLITS;  // buckets at most (+1 for the invalid keys)

// splits (global, BK_MAXB + 1 entries) or null; the CTA copies them to
// shared memory (after its BK_MAXB + 1 counters)
__device__ __forceinline__ BucketArgs bucket_args_shared(BucketArgs ba, const uint32_t *splits,
                                                         uint32_t *sp) {
  if (splits) {
    for (uint32_t b = threadIdx.x; b <= ba.nb; b += BK_T) sp[b] = splits[b];
    ba.sp = sp;
  }
  return ba;
}

__global__ void __launch_bounds__(BK_T)
    k_bucket_count(const uint64_t *keys, uint64_t k, BucketArgs ba0, const uint32_t *splits,
                   uint32_t nct, uint32_t *counts) {
  extern __shared__ uint32_t bk_smem[];
  uint32_t *h = bk_smem;
  const BucketArgs ba = bucket_args_shared(ba0, splits, bk_smem + BK_MAXB + 1);
  for (uint32_t b = threadIdx.x; b <= ba.nb; b += BK_T) h[b] = 0;
  __syncthreads();
  const uint64_t base = (uint64_t)blockIdx.x * BK_TILE;
  for (uint32_t j = threadIdx.x; j < BK_TILE; j += BK_T) {
    const uint64_t i = base + j;
    if (i < k) atomicAdd(&h[ba.of(keys[i])], 1u);
  }
  __syncthreads();
  for (uint32_t b = threadIdx.x; b <= ba.nb; b += BK_T)
    counts[(uint64_t)b * nct + blockIdx.x] = h[b];
}

struct LoadCnt32 {
  const uint32_t *c;
  __device__ uint64_t operator()(uint64_t i) const { return c[i]; }
};

__global__ void __launch_bounds__(BK_T)
    k_bucket_place(const uint64_t *keys, uint64_t k, BucketArgs ba0, const uint32_t *splits,
                   uint32_t nct, const uint64_t *offm, uint64_t *out) {
  extern __shared__ uint32_t bk_smem[];
  uint32_t *fill = bk_smem;
  const BucketArgs ba = bucket_args_shared(ba0, splits, bk_smem + BK_MAXB + 1);
  for (uint32_t b = threadIdx.x; b <= ba.nb; b += BK_T) fill[b] = 0;
  __syncthreads();
  const uint64_t base = (uint64_t)blockIdx.x * BK_TILE;
  for (uint32_t j = threadIdx.x; j < BK_TILE; j += BK_T) {
    const uint64_t i = base + j;
    if (i < k) {
      const uint64_t x = keys[i];
      const uint32_t b = ba.of(x);
      out[offm[(uint64_t)b * nct + blockIdx.x] + atomicAdd(&fill[b], 1u)] = x;
    }
  }
}

// Bucket boundaries: bucket b holds offm[b * stride] .. offm[(b+1) * stride].
struct BucketOff {
  const uint64_t *offm;
  uint32_t stride;
  __device__ uint64_t operator()(uint64_t b) const { return offm[b * stride]; }
};

// Ascending bitonic network over the 32 lanes of a warp, one value per lane.
__device__ __forceinline__ uint64_t warp_bitonic32(uint64_t v, uint32_t lane) {
#pragma unroll
  for (uint32_t size = 2; size <= 32; size <<= 1) {
#pragma unroll
    for (uint32_t stride = size >> 1; stride > 0; stride >>= 1) {
      const uint64_t o = __shfl_xor_sync(0xFFFFFFFFu, v, stride);
      const bool keep_min = ((lane & size) == 0) == ((lane & stride) == 0);
      v = keep_min ? (o < v ? o : v) : (o > v ? o : v);
    }
  }
  return v;
}

// Ascending bitonic sort of P (a power of two) values in shared memory by
// `nt` threads with index t; `bar` synchronises them.
template <typename Bar>
__device__ __forceinline__ void smem_bitonic(uint64_t *v, uint32_t P, uint32_t t, uint32_t nt,
                                             Bar bar) {
  for (uint32_t size = 2; size <= P; size <<= 1) {
    for (uint32_t stride = size >> 1; stride > 0; stride >>= 1) {
      for (uint32_t c = t; c < P / 2; c += nt) {
        const uint32_t lo = 2 * c - (c & (stride - 1));
        const uint32_t hi = lo + stride;
        const uint64_t x = v[lo], y = v[hi];
        if ((x > y) == ((lo & size) == 0)) {
          v[lo] = y;
          v[hi] = x;
        }
      }
      bar();
    }
  }
}

// Ascending bitonic network over N registers of one thread (all indices
// resolve at compile time, so the values stay in registers).
template <int N>
__device__ __forceinline__ void thread_bucket_sort(uint64_t *keys, uint64_t base, uint32_t c) {
  uint64_t r[N];
#pragma unroll
  for (int i = 0; i < N; i++) r[i] = (uint32_t)i < c ? keys[base + i] : BK_INVALID;
#pragma unroll
  for (int size = 2; size <= N; size <<= 1) {
#pragma unroll
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
#pragma unroll
      for (int i = 0; i < N; i++) {
        const int j = i ^ stride;
        if (j > i) {
          const uint64_t a = r[i], b = r[j];
          const bool sw = ((i & size) == 0) ? (a > b) : (a < b);
          r[i] = sw ? b : a;
          r[j] = sw ? a : b;
        }
      }
    }
  }
#pragma unroll
  for (int i = 0; i < N; i++)
    if ((uint32_t)i < c) keys[base + i] = r[i];
}

// A thread per bucket: buckets of 2..16 keys sorted in the thread's
// registers (network size by the warp's largest such bucket), 17..32 by the
// whole warp; larger ones listed by size for the shared-memory kernels;
// those above BUCKET_SEG_MAX flagged.  lists: 3 lists of `cap` entries,
// nlist their 3 counts.
__global__ void k_bucket_sort_small(BucketOff off, uint32_t nb, uint64_t *keys, uint32_t *lists,
                                    uint64_t cap, unsigned long long *nlist, uint32_t *err) {
  const uint64_t b = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t base = b < nb ? off(b) : 0;
  const uint32_t c = b < nb ? (uint32_t)(off(b + 1) - base) : 0u;
  if (c > 32) {
    if (c > BUCKET_SEG_MAX) {
      atomicOr(err, ERR_BIGSEG);
    } else {
      const int t = c <= BK_MID ? 0 : c <= BK_BIG ? 1 : 2;
      lists[t * cap + atomicAdd(nlist + t, 1ull)] = (uint32_t)b;
    }
  }
  const uint32_t ct = (c >= 2 && c <= 16) ? c : 0u;
  const uint32_t wmax = __reduce_max_sync(0xFFFFFFFFu, ct);
  if (ct) {
    if (wmax <= 4)
      thread_bucket_sort<4>(keys, base, ct);
    else if (wmax <= 8)
      thread_bucket_sort<8>(keys, base, ct);
    else
      thread_bucket_sort<16>(keys, base, ct);
  }
  uint32_t todo = __ballot_sync(0xFFFFFFFFu, c > 16 && c <= 32);
  while (todo) {
    const uint32_t j = __ffs(todo) - 1;
    todo &= todo - 1;
    const uint64_t bj = __shfl_sync(0xFFFFFFFFu, base, j);
    const uint32_t cj = __shfl_sync(0xFFFFFFFFu, c, j);
    uint64_t v = lane < cj ? keys[bj + lane] : BK_INVALID;
    v = warp_bitonic32(v, lane);
    if (lane < cj) keys[bj + lane] = v;
  }
}

// Ascending bitonic sort of 32 * E values held by a warp in registers, lane
// l holding positions l * E .. l * E + E - 1 in r[0 .. E-1]: partners less
// than E apart are in the same lane, the others E * 2^j apart in lane
// l ^ 2^j (shuffles).  Every index resolves at compile time.
template <int E>
__device__ __forceinline__ void warp_regs_bitonic(uint64_t (&r)[E], uint32_t lane) {
  constexpr int N = 32 * E;
#pragma unroll
  for (int size = 2; size <= N; size <<= 1) {
#pragma unroll
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      if (stride < E) {
#pragma unroll
        for (int e = 0; e < E; e++) {
          if ((e & stride) == 0) {
            const int f = e | stride;
            const uint32_t pos = lane * E + e;  // (pos & size) is the block's direction
            const bool up = (pos & size) == 0;
            const uint64_t x = r[e], y = r[f];
            const bool sw = up ? (x > y) : (x < y);
            r[e] = sw ? y : x;
            r[f] = sw ? x : y;
          }
        }
      } else {
        const int lx = stride / E;  // partner lane offset
#pragma unroll
        for (int e = 0; e < E; e++) {
          const uint64_t o = __shfl_xor_sync(0xFFFFFFFFu, r[e], lx);
          const uint32_t pos = lane * E + e;
          const bool up = (pos & size) == 0, lower = (pos & stride) == 0;
          r[e] = (up == lower) ? (o < r[e] ? o : r[e]) : (o > r[e] ? o : r[e]);
        }
      }
    }
  }
}

template <int E>
__device__ __forceinline__ void warp_regs_sort_bucket(uint64_t *keys, uint64_t base, uint32_t c,
                                                      uint32_t lane) {
  uint64_t r[E];
#pragma unroll
  for (int e = 0; e < E; e++) {
    const uint32_t t = lane * E + e;
    r[e] = t < c ? keys[base + t] : BK_INVALID;
  }
  warp_regs_bitonic<E>(r, lane);
#pragma unroll
  for (int e = 0; e < E; e++) {
    const uint32_t t = lane * E + e;
    if (t < c) keys[base + t] = r[e];
  }
}

// A warp per listed bucket of 33..BK_MID keys, sorted in registers (no
// shared memory: the 64-bit compare-exchanges in shared memory met bank
// conflicts at most strides).
constexpr uint32_t BK_MID_WARPS = 8;
__global__ void __launch_bounds__(BK_MID_WARPS * 32)
    k_bucket_sort_mid(BucketOff off, const uint32_t *list, const unsigned long long *nlist,
                      uint64_t *keys) {
  const uint32_t w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint64_t nm = *nlist;
  for (uint64_t i = (uint64_t)blockIdx.x * BK_MID_WARPS + w; i < nm;
       i += (uint64_t)gridDim.x * BK_MID_WARPS) {
    const uint32_t b = list[i];
    const uint64_t base = off(b);
    const uint32_t c = (uint32_t)(off(b + 1) - base);
    if (c <= 64) warp_regs_sort_bucket<2>(keys, base, c, lane);
    else if (c <= 128) warp_regs_sort_bucket<4>(keys, base, c, lane);
    else warp_regs_sort_bucket<8>(keys, base, c, lane);  // (c <= BK_MID = 256)
  }
}

// A CTA per listed bucket of more than BK_MID keys (at most PMAX), sorted in
// shared memory: static for PMAX = BK_BIG, dynamic otherwise.
template <uint32_t PMAX, uint32_t NT>
__global__ void __launch_bounds__(NT)
    k_bucket_sort_cta(BucketOff off, const uint32_t *list, const unsigned long long *nlist,
                      uint64_t *keys) {
  __shared__ uint64_t sstat[PMAX <= BK_BIG ? PMAX : 1];
  extern __shared__ uint64_t sdyn[];
  uint64_t *v = PMAX <= BK_BIG ? sstat : sdyn;
  const uint64_t nbg = *nlist;
  for (uint64_t i = blockIdx.x; i < nbg; i += gridDim.x) {
    const uint32_t b = list[i];
    const uint64_t base = off(b);
    const uint32_t c = (uint32_t)(off(b + 1) - base);
    uint32_t P = 2 * BK_MID;
    while (P < c) P <<= 1;
    for (uint32_t t = threadIdx.x; t < P; t += NT) v[t] = t < c ? keys[base + t] : BK_INVALID;
    __syncthreads();
    smem_bitonic(v, P, threadIdx.x, NT, [] { __syncthreads(); });
    for (uint32_t t = threadIdx.x; t < c; t += NT) keys[base + t] = v[t];
    __syncthreads();
  }
}

constexpr uint32_t SORT_SMALL_T = 512;

__global__ void __launch_bounds__(SORT_SMALL_T) k_sort_small(const uint64_t *in, uint32_t k,
                                                              uint64_t *out) {
  __shared__ uint64_t v[SORT_SMALL_MAX];
  uint32_t P = 2;
  while (P < k) P <<= 1;
  // padding with the largest key: the first k sorted values are the keys
  for (uint32_t t = threadIdx.x; t < P; t += SORT_SMALL_T) v[t] = t < k ? in[t] : BK_INVALID;
  __syncthreads();
  smem_bitonic(v, P, threadIdx.x, SORT_SMALL_T, [] { __syncthreads(); });
  for (uint32_t t = threadIdx.x; t < k; t += SORT_SMALL_T) out[t] = v[t];
}

struct BucketLayout {
  uint32_t nb, shift, nct;
  uint64_t cells;  // (nb + 1) * nct
  uint64_t list_cap;
  uint64_t cnt_w, off_w, scan_w, list_w;  // words of each part
  uint64_t total() const { return cnt_w + off_w + scan_w + list_w + 3; }
};

BucketLayout bucket_layout(uint64_t k, uint32_t n, bool splits) {
  BucketLayout L{};
  if (splits) {  // the split points' BK_MAXB buckets
    L.nb = BK_MAXB;
  } else {  // about 128 keys per bucket, at most BK_MAXB: bucket = source >> shift
    const uint64_t target = std::max<uint64_t>(1, std::min<uint64_t>(BK_MAXB, k / 128));
    L.shift = 0;
    while (L.shift < 31 && ceil_div((uint64_t)n, 1ull << L.shift) > target) L.shift++;
    L.nb = (uint32_t)ceil_div((uint64_t)n, 1ull << L.shift);
  }
  L.nct = (uint32_t)ceil_div(k, BK_TILE);
  L.cells = ((uint64_t)L.nb + 1) * L.nct;
  L.list_cap = std::min<uint64_t>(L.nb, k / 33) + 1;
  L.cnt_w = ceil_div(L.cells, 2);
  L.off_w = L.cells + 1;
  L.scan_w = scan_tmp_elems(L.cells) + 4;
  L.list_w = ceil_div(3 * L.list_cap, 2);
  return L;
}

// split j = the source of sorted key j * k / BK_MAXB (sources of invalid
// keys read as n): BK_MAXB buckets of about equal counts for batches drawn
// like this one
__global__ void k_bucket_learn(const uint64_t *sorted, uint64_t k, uint32_t n, uint32_t *splits) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j > BK_MAXB) return;
  uint32_t v = n;
  if (j == 0) {
    v = 0;
  } else if (j < BK_MAXB) {
    const uint64_t x = sorted[(uint64_t)j * k / BK_MAXB];
    v = x == BK_INVALID ? n : (uint32_t)(x >> 32);
  }
  splits[j] = v;
}

}  // namespace

void bucket_learn_splits(const uint64_t *sorted, uint64_t k, uint32_t n, uint32_t *splits,
                         cudaStream_t s, Profiler &prof) {
  if (k == 0) return;
  TRC_LAUNCH(prof, s, "bsort_learn", ceil_div(BUCKET_SPLITS + 1, 256), 256, 0, k_bucket_learn,
             sorted, k, n, splits);
}

uint64_t bucket_tmp_elems(uint64_t k, uint32_t n, bool splits) {
  return bucket_layout(k, n, splits).total();
}

uint64_t *sort_small_u64(const uint64_t *keys, uint64_t *alt, uint64_t k, cudaStream_t s,
                         Profiler &prof) {
  if (k > SORT_SMALL_MAX) throw_error(TRC_ERR_INVALID, "sort_small_u64: more than 2048 keys");
  if (k == 0) return alt;
  TRC_LAUNCH(prof, s, "sort_small", 1, SORT_SMALL_T, 0, k_sort_small, keys, (uint32_t)k, alt);
  return alt;
}

uint64_t *bucket_sort_u64(const uint64_t *keys, uint64_t *alt, uint64_t k, uint32_t n,
                          uint64_t *tmp, cudaStream_t s, Profiler &prof, uint32_t *err,
                          const uint32_t *splits) {
  if (k == 0) return alt;
  const BucketLayout L = bucket_layout(k, n, splits != nullptr);
  const BucketArgs ba{L.nb, L.shift, nullptr};
  uint32_t *counts = reinterpret_cast<uint32_t *>(tmp);
  uint64_t *offm = tmp + L.cnt_w;
  uint64_t *st = offm + L.off_w;
  uint32_t *lists = reinterpret_cast<uint32_t *>(st + L.scan_w);
  unsigned long long *nlist = reinterpret_cast<unsigned long long *>(st + L.scan_w + L.list_w);
  TRC_CUDA(cudaMemsetAsync(nlist, 0, 3 * 8, s));
  const int smem = (int)(2 * (BK_MAXB + 1) * sizeof(uint32_t));  // counters + split points
  TRC_CUDA(cudaFuncSetAttribute(k_bucket_count, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  TRC_CUDA(cudaFuncSetAttribute(k_bucket_place, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  TRC_LAUNCH(prof, s, "bsort_count", L.nct, BK_T, smem, k_bucket_count, keys, k, ba, splits, L.nct,
             counts);
  exclusive_scan(LoadCnt32{counts}, L.cells, offm, st, s, prof, "bsort_scan");
  TRC_LAUNCH(prof, s, "bsort_place", L.nct, BK_T, smem, k_bucket_place, keys, k, ba, splits, L.nct,
             offm, alt);
  const BucketOff off{offm, L.nct};
  TRC_LAUNCH(prof, s, "bsort_small", ceil_div((uint64_t)L.nb, 256), 256, 0, k_bucket_sort_small,
             off, L.nb, alt, lists, L.list_cap, nlist, err);
  const unsigned sms = (unsigned)num_sms();
  TRC_LAUNCH(prof, s, "bsort_mid", sms * 4, BK_MID_WARPS * 32, 0, k_bucket_sort_mid, off, lists,
             nlist, alt);
  TRC_LAUNCH(prof, s, "bsort_big", sms * 4, 256, 0, (k_bucket_sort_cta<BK_BIG, 256>), off,
             lists + L.list_cap, nlist + 1, alt);
  const int huge_smem = (int)(BUCKET_SEG_MAX * sizeof(uint64_t));
  TRC_CUDA(cudaFuncSetAttribute(k_bucket_sort_cta<BUCKET_SEG_MAX, 1024>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, huge_smem));
  TRC_LAUNCH(prof, s, "bsort_huge", sms, 1024, huge_smem, (k_bucket_sort_cta<BUCKET_SEG_MAX, 1024>),
             off, lists + 2 * L.list_cap, nlist + 2, alt);
  return alt;
}

// ---------------------------------------------------------------------------
// Merge path.  Output tile t covers diagonals [t*MT, (t+1)*MT); its split
// points are found by binary search, the two input ranges staged in shared
// memory, and each thread merges MI consecutive outputs.
constexpr int MT_T = 128;
constexpr int MT_I = 8;
constexpr int MT = MT_T * MT_I;  // 1024 outputs per tile

__device__ __forceinline__ uint64_t merge_path_split(const uint64_t *A, uint64_t na,
                                                     const uint64_t *B, uint64_t nb,
                                                     uint64_t diag) {
  uint64_t lo = diag > nb ? diag - nb : 0;
  uint64_t hi = diag < na ? diag : na;
  while (lo < hi) {
    uint64_t mid = (lo + hi) >> 1;
    if (A[mid] <= B[diag - 1 - mid]) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

__global__ void __launch_bounds__(MT_T) k_merge(const uint64_t *A, uint64_t na, const uint64_t *B,
                                                uint64_t nb, uint64_t *out) {
  __shared__ uint64_t sm[MT];
  __shared__ uint64_t split[2];
  uint64_t total = na + nb;
  uint64_t d0 = (uint64_t)blockIdx.x * MT;
  uint64_t d1 = d0 + MT < total ? d0 + MT : total;
  if (threadIdx.x < 2) split[threadIdx.x] = merge_path_split(A, na, B, nb, threadIdx.x ? d1 : d0);
  __syncthreads();
  uint64_t a0 = split[0], a1 = split[1];
  uint64_t b0 = d0 - a0, b1 = d1 - a1;
  uint32_t la = (uint32_t)(a1 - a0), lb = (uint32_t)(b1 - b0);
  for (uint32_t i = threadIdx.x; i < la; i += MT_T) sm[i] = A[a0 + i];
  for (uint32_t i = threadIdx.x; i < lb; i += MT_T) sm[la + i] = B[b0 + i];
  __syncthreads();
  // thread-local split inside the tile
  uint32_t diag = threadIdx.x * MT_I;
  uint32_t tot = la + lb;
  if (diag >= tot) return;
  const uint64_t *SA = sm, *SB = sm + la;
  uint32_t lo = diag > lb ? diag - lb : 0, hi = diag < la ? diag : la;
  while (lo < hi) {
    uint32_t mid = (lo + hi) >> 1;
    if (SA[mid] <= SB[diag - 1 - mid]) lo = mid + 1;
    else hi = mid;
  }
  uint32_t i = lo, j = diag - lo;
  uint32_t end = diag + MT_I < tot ? diag + MT_I : tot;
  for (uint32_t o = diag; o < end; o++) {
    bool takeA = j >= lb || (i < la && SA[i] <= SB[j]);
    out[d0 + o] = takeA ? SA[i++] : SB[j++];
  }
}

void merge_u64(const uint64_t *A, uint64_t na, const uint64_t *B, uint64_t nb, uint64_t *out,
               cudaStream_t s, Profiler &prof) {
  uint64_t tiles = ceil_div(na + nb, MT);
  TRC_LAUNCH(prof, s, "merge", tiles, MT_T, 0, k_merge, A, na, B, nb, out);
}

// ---------------------------------------------------------------------------
// Sorted difference A \ B with B a subset of A (deleted edges all exist):
// every element of B is located in A by binary search (|B| log |A| work, B is
// the small side) and flagged, then A is compacted without the flagged ones.
__global__ void k_flag_members(const uint64_t *A, uint64_t na, const uint64_t *B, uint64_t nb,
                               uint8_t *flags) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nb) return;
  uint64_t x = B[i];
  uint64_t lo = 0, hi = na;
  while (lo < hi) {
    uint64_t mid = (lo + hi) >> 1;
    if (A[mid] < x) lo = mid + 1;
    else hi = mid;
  }
  if (lo < na && A[lo] == x) flags[lo] = 1;
}

struct NotFlagged {
  const uint8_t *f;
  __device__ bool operator()(uint64_t i) const { return f[i] == 0; }
};

void difference_u64(const uint64_t *A, uint64_t na, const uint64_t *B, uint64_t nb,
                    uint64_t *out, uint64_t *count, uint8_t *flags, uint64_t *tmp,
                    cudaStream_t s, Profiler &prof) {
  if (na) TRC_CUDA(cudaMemsetAsync(flags, 0, na, s));
  TRC_LAUNCH(prof, s, "diff_flag", ceil_div(nb, 256), 256, 0, k_flag_members, A, na, B, nb, flags);
  select_if(NotFlagged{flags}, LoadU64{A}, na, out, count, tmp, s, prof);
}

}  // namespace trc
