// prims.cuh -- data-parallel primitives for the update pipeline: exclusive
// scan, order-preserving select (stream compaction), LSD radix sort of
// 64-bit keys, merge-path merge and sorted difference.  Each primitive is a
// few tiled kernels; tiles are sized so that a grid is many waves of the
// 148 SMs for the batch sizes the path sees (1e1..1e9 keys).
#pragma once

#include "trc_common.cuh"

namespace trc {

constexpr int PT = 256;          // threads per CTA for the primitives
constexpr int PI = 8;            // items per thread
constexpr int PTILE = PT * PI;   // 2048 items per tile

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31; }
__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

template <typename T>
__device__ __forceinline__ T warp_incl_scan(T v) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T t = __shfl_up_sync(0xFFFFFFFFu, v, o);
    if ((int)lane_id() >= o) v += t;
  }
  return v;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
  return v;
}

// Block-wide exclusive scan of one value per thread; returns the exclusive
// prefix and sets `total`.  `ws` is shared scratch of NT/32 entries.
template <typename T, int NT>
__device__ __forceinline__ T block_excl_scan(T v, T *ws, T &total) {
  T inc = warp_incl_scan(v);
  int w = threadIdx.x >> 5;
  if (lane_id() == 31) ws[w] = inc;
  __syncthreads();
  if (w == 0) {
    T x = (lane_id() < NT / 32) ? ws[lane_id()] : T(0);
    T xi = warp_incl_scan(x);
    if (lane_id() < NT / 32) ws[lane_id()] = xi - x;
    if (lane_id() == NT / 32 - 1) ws[NT / 32] = xi;
  }
  __syncthreads();
  T r = inc - v + ws[w];
  total = ws[NT / 32];
  __syncthreads();
  return r;
}

// ------------------------------------------------------------------- scan
// Exclusive scan of f(i), i < n, into out[0..n] (out[n] = total).  The
// functor returns uint64_t.  Three phases: tile sums, scan of tile sums
// (recursive), tile scan with the tile offset.

template <typename F>
__global__ void k_tile_sum(F f, uint64_t n, uint64_t *tile_sums) {
  __shared__ uint64_t ws[PT / 32 + 1];
  uint64_t base = (uint64_t)blockIdx.x * PTILE;
  uint64_t s = 0;
#pragma unroll
  for (int i = 0; i < PI; i++) {
    uint64_t idx = base + (uint64_t)i * PT + threadIdx.x;
    if (idx < n) s += f(idx);
  }
  uint64_t tot;
  block_excl_scan<uint64_t, PT>(s, ws, tot);
  if (threadIdx.x == 0) tile_sums[blockIdx.x] = tot;
}

// The tile goes through shared memory so that global loads and stores are
// coalesced (item i*PT + t by thread t) while each thread scans PI
// consecutive items; a pad word after every 16 keeps both access patterns
// free of bank conflicts.
__device__ __forceinline__ uint32_t pad16(uint32_t j) { return j + (j >> 4); }

template <typename F>
__global__ void k_tile_scan(F f, uint64_t n, const uint64_t *tile_off, uint64_t *out) {
  __shared__ uint64_t sv[PTILE + PTILE / 16];
  __shared__ uint64_t ws[PT / 32 + 1];
  const uint64_t base = (uint64_t)blockIdx.x * PTILE;
#pragma unroll
  for (int i = 0; i < PI; i++) {
    const uint32_t j = i * PT + threadIdx.x;
    sv[pad16(j)] = base + j < n ? f(base + j) : 0;
  }
  __syncthreads();
  uint64_t v[PI];
  uint64_t s = 0;
#pragma unroll
  for (int i = 0; i < PI; i++) {
    v[i] = sv[pad16(threadIdx.x * PI + i)];
    s += v[i];
  }
  uint64_t tot;
  uint64_t ex = block_excl_scan<uint64_t, PT>(s, ws, tot);
  ex += tile_off[blockIdx.x];
#pragma unroll
  for (int i = 0; i < PI; i++) {
    sv[pad16(threadIdx.x * PI + i)] = ex;
    ex += v[i];
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < PI; i++) {
    const uint32_t j = i * PT + threadIdx.x;
    if (base + j < n) out[base + j] = sv[pad16(j)];
  }
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == PT - 1) out[n] = ex;
}

struct LoadU64 {
  const uint64_t *p;
  __device__ uint64_t operator()(uint64_t i) const { return p[i]; }
};

struct LoadU32 {
  const uint32_t *p;
  __device__ uint64_t operator()(uint64_t i) const { return p[i]; }
};

class Scratch;

// Exclusive scan into out[0..n]; tmp needs scan_tmp_elems(n) entries.
inline uint64_t scan_tmp_elems(uint64_t n) {
  uint64_t t = ceil_div(n, PTILE);
  if (t <= 1) return 2;
  return 2 * t + 1 + scan_tmp_elems(t);
}

template <typename F>
void exclusive_scan(F f, uint64_t n, uint64_t *out, uint64_t *tmp, cudaStream_t s, Profiler &prof,
                    const char *tag = "scan") {
  if (n == 0) {
    TRC_CUDA(cudaMemsetAsync(out, 0, sizeof(uint64_t), s));
    return;
  }
  const std::string t_sum = std::string(tag) + ".sum", t_tile = std::string(tag) + ".tile";
  uint64_t tiles = ceil_div(n, PTILE);
  if (tiles == 1) {
    TRC_CUDA(cudaMemsetAsync(tmp, 0, sizeof(uint64_t), s));
    TRC_LAUNCH(prof, s, t_tile.c_str(), 1, PT, 0, k_tile_scan<F>, f, n, tmp, out);
    return;
  }
  uint64_t *sums = tmp;              // tiles entries
  uint64_t *offs = tmp + tiles;      // tiles+1 entries
  TRC_LAUNCH(prof, s, t_sum.c_str(), tiles, PT, 0, k_tile_sum<F>, f, n, sums);
  exclusive_scan(LoadU64{sums}, tiles, offs, offs + tiles + 1, s, prof, "scan_tiles");
  TRC_LAUNCH(prof, s, t_tile.c_str(), tiles, PT, 0, k_tile_scan<F>, f, n, offs, out);
}

// ----------------------------------------------------------------- select
// Order-preserving compaction: out[j] = val(i) for the j-th i < n with
// pred(i).  *count (device) receives the number selected.

template <typename P>
struct PredCount {
  P p;
  __device__ uint64_t operator()(uint64_t i) const { return p(i) ? 1 : 0; }
};

// Round i of a tile covers items i*PT + t (coalesced predicate and value
// reads); an item's rank in the tile is the selected count of earlier
// rounds, then of earlier warps of its round, then of earlier lanes, so
// consecutive selected items go to consecutive slots from consecutive lanes.
template <typename P, typename V, typename T>
__global__ void k_select_scatter(P pred, V val, uint64_t n, const uint64_t *tile_off, T *out,
                                 uint64_t *count) {
  constexpr int NW = PT / 32;
  static_assert(PI * NW == 64, "one warp scans the tile's (round, warp) counts, two per lane");
  __shared__ uint32_t wc[PI * NW + 1];  // + the tile's total
  const uint64_t base = (uint64_t)blockIdx.x * PTILE;
  const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  uint32_t m[PI];
#pragma unroll
  for (int i = 0; i < PI; i++) {
    const uint64_t idx = base + (uint64_t)i * PT + threadIdx.x;
    m[i] = __ballot_sync(0xFFFFFFFFu, idx < n && pred(idx));
    if (lane == 0) wc[i * NW + w] = __popc(m[i]);
  }
  __syncthreads();
  if (w == 0) {
    const uint32_t a = wc[2 * lane], b = wc[2 * lane + 1];
    const uint32_t in = warp_incl_scan(a + b);
    const uint32_t ex = in - (a + b);
    wc[2 * lane] = ex;
    wc[2 * lane + 1] = ex + a;
    if (lane == 31) wc[PI * NW] = in;
  }
  __syncthreads();
  // (tile_off null: a single tile, its own offset 0 and total the count)
  const uint64_t off = tile_off ? tile_off[blockIdx.x] : 0;
  const uint32_t lt = lanemask_lt();
#pragma unroll
  for (int i = 0; i < PI; i++) {
    if ((m[i] >> lane) & 1u)
      out[off + wc[i * NW + w] + __popc(m[i] & lt)] = val(base + (uint64_t)i * PT + threadIdx.x);
  }
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0)
    *count = tile_off ? tile_off[gridDim.x] : wc[PI * NW];
}

template <typename P, typename V, typename T>
void select_if(P pred, V val, uint64_t n, T *out, uint64_t *count, uint64_t *tmp, cudaStream_t s,
               Profiler &prof, const char *tag = "select") {
  if (n == 0) {
    TRC_CUDA(cudaMemsetAsync(count, 0, sizeof(uint64_t), s));
    return;
  }
  const std::string t_cnt = std::string(tag) + ".count", t_sc = std::string(tag) + ".scatter";
  uint64_t tiles = ceil_div(n, PTILE);
  auto kscatter = k_select_scatter<P, V, T>;
  if (tiles == 1) {  // one launch: the tile counts, ranks and writes its items
    TRC_LAUNCH(prof, s, t_sc.c_str(), 1, PT, 0, kscatter, pred, val, n, (const uint64_t *)nullptr,
               out, count);
    return;
  }
  uint64_t *sums = tmp;
  uint64_t *offs = tmp + tiles;
  TRC_LAUNCH(prof, s, t_cnt.c_str(), tiles, PT, 0, k_tile_sum<PredCount<P>>, PredCount<P>{pred}, n,
             sums);
  exclusive_scan(LoadU64{sums}, tiles, offs, offs + tiles + 1, s, prof, "scan_tiles");
  TRC_LAUNCH(prof, s, t_sc.c_str(), tiles, PT, 0, kscatter, pred, val, n, offs, out, count);
}

inline uint64_t select_tmp_elems(uint64_t n) {
  uint64_t t = ceil_div(n, PTILE);
  return 2 * t + 1 + scan_tmp_elems(t) + 2;
}

// ------------------------------------------------------------- radix sort
// LSD radix sort of 64-bit keys, 8-bit digits, stable, one sweep per digit
// (prims.cu).  Only the digit positions listed are sorted (keys are
// (src<<32)|dst with src,dst < 2^b, so the digits at shifts 0,8,..<b and
// 32,40,..<32+b suffice).
constexpr int RS_T = 256;
constexpr int RS_I = 16;
constexpr int RS_TILE = RS_T * RS_I;  // 4096 keys
constexpr int RS_W = RS_T / 32;

// The bounded look-back wait of the scatter passes: a tile gives up after
// spin_limit polls of a predecessor that has not published.  withhold_first
// (tests of that bound only) starts the tile ids at 1, so no tile 0 ever
// publishes and every wait runs out; the keys of tile 0 are then not sorted
// and the call must fail.
struct SortWait {
  uint32_t spin_limit = 1u << 22;
  uint32_t withhold_first = 0;
};

// Sorts keys[0..n) using alt as the ping-pong buffer; returns the buffer that
// holds the result (keys or alt).  tmp needs radix_tmp_elems(n) entries.
// err: device error word; ERR_TIMEOUT is or-ed in if a look-back wait gave
// up (the caller must then fail the call).
uint64_t *radix_sort_u64(uint64_t *keys, uint64_t *alt, uint64_t n, uint32_t vbits,
                         uint64_t *tmp, cudaStream_t s, Profiler &prof, uint32_t *err,
                         const SortWait &wait = SortWait{});
// Same, over an explicit list of at most 8 digit shifts (least significant
// first).
uint64_t *radix_sort_u64_shifts(uint64_t *keys, uint64_t *alt, uint64_t n, const int *shifts,
                                int ns, uint64_t *tmp, cudaStream_t s, Profiler &prof,
                                uint32_t *err, const SortWait &wait = SortWait{});
uint64_t radix_tmp_elems(uint64_t n);

// ------------------------------------------------------------ bucket sort
// Sorts k keys (src<<32|dst with src < n, or KEY_INVALID = ~0) ascending in
// one MSD pass plus whole-bucket sorts.  Buckets are source ranges: with
// `splits` (BUCKET_SPLITS + 1 non-decreasing source ids, splits[0] = 0, as
// bucket_learn_splits writes them) bucket b holds the sources
// [splits[b], splits[b+1]), so a batch drawn like the one the splits were
// learned from fills the buckets about evenly however skewed its sources
// are; without, bucket = source >> shift (about 128 keys per bucket for
// uniform sources).  Tiles of 16384 keys count their buckets in shared
// memory, one scan of the (bucket, tile) counts gives every tile its output
// offsets, the tiles place their keys, and each bucket is then sorted whole
// (up to 16 keys in a thread's registers, up to 32 across a warp, up to 256
// in a warp's shared memory, up to BUCKET_SEG_MAX by a CTA).  No global
// atomics.  A bucket above BUCKET_SEG_MAX keys is left unsorted and
// ERR_BIGSEG or-ed into err: the caller must then sort with the radix sort
// instead.  Writes the sorted keys to alt (keys is left unchanged) and
// returns alt.  tmp: bucket_tmp_elems(k, n, splits != null) entries.
constexpr uint32_t BUCKET_SEG_MAX = 16384;
constexpr uint32_t BUCKET_SPLITS = 8192;
uint64_t *bucket_sort_u64(const uint64_t *keys, uint64_t *alt, uint64_t k, uint32_t n,
                          uint64_t *tmp, cudaStream_t s, Profiler &prof, uint32_t *err,
                          const uint32_t *splits);
uint64_t bucket_tmp_elems(uint64_t k, uint32_t n, bool splits);
// Sort of at most SORT_SMALL_MAX keys by one CTA (a bitonic network in shared
// memory): one launch where the radix sort takes eleven operations.  Writes
// the sorted keys to alt (keys unchanged) and returns alt.
constexpr uint32_t SORT_SMALL_MAX = 2048;
uint64_t *sort_small_u64(const uint64_t *keys, uint64_t *alt, uint64_t k, cudaStream_t s,
                         Profiler &prof);
// Split points for the next batches from a sorted batch of k keys: split j =
// the source of key j * k / BUCKET_SPLITS (n for invalid keys), split 0 = 0,
// split BUCKET_SPLITS = n.
void bucket_learn_splits(const uint64_t *sorted, uint64_t k, uint32_t n, uint32_t *splits,
                         cudaStream_t s, Profiler &prof);

// ------------------------------------------------------------ merge path
// Merge of two sorted u64 arrays without common elements (A first on ties).
__global__ void k_merge(const uint64_t *A, uint64_t na, const uint64_t *B, uint64_t nb,
                        uint64_t *out);
void merge_u64(const uint64_t *A, uint64_t na, const uint64_t *B, uint64_t nb, uint64_t *out,
               cudaStream_t s, Profiler &prof);

// out = A \ B for sorted unique A and sorted B that is a subset of A.
// flags: na bytes; tmp: select_tmp_elems(na).
void difference_u64(const uint64_t *A, uint64_t na, const uint64_t *B, uint64_t nb,
                    uint64_t *out, uint64_t *count, uint8_t *flags, uint64_t *tmp,
                    cudaStream_t s, Profiler &prof);

}  // namespace trc
