// prims.cu -- radix sort, merge-path merge and sorted difference of 64-bit
// keys (declarations and the scan/select templates are in prims.cuh).
#include "prims.cuh"

namespace trc {

// ---------------------------------------------------------------------------
// Radix sort.  Per 8-bit digit: (1) per-tile digit histogram, written
// digit-major so that (2) one exclusive scan gives every (digit, tile) its
// global output offset, then (3) a stable scatter: each warp ranks its keys
// with __match_any_sync, warps are combined with a per-digit prefix in
// shared memory.

__global__ void k_rs_hist(const uint64_t *in, uint64_t n, int shift, uint32_t ntiles,
                          uint64_t *hist) {
  __shared__ uint32_t h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  uint64_t base = (uint64_t)blockIdx.x * RS_TILE;
#pragma unroll 4
  for (int i = 0; i < RS_I; i++) {
    uint64_t idx = base + (uint64_t)i * RS_T + threadIdx.x;
    if (idx < n) atomicAdd(&h[(uint32_t)(in[idx] >> shift) & 255u], 1u);
  }
  __syncthreads();
  hist[(uint64_t)threadIdx.x * ntiles + blockIdx.x] = h[threadIdx.x];
}

__global__ void __launch_bounds__(RS_T) k_rs_scatter(const uint64_t *in, uint64_t *out, uint64_t n,
                                                     int shift, uint32_t ntiles,
                                                     const uint64_t *offs) {
  __shared__ uint32_t wh[RS_W][256];
  __shared__ uint64_t tbase[256];
  for (int i = threadIdx.x; i < RS_W * 256; i += RS_T) (&wh[0][0])[i] = 0;
  tbase[threadIdx.x] = offs[(uint64_t)threadIdx.x * ntiles + blockIdx.x];
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // warp w owns keys [base, base + RS_I*32) of the tile, slot-major
  uint64_t base = (uint64_t)blockIdx.x * RS_TILE + (uint64_t)warp * (RS_I * 32);
  uint64_t k[RS_I];
  uint32_t rank[RS_I];
  uint32_t lt = lanemask_lt();
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
    uint32_t d = threadIdx.x, run = 0;
#pragma unroll
    for (int w = 0; w < RS_W; w++) {
      uint32_t c = wh[w][d];
      wh[w][d] = run;
      run += c;
    }
  }
  __syncthreads();
#pragma unroll
  for (int s = 0; s < RS_I; s++) {
    uint64_t idx = base + (uint64_t)s * 32 + lane;
    if (idx < n) {
      uint32_t d = (uint32_t)(k[s] >> shift) & 255u;
      out[tbase[d] + wh[warp][d] + rank[s]] = k[s];
    }
  }
}

uint64_t radix_tmp_elems(uint64_t n) {
  uint64_t tiles = ceil_div(n, RS_TILE);
  return tiles * 256 + scan_tmp_elems(tiles * 256) + tiles * 256 + 2;
}

uint64_t *radix_sort_u64(uint64_t *keys, uint64_t *alt, uint64_t n, uint32_t vbits,
                         uint64_t *tmp, cudaStream_t s, Profiler &prof) {
  // digit shifts: dst bits [0,vbits) and src bits [32,32+vbits)
  int shifts[16];
  int ns = 0;
  for (int sh = 0; sh < (int)vbits; sh += 8) shifts[ns++] = sh;
  for (int sh = 32; sh < 32 + (int)vbits; sh += 8) shifts[ns++] = sh;
  return radix_sort_u64_shifts(keys, alt, n, shifts, ns, tmp, s, prof);
}

uint64_t *radix_sort_u64_shifts(uint64_t *keys, uint64_t *alt, uint64_t n, const int *shifts,
                                int ns, uint64_t *tmp, cudaStream_t s, Profiler &prof) {
  if (n <= 1) return keys;
  uint32_t ntiles = (uint32_t)ceil_div(n, RS_TILE);
  uint64_t *hist = tmp;
  uint64_t *offs = tmp + (uint64_t)ntiles * 256;
  uint64_t *stmp = offs + (uint64_t)ntiles * 256 + 1;
  uint64_t *cur = keys, *nxt = alt;
  for (int i = 0; i < ns; i++) {
    TRC_LAUNCH(prof, s, "radix_hist", ntiles, RS_T, 0, k_rs_hist, cur, n, shifts[i], ntiles, hist);
    exclusive_scan(LoadU64{hist}, (uint64_t)ntiles * 256, offs, stmp, s, prof);
    TRC_LAUNCH(prof, s, "radix_scatter", ntiles, RS_T, 0, k_rs_scatter, cur, nxt, n, shifts[i],
               ntiles, offs);
    uint64_t *t = cur;
    cur = nxt;
    nxt = t;
  }
  return cur;
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
