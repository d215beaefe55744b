// msbfs.cu -- multi-source BFS: up to 64 sources at once as one bit per
// source in a 64-bit mask per vertex (the batching layer; the reference runs
// BFS_with_edge_map once per source, include/BFS.h:41-84).
//
// Per vertex: seen[v] (sources that reached v), front[v] (sources whose
// frontier holds v at this level).  A level computes, for every vertex,
// reach = OR of front over its neighbours; new = reach & ~seen[v] gives the
// sources discovering v at level L+1.  Two directions, as in the single-
// source BFS:
//   pull  -- every vertex not yet seen by every live source (one whose
//            frontier is not empty) ORs its neighbours' front masks,
//            stopping once nothing more can be added
//            (4 lanes per inline-only vertex, a warp per larger vertex);
//   push  -- when few vertices are in any frontier, each active vertex ORs
//            its mask into its neighbours' next masks (64-bit atomicOr).
// Levels are written vertex-major (one 256-byte row per vertex, contiguous
// writes) and transposed to one row per source at the end.
#include <algorithm>
#include <vector>

#include "graph.cuh"

namespace trc {

namespace {
constexpr int MT = 256;

__device__ __forceinline__ uint64_t shfl_or64(uint64_t x, int o) {
  uint32_t lo = (uint32_t)x, hi = (uint32_t)(x >> 32);
  lo |= __shfl_xor_sync(0xFFFFFFFFu, lo, o);
  hi |= __shfl_xor_sync(0xFFFFFFFFu, hi, o);
  return ((uint64_t)hi << 32) | lo;
}

struct MSState {
  uint64_t *seen;
  const uint64_t *front;
  uint64_t *next;   // pull: written per vertex; push: OR-accumulated
  uint32_t *lvrow;  // n x k levels, vertex-major; null: summary only
  uint32_t k;
  uint64_t live;    // sources whose frontier is not empty at this level:
                    // only their bits can still be discovered
  uint32_t level;   // the level being discovered (L+1)
};

__device__ __forceinline__ void write_levels(const MSState &s, uint64_t v, uint64_t nw) {
  while (nw) {
    int i = __ffsll((long long)nw) - 1;
    nw &= nw - 1;
    s.lvrow[v * s.k + i] = s.level;
  }
}

// OR of x over the warp into *dst (one atomic per warp); every lane calls
__device__ __forceinline__ void warp_or_into(uint64_t x, unsigned long long *dst) {
  uint32_t lo = __reduce_or_sync(0xFFFFFFFFu, (uint32_t)x);
  uint32_t hi = __reduce_or_sync(0xFFFFFFFFu, (uint32_t)(x >> 32));
  uint64_t r = ((uint64_t)hi << 32) | lo;
  if ((threadIdx.x & 31) == 0 && r) atomicOr(dst, (unsigned long long)r);
}

__device__ __forceinline__ void ms_commit(const MSState &s, uint32_t v, uint64_t reach) {
  uint64_t sv = s.seen[v];
  uint64_t nw = reach & ~sv;
  s.next[v] = nw;
  if (nw) {
    s.seen[v] = sv | nw;
    if (s.lvrow) write_levels(s, v, nw);
  }
}

// List appends with one atomic per CTA (a list counter is one address:
// per-item or per-warp atomics on it serialise).  Every thread of the CTA
// must call; returns the thread's slot.
__device__ __forceinline__ uint32_t cta_append(bool take, uint32_t *counter, uint32_t *sh) {
  const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const uint32_t m = __ballot_sync(0xFFFFFFFFu, take);
  if (lane == 0) sh[w] = __popc(m);
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t t = 0;
    for (uint32_t k = 0; k < (blockDim.x >> 5); k++) {
      const uint32_t c = sh[k];
      sh[k] = t;
      t += c;
    }
    sh[MT / 32] = t ? atomicAdd(counter, t) : 0u;
  }
  __syncthreads();
  const uint32_t pos = sh[MT / 32] + sh[w] + __popc(m & lanemask_lt());
  __syncthreads();
  return pos;
}

// pull, one thread per inline-only vertex: the 64-byte row as four 16-byte
// loads, then all of its (at most 16) neighbours' front masks in flight
__global__ void __launch_bounds__(MT) k_ms_pull_S(DevView G, const uint32_t *V, uint64_t nV,
                                                  MSState s) {
  const uint64_t vi = (uint64_t)blockIdx.x * MT + threadIdx.x;
  if (vi >= nV) return;
  const uint32_t v = V[vi];
  if ((s.seen[v] & s.live) == s.live) {
    s.next[v] = 0;
    return;
  }
  const uint32_t d = G.deg[v];
  const uint4 *row = reinterpret_cast<const uint4 *>(G.inl + (uint64_t)v * K_INLINE);
  uint32_t x[K_INLINE];
#pragma unroll
  for (uint32_t q = 0; q < K_INLINE / 4; q++) {
    const uint4 t = q * 4 < d ? __ldg(row + q) : make_uint4(0, 0, 0, 0);
    x[4 * q] = t.x;
    x[4 * q + 1] = t.y;
    x[4 * q + 2] = t.z;
    x[4 * q + 3] = t.w;
  }
  uint64_t reach = 0;
#pragma unroll
  for (uint32_t e = 0; e < K_INLINE; e++)
    if (e < d) reach |= s.front[x[e]];
  ms_commit(s, v, reach);
}

// pull, 8 lanes per vertex of 17..cut neighbours (inline row, then the PMA
// segment by rank), 8 ranks per lane per step with every load issued
// first, stopping once seen | reach covers every live source
__global__ void __launch_bounds__(MT) k_ms_pull_G8(DevView G, const uint32_t *V, uint64_t nV,
                                                   MSState s) {
  constexpr uint32_t U = 8;
  const uint64_t gt = (uint64_t)blockIdx.x * MT + threadIdx.x;
  const uint64_t vi = gt >> 3;
  const uint32_t q = gt & 7;
  const uint32_t lane = threadIdx.x & 31;
  const unsigned mask = 0xFFu << (lane & ~7u);
  if (vi >= nV) return;  // (whole groups: nV groups of 8 lanes)
  const uint32_t v = V[vi];
  const uint64_t sv = s.seen[v];
  if ((sv & s.live) == s.live) {
    if (q == 0) s.next[v] = 0;
    return;
  }
  const uint32_t d = G.deg[v];
  const uint32_t *row = G.inl + (uint64_t)v * K_INLINE;
  const uint32_t *seg = G.pma + G.pbeg[v] - K_INLINE;  // indexed by rank
  uint64_t reach = 0;
  for (uint32_t j0 = 0; j0 < d; j0 += 8 * U) {  // (group-uniform trip count)
    uint32_t x[U];
#pragma unroll
    for (uint32_t k = 0; k < U; k++) {
      const uint32_t j = j0 + q + 8 * k;
      x[k] = j < d ? (j < K_INLINE ? row[j] : __ldcs(seg + j)) : 0u;
    }
#pragma unroll
    for (uint32_t k = 0; k < U; k++)
      if (j0 + q + 8 * k < d) reach |= s.front[x[k]];
#pragma unroll
    for (int o = 4; o > 0; o >>= 1) {
      const uint32_t lo = __shfl_xor_sync(mask, (uint32_t)reach, o, 8);
      const uint32_t hi = __shfl_xor_sync(mask, (uint32_t)(reach >> 32), o, 8);
      reach |= ((uint64_t)hi << 32) | lo;
    }
    if (((reach | sv) & s.live) == s.live) break;  // (group-uniform)
  }
  if (q == 0) ms_commit(s, v, reach);
}

// pull, one warp per vertex, stopping once seen | reach covers every live
// source
__global__ void __launch_bounds__(MT) k_ms_pull_W(DevView G, const uint32_t *V, uint64_t nV,
                                                  MSState s) {
  uint64_t w = ((uint64_t)blockIdx.x * MT + threadIdx.x) >> 5;
  uint32_t lane = threadIdx.x & 31;
  if (w >= nV) return;
  uint32_t v = V[w];
  uint64_t sv = s.seen[v];
  if ((sv & s.live) == s.live) {
    if (lane == 0) s.next[v] = 0;
    return;
  }
  NbrList L = nbr_list(G, v);
  uint64_t reach = 0;
  for (uint32_t j0 = 0; j0 < L.deg; j0 += 32) {
    uint32_t j = j0 + lane;
    if (j < L.deg) reach |= s.front[L.at(j)];
    uint64_t r = reach;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) r = shfl_or64(r, o);
    reach = r;
    if (((reach | sv) & s.live) == s.live) break;
  }
  if (lane == 0) ms_commit(s, v, reach);
}

// push: every vertex of the active list ORs its front mask into its
// neighbours' accumulators, skipping neighbours that every source in the
// mask has already seen.  The first OR into an accumulator appends the
// neighbour to the touched list T.  Edge-balanced: the active lists are cut
// into list_piece()s (off = exclusive prefix of the piece counts) and every
// warp of the grid takes an equal share of them.  front is left as it is
// (cleared after the level).
// One piece (p, len) of a pushing vertex with source mask m.
__device__ __forceinline__ void ms_push_piece(const uint32_t *p, uint32_t len, uint64_t m,
                                              const uint64_t *seen, unsigned long long *acc,
                                              uint32_t *T, uint32_t *tcnt, uint32_t lane) {
  uint32_t x = 0;
  bool first = false;
  if (lane < len) {
    x = p[lane];
    if ((m & ~seen[x]) != 0) first = atomicOr(acc + x, (unsigned long long)m) == 0;
  }
  const uint32_t b = __ballot_sync(0xFFFFFFFFu, first);
  uint32_t base = 0;
  if (b) {
    if (lane == 0) base = atomicAdd(tcnt, __popc(b));
    base = __shfl_sync(0xFFFFFFFFu, base, 0);
  }
  if (first) T[base + __popc(b & lanemask_lt())] = x;
}

__global__ void __launch_bounds__(MT) k_ms_push(DevView G, const uint32_t *F, uint32_t nf,
                                                const uint64_t *off, const uint64_t *front,
                                                const uint64_t *seen, unsigned long long *acc,
                                                uint32_t *T, uint32_t *tcnt) {
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t W = ((uint64_t)gridDim.x * MT) >> 5;
  const uint64_t w = ((uint64_t)blockIdx.x * MT + threadIdx.x) >> 5;
  const uint64_t Tn = off[nf];
  const uint64_t lo = Tn * w / W, hi = Tn * (w + 1) / W;
  if (lo >= hi) return;
  // the vertex of piece lo: the i with off[i] <= lo < off[i+1]
  uint32_t a = 0, b = nf;
  while (b - a > 1) {
    const uint32_t mid = (a + b) >> 1;
    if (off[mid] <= lo) a = mid;
    else b = mid;
  }
  uint32_t i = a, u = F[i];
  uint64_t m = front[u];
  NbrList L = nbr_list(G, u);
  uint64_t vbeg = off[i], vend = off[i + 1];
  for (uint64_t t = lo; t < hi; t++) {
    while (t >= vend) {  // (t < off[nf], so i + 1 < nf here)
      i++;
      u = F[i];
      m = front[u];
      L = nbr_list(G, u);
      vbeg = vend;
      vend = off[i + 1];
    }
    const uint32_t *p;
    uint32_t len;
    list_piece(L, (uint32_t)(t - vbeg), p, len);
    if (len) ms_push_piece(p, len, m, seen, acc, T, tcnt, lane);  // (warp-uniform)
  }
}

// after a push: commit the touched accumulators into seen / next and append
// the vertices with new sources to the next active list (grid-stride over
// the device-side count of T)
__global__ void k_ms_commit_list(MSState s, const uint32_t *T, const uint32_t *tcnt,
                                 unsigned long long *acc, uint32_t *list, uint32_t *list_cnt,
                                 unsigned long long *any) {
  __shared__ uint32_t sh[MT / 32 + 2];
  const uint32_t nt = *tcnt;
  const uint64_t stride = (uint64_t)gridDim.x * MT;
  for (uint64_t base = (uint64_t)blockIdx.x * MT; base < nt; base += stride) {
    uint64_t i = base + threadIdx.x;
    uint64_t nw = 0;
    uint32_t v = 0;
    if (i < nt) {
      v = T[i];
      uint64_t a = acc[v];
      acc[v] = 0;
      uint64_t sv = s.seen[v];
      nw = a & ~sv;
      if (nw) {
        s.seen[v] = sv | nw;
        s.next[v] = nw;
        if (s.lvrow) write_levels(s, v, nw);
      }
    }
    const uint32_t pos = cta_append(nw != 0, list_cnt, sh);
    if (nw) list[pos] = v;
    warp_or_into(nw, any);
  }
}

// clears front[v] for the vertices of the old active list (after a pull
// level, so that the array is all-zero when it becomes `next`)
__global__ void k_ms_clear(uint64_t *front, const uint32_t *F, uint32_t nf) {
  uint64_t i = (uint64_t)blockIdx.x * MT + threadIdx.x;
  if (i < nf) front[F[i]] = 0;
}

// active list after a pull step; `any` (optional) collects the sources
// that discovered a vertex at this level
__global__ void k_ms_collect(uint32_t n, const uint64_t *front, uint32_t *list, uint32_t *cnt,
                             unsigned long long *any) {
  __shared__ uint32_t sh[MT / 32 + 2];
  uint64_t v = (uint64_t)blockIdx.x * MT + threadIdx.x;
  uint64_t f = v < n ? front[v] : 0;
  const uint32_t pos = cta_append(f != 0, cnt, sh);
  if (f) list[pos] = (uint32_t)v;
  if (any) warp_or_into(f, any);
}

// per source: vertices reached (popcount of each bit of seen over all
// vertices), one ballot per bit per 32 vertices
__global__ void k_ms_count(uint32_t n, const uint64_t *seen, unsigned long long *cnt) {
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t warps = (uint64_t)gridDim.x * (MT / 32);
  uint32_t c0 = 0, c1 = 0;
  for (uint64_t base = ((uint64_t)blockIdx.x * MT + threadIdx.x - lane); base < n;
       base += warps * 32) {
    uint64_t v = base + lane;
    uint64_t x = v < n ? seen[v] : 0;
#pragma unroll
    for (int i = 0; i < 32; i++) {
      uint32_t b = __popc(__ballot_sync(0xFFFFFFFFu, (x >> i) & 1));
      if (lane == i) c0 += b;
    }
#pragma unroll
    for (int i = 0; i < 32; i++) {
      uint32_t b = __popc(__ballot_sync(0xFFFFFFFFu, (x >> (32 + i)) & 1));
      if (lane == i) c1 += b;
    }
  }
  if (c0) atomicAdd(cnt + lane, (unsigned long long)c0);
  if (c1) atomicAdd(cnt + 32 + lane, (unsigned long long)c1);
}

// After the masks were zeroed and the levels filled with TRC_UNREACHED:
// source i's bit in its vertex's masks, and its level 0.
__global__ void k_ms_seed(uint32_t k, const uint32_t *src, unsigned long long *seen,
                          unsigned long long *front, uint32_t *lvrow) {
  const uint32_t i = threadIdx.x;
  if (i >= k) return;
  const uint32_t v = src[i];
  atomicOr(seen + v, 1ull << i);
  atomicOr(front + v, 1ull << i);
  if (lvrow) lvrow[(uint64_t)v * k + i] = 0u;
}

// levels (vertex-major n x k) -> out (source-major k x n), 32x32 tiles
__global__ void k_ms_transpose(const uint32_t *lvrow, uint32_t n, uint32_t k, uint32_t *out) {
  __shared__ uint32_t t[32][33];
  uint64_t v0 = (uint64_t)blockIdx.x * 32;
  uint32_t i0 = blockIdx.y * 32;
  for (uint32_t r = threadIdx.y; r < 32; r += blockDim.y) {
    uint64_t v = v0 + r;
    uint32_t i = i0 + threadIdx.x;
    if (v < n && i < k) t[r][threadIdx.x] = lvrow[v * k + i];
  }
  __syncthreads();
  for (uint32_t r = threadIdx.y; r < 32; r += blockDim.y) {
    uint32_t i = i0 + r;
    uint64_t v = v0 + threadIdx.x;
    if (v < n && i < k) out[(uint64_t)i * n + v] = t[threadIdx.x][r];
  }
}

// ---------------------------------------------------------------------------
// Multi-source BC (Brandes per source, as the reference's BC, include/BC.h:
// 99-157, for up to 64 sources at once).  The forward levels come from the
// multi-source BFS above; per level L+1 the vertices discovered (active list,
// new-source mask next[v]) get, for each new source s,
//   sigma[v][s] = sum of sigma[u][s] over neighbours u with s in front[u]
// (front = level-L masks).  Each level's (vertex, mask) pairs are kept in
// compact form; the backward pass walks them from the deepest level:
//   dep[v][s] = sum of dep[w][s] over neighbours w at level L+1 for s,
//               plus 1/sigma[v][s];
// and the result is (dep - 1/sigma) / (1/sigma) (NaN where s does not reach
// v), source-major.  sigma and dep are vertex-major (k doubles per vertex);
// lane l of a warp owns sources l and l + 32, neighbours are visited in
// sorted order, so every sum runs in the reference's order.

__device__ __forceinline__ uint64_t shfl64(uint64_t x, int src) {
  uint32_t lo = __shfl_sync(0xFFFFFFFFu, (uint32_t)x, src);
  uint32_t hi = __shfl_sync(0xFFFFFFFFu, (uint32_t)(x >> 32), src);
  return ((uint64_t)hi << 32) | lo;
}

// Sums val[u][s] over the neighbours u of v with s in (mask[u] & want), for
// lane l's sources l and l + 32 (warp-uniform v).
__device__ __forceinline__ void mbc_gather(const DevView &G, uint32_t v, uint64_t want,
                                           const uint64_t *mask, const double *val, uint32_t k,
                                           uint32_t lane, double &a0, double &a1) {
  NbrList L = nbr_list(G, v);
  for (uint32_t j0 = 0; j0 < L.deg; j0 += 32) {
    const uint32_t j = j0 + lane;
    const uint32_t u = j < L.deg ? L.at(j) : 0u;
    const uint64_t mu = j < L.deg ? (mask[u] & want) : 0ull;
    uint32_t ball = __ballot_sync(0xFFFFFFFFu, mu != 0);
    // up to MBC_BATCH contributing neighbours at a time: their rows loaded
    // first, then added in neighbour order (the sums stay in the same order)
    constexpr int MBC_BATCH = 4;
    while (ball) {
      double r0[MBC_BATCH], r1[MBC_BATCH];
#pragma unroll
      for (int t = 0; t < MBC_BATCH; t++) {
        r0[t] = 0.0;
        r1[t] = 0.0;
        if (ball) {  // (warp-uniform)
          const int b = __ffs(ball) - 1;
          ball &= ball - 1;
          const uint32_t uu = __shfl_sync(0xFFFFFFFFu, u, b);
          const uint64_t mm = shfl64(mu, b);
          const double *row = val + (uint64_t)uu * k;
          if (lane < k && ((mm >> lane) & 1)) r0[t] = row[lane];
          if (lane + 32 < k && ((mm >> (lane + 32)) & 1)) r1[t] = row[lane + 32];
        }
      }
#pragma unroll
      for (int t = 0; t < MBC_BATCH; t++) {
        a0 += r0[t];
        a1 += r1[t];
      }
    }
  }
}

// sigma of the vertices discovered this level (grid-stride over the device
// count of the active list)
__global__ void k_mbc_sigma(DevView G, const uint32_t *A, const uint32_t *cnt, const uint64_t *front,
                            const uint64_t *next, double *sigma, uint32_t k) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t na = *cnt;
  const uint64_t stride = ((uint64_t)gridDim.x * MT) >> 5;
  for (uint64_t w = ((uint64_t)blockIdx.x * MT + threadIdx.x) >> 5; w < na; w += stride) {
    const uint32_t v = A[w];
    const uint64_t nm = next[v];
    double a0 = 0.0, a1 = 0.0;
    mbc_gather(G, v, nm, front, sigma, k, lane, a0, a1);
    double *row = sigma + (uint64_t)v * k;
    if (lane < k && ((nm >> lane) & 1)) row[lane] = a0;
    if (lane + 32 < k && ((nm >> (lane + 32)) & 1)) row[lane + 32] = a1;
  }
}

// compact copy of a level: ord[i] = A[i], om[i] = mask[A[i]]
__global__ void k_mbc_store(const uint32_t *A, const uint32_t *cnt, const uint64_t *mask,
                            uint32_t *ord, uint64_t *om) {
  const uint32_t na = *cnt;
  const uint64_t stride = (uint64_t)gridDim.x * MT;
  for (uint64_t i = (uint64_t)blockIdx.x * MT + threadIdx.x; i < na; i += stride) {
    const uint32_t v = A[i];
    ord[i] = v;
    om[i] = mask[v];
  }
}

__global__ void k_mbc_scatter(const uint32_t *ord, const uint64_t *om, uint32_t cnt,
                              uint64_t *dense) {
  const uint64_t i = (uint64_t)blockIdx.x * MT + threadIdx.x;
  if (i < cnt) dense[ord[i]] = om[i];
}

__global__ void k_mbc_back(DevView G, const uint32_t *ord, const uint64_t *om, uint32_t cnt,
                           const uint64_t *fnext, const double *sigma, double *dep, uint32_t k) {
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t w = ((uint64_t)blockIdx.x * MT + threadIdx.x) >> 5;
  if (w >= cnt) return;
  const uint32_t v = ord[w];
  const uint64_t fm = om[w];
  double a0 = 0.0, a1 = 0.0;
  mbc_gather(G, v, fm, fnext, dep, k, lane, a0, a1);
  const double *sg = sigma + (uint64_t)v * k;
  double *row = dep + (uint64_t)v * k;
  if (lane < k && ((fm >> lane) & 1)) row[lane] = a0 + 1.0 / sg[lane];
  if (lane + 32 < k && ((fm >> (lane + 32)) & 1)) row[lane + 32] = a1 + 1.0 / sg[lane + 32];
}

__global__ void k_mbc_seed(const uint32_t *src, uint32_t k, double *sigma) {
  const uint32_t i = threadIdx.x;
  if (i < k) sigma[(uint64_t)src[i] * k + i] = 1.0;
}

// out[s * n + v] = (dep - 1/sigma) / (1/sigma), through 32 x 32 tiles
__global__ void k_mbc_final(const double *dep, const double *sigma, uint32_t n, uint32_t k,
                            double *out) {
  __shared__ double t[32][33];
  const uint64_t v0 = (uint64_t)blockIdx.x * 32;
  const uint32_t i0 = blockIdx.y * 32;
  for (uint32_t r = threadIdx.y; r < 32; r += blockDim.y) {
    const uint64_t v = v0 + r;
    const uint32_t i = i0 + threadIdx.x;
    if (v < n && i < k) {
      const double inv = 1.0 / sigma[v * k + i];
      t[r][threadIdx.x] = (dep[v * k + i] - inv) / inv;
    }
  }
  __syncthreads();
  for (uint32_t r = threadIdx.y; r < 32; r += blockDim.y) {
    const uint32_t i = i0 + r;
    const uint64_t v = v0 + threadIdx.x;
    if (v < n && i < k) out[(uint64_t)i * n + v] = t[threadIdx.x][r];
  }
}
}  // namespace

// Initial state of a multi-source traversal: every mask zero, every level
// TRC_UNREACHED (byte fills), then the sources' bits and levels.
void Graph::ms_init(uint32_t k, const uint32_t *dsrc, uint64_t *seen, uint64_t *front,
                    uint64_t *next, uint32_t *lvrow, unsigned long long *acc) {
  for (void *p : {(void *)seen, (void *)front, (void *)next, (void *)acc})
    TRC_CUDA(cudaMemsetAsync(p, 0, (uint64_t)n * 8, stream));
  if (lvrow) TRC_CUDA(cudaMemsetAsync(lvrow, 0xFF, (uint64_t)n * k * 4, stream));
  TRC_LAUNCH(prof, stream, "ms_init", 1, 64, 0, k_ms_seed, k, dsrc,
             (unsigned long long *)seen, (unsigned long long *)front, lvrow);
}

void Graph::ms_push_level(const uint32_t *F, uint32_t nf, const uint64_t *front,
                          const uint64_t *seen, unsigned long long *acc, uint32_t *T,
                          uint32_t *tcnt, PieceBufs &pb) {
  const uint64_t *off = piece_offsets(F, nf, pb, "ms_push_scan");
  const DevView G = view();
  TRC_LAUNCH(prof, stream, "ms_push", (unsigned)num_sms() * 8, MT, 0, k_ms_push, G, F, nf, off,
             front, seen, acc, T, tcnt);
}

void Graph::msbfs(const uint32_t *sources, uint32_t k, uint32_t *levels, uint32_t flags) {
  if (!levels) throw_error(TRC_ERR_INVALID, "null pointer");
  msbfs_run(sources, k, levels, flags, nullptr, nullptr);
}

void Graph::msbfs_summary(const uint32_t *sources, uint32_t k, uint64_t *reached, uint32_t *ecc) {
  if (!reached || !ecc) throw_error(TRC_ERR_INVALID, "null pointer");
  msbfs_run(sources, k, nullptr, 0, reached, ecc);
}

// levels != null: per-source levels; otherwise reached / ecc (host arrays
// of k) get the number of vertices each source reaches and its deepest level
void Graph::msbfs_run(const uint32_t *sources, uint32_t k, uint32_t *levels, uint32_t flags,
                      uint64_t *reached, uint32_t *ecc) {
  if (k == 0) return;
  if (k > 64) throw_error(TRC_ERR_INVALID, "at most 64 sources per multi-source BFS");
  if (!sources) throw_error(TRC_ERR_INVALID, "null pointer");
  const bool summary = levels == nullptr;
  std::vector<uint32_t> hsrc(k);
  if (flags & TRC_DEVICE_PTR) {
    TRC_CUDA(cudaMemcpyAsync(hsrc.data(), sources, k * 4, cudaMemcpyDeviceToHost, stream));
    sync();
  } else {
    std::copy(sources, sources + k, hsrc.begin());
  }
  for (uint32_t x : hsrc)
    if (x >= n) throw_error(TRC_ERR_INVALID, "source vertex out of range");
  ensure_lists();
  DBuf<uint64_t> seenb, fa, fb, accb;
  DBuf<uint32_t> lvb, outb, srcb, lst, cnt;
  for (auto *b : {&seenb, &fa, &fb, &accb}) b->bind(&budget);
  for (auto *b : {&lvb, &outb, &srcb, &lst, &cnt}) b->bind(&budget);
  uint64_t *seen = seenb.alloc_exact(n), *front = fa.alloc_exact(n), *next = fb.alloc_exact(n);
  unsigned long long *acc = (unsigned long long *)accb.alloc_exact(n);
  uint32_t *lvrow = summary ? nullptr : lvb.alloc_exact((uint64_t)n * k);
  uint32_t *dsrc = srcb.alloc_exact(k);
  DBuf<uint64_t> anyb;
  anyb.bind(&budget);
  // [0] sources that discovered a vertex this level (the next level's live
  // sources), [1..64] reach counts
  unsigned long long *any = (unsigned long long *)anyb.alloc_exact(65);
  std::vector<uint32_t> depth(k, 0);
  // active lists (double-buffered) and the touched list of push levels
  DBuf<uint32_t> lst2, tl;
  lst2.bind(&budget);
  tl.bind(&budget);
  uint32_t *L[2] = {lst.alloc_exact(n), lst2.alloc_exact(n)};
  uint32_t *T = tl.alloc_exact(n);
  uint32_t *c = cnt.alloc_exact(4);  // [1] next active, [2] touched, [3] pushing hubs
  PieceBufs pbufs(&budget);  // push levels: piece counts, prefix, scan scratch
  TRC_CUDA(cudaMemcpyAsync(dsrc, hsrc.data(), k * 4, cudaMemcpyHostToDevice, stream));
  ms_init(k, dsrc, seen, front, next, lvrow, acc);
  // initial active list = the distinct sources
  std::vector<uint32_t> act(hsrc);
  std::sort(act.begin(), act.end());
  act.erase(std::unique(act.begin(), act.end()), act.end());
  int cur = 0;
  TRC_CUDA(cudaMemcpyAsync(L[cur], act.data(), act.size() * 4, cudaMemcpyHostToDevice, stream));
  uint32_t nact = (uint32_t)act.size();
  uint64_t live = k == 64 ? ~0ull : ((1ull << k) - 1);
  const uint64_t dense_at = n / push_pull_divisor();
  const unsigned commit_grid = (unsigned)std::max(1, num_sms() * 8);
  DevView G = view();
  uint32_t level = 0;
  // invariants at the start of a level: front is non-zero exactly on
  // L[cur] (nact vertices), next and acc are all-zero
  while (nact > 0) {
    level++;
    TRC_CUDA(cudaMemsetAsync(c, 0, 16, stream));
    TRC_CUDA(cudaMemsetAsync(any, 0, 8, stream));
    MSState s{seen, front, next, lvrow, k, live, level};
    uint32_t *nl = L[cur ^ 1];
    if ((uint64_t)nact >= dense_at && dense_at > 0) {
      TRC_LAUNCH(prof, stream, "ms_pull_S", ceil_div(lists.nS, MT), MT, 0, k_ms_pull_S, G,
                 lists.S.get(), lists.nS, s);
      TRC_LAUNCH(prof, stream, "ms_pull_M8", ceil_div(lists.nM1 * 8, MT), MT, 0, k_ms_pull_G8, G,
                 lists.M1.get(), lists.nM1, s);
      TRC_LAUNCH(prof, stream, "ms_pull_M", ceil_div(lists.nM2 * 32, MT), MT, 0, k_ms_pull_W, G,
                 lists.M2.get(), lists.nM2, s);
      TRC_LAUNCH(prof, stream, "ms_pull_H", ceil_div(lists.nH * 32, MT), MT, 0, k_ms_pull_W, G,
                 lists.Hv.get(), lists.nH, s);
      // isolated vertices are in no class list; their next mask stays 0
      TRC_LAUNCH(prof, stream, "ms_collect", ceil_div(n, MT), MT, 0, k_ms_collect, n, next, nl,
                 c + 1, any);
      TRC_LAUNCH(prof, stream, "ms_clear", ceil_div(nact, MT), MT, 0, k_ms_clear, front, L[cur],
                 nact);
    } else {
      ms_push_level(L[cur], nact, front, seen, acc, T, c + 2, pbufs);
      TRC_LAUNCH(prof, stream, "ms_commit", commit_grid, MT, 0, k_ms_commit_list, s, T, c + 2,
                 acc, nl, c + 1, any);
      TRC_LAUNCH(prof, stream, "ms_clear", ceil_div(nact, MT), MT, 0, k_ms_clear, front, L[cur],
                 nact);
    }
    uint32_t hc[2];
    uint64_t hany = 0;
    TRC_CUDA(cudaMemcpyAsync(hc, c, 8, cudaMemcpyDeviceToHost, stream));
    TRC_CUDA(cudaMemcpyAsync(&hany, any, 8, cudaMemcpyDeviceToHost, stream));
    sync();
    nact = hc[1];
    live = hany;
    for (uint32_t i = 0; i < k; i++)
      if ((hany >> i) & 1) depth[i] = level;
    std::swap(front, next);
    cur ^= 1;
  }
  if (summary) {
    TRC_CUDA(cudaMemsetAsync(any + 1, 0, 64 * 8, stream));
    TRC_LAUNCH(prof, stream, "ms_count", (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(
                                             ceil_div(n, MT), (uint64_t)num_sms() * 8)),
               MT, 0, k_ms_count, n, seen, any + 1);
    uint64_t cnts[64];
    TRC_CUDA(cudaMemcpyAsync(cnts, any + 1, 64 * 8, cudaMemcpyDeviceToHost, stream));
    sync();
    for (uint32_t i = 0; i < k; i++) {
      reached[i] = cnts[i];
      ecc[i] = depth[i];
    }
    return;
  }
  bool dev = flags & TRC_DEVICE_PTR;
  uint32_t *out = dev ? levels : outb.alloc_exact((uint64_t)n * k);
  dim3 grid((unsigned)ceil_div(n, 32), (unsigned)ceil_div(k, 32));
  dim3 block(32, 8);
  k_ms_transpose<<<grid, block, 0, stream>>>(lvrow, n, k, out);
  prof.launches++;
  TRC_CUDA(cudaGetLastError());
  if (!dev) TRC_CUDA(cudaMemcpyAsync(levels, out, (uint64_t)n * k * 4, cudaMemcpyDeviceToHost, stream));
  sync();
}


// Compact per-level storage that grows by copying (device order preserved).
struct LevelStore {
  DBuf<uint32_t> ord[2];
  DBuf<uint64_t> om[2];
  int cur = 0;
  uint64_t cap = 0;
  void bind(Budget *b) {
    for (int i = 0; i < 2; i++) {
      ord[i].bind(b);
      om[i].bind(b);
    }
  }
  // room for `need` entries, keeping the first `used`
  void reserve(uint64_t need, uint64_t used, cudaStream_t s) {
    if (need <= cap) return;
    uint64_t nc = std::max<uint64_t>(need, cap * 2);
    int o = cur ^ 1;
    ord[o].alloc_exact(nc);
    om[o].alloc_exact(nc);
    if (used) {
      TRC_CUDA(cudaMemcpyAsync(ord[o].get(), ord[cur].get(), used * 4, cudaMemcpyDeviceToDevice, s));
      TRC_CUDA(cudaMemcpyAsync(om[o].get(), om[cur].get(), used * 8, cudaMemcpyDeviceToDevice, s));
    }
    ord[cur].reset();
    om[cur].reset();
    cur = o;
    cap = nc;
  }
  uint32_t *o32() { return ord[cur].get(); }
  uint64_t *o64() { return om[cur].get(); }
};

void Graph::msbc(const uint32_t *sources, uint32_t k, double *out_user, uint32_t flags) {
  if (k == 0) return;
  if (k > 64) throw_error(TRC_ERR_INVALID, "at most 64 sources per multi-source BC");
  if (!sources || !out_user) throw_error(TRC_ERR_INVALID, "null pointer");
  std::vector<uint32_t> hsrc(k);
  if (flags & TRC_DEVICE_PTR) {
    TRC_CUDA(cudaMemcpyAsync(hsrc.data(), sources, k * 4, cudaMemcpyDeviceToHost, stream));
    sync();
  } else {
    std::copy(sources, sources + k, hsrc.begin());
  }
  for (uint32_t x : hsrc)
    if (x >= n) throw_error(TRC_ERR_INVALID, "source vertex out of range");
  ensure_lists();
  DBuf<uint64_t> seenb, fa, fb, accb;
  DBuf<uint32_t> srcb, lst, lst2, tl, cnt;
  DBuf<double> sigb, depb, outb;
  for (auto *b : {&seenb, &fa, &fb, &accb}) b->bind(&budget);
  for (auto *b : {&srcb, &lst, &lst2, &tl, &cnt}) b->bind(&budget);
  for (auto *b : {&sigb, &depb, &outb}) b->bind(&budget);
  uint64_t *seen = seenb.alloc_exact(n), *front = fa.alloc_exact(n), *next = fb.alloc_exact(n);
  unsigned long long *acc = (unsigned long long *)accb.alloc_exact(n);
  double *sigma = sigb.alloc_exact((uint64_t)n * k), *dep = depb.alloc_exact((uint64_t)n * k);
  uint32_t *dsrc = srcb.alloc_exact(k);
  uint32_t *L[2] = {lst.alloc_exact(n), lst2.alloc_exact(n)};
  uint32_t *T = tl.alloc_exact(n);
  uint32_t *c = cnt.alloc_exact(4);  // [1] next active, [2] touched, [3] pushing hubs
  PieceBufs pbufs(&budget);  // push levels: piece counts, prefix, scan scratch
  DBuf<uint64_t> anyb;
  anyb.bind(&budget);
  unsigned long long *any = (unsigned long long *)anyb.alloc_exact(1);
  LevelStore lv;
  lv.bind(&budget);
  TRC_CUDA(cudaMemcpyAsync(dsrc, hsrc.data(), k * 4, cudaMemcpyHostToDevice, stream));
  TRC_CUDA(cudaMemsetAsync(sigma, 0, (uint64_t)n * k * 8, stream));
  TRC_CUDA(cudaMemsetAsync(dep, 0, (uint64_t)n * k * 8, stream));
  ms_init(k, dsrc, seen, front, next, nullptr, acc);
  TRC_LAUNCH(prof, stream, "mbc_seed", 1, 64, 0, k_mbc_seed, dsrc, k, sigma);
  std::vector<uint32_t> act(hsrc);
  std::sort(act.begin(), act.end());
  act.erase(std::unique(act.begin(), act.end()), act.end());
  int cur = 0;
  uint32_t nact = (uint32_t)act.size();
  TRC_CUDA(cudaMemcpyAsync(L[cur], act.data(), nact * 4, cudaMemcpyHostToDevice, stream));
  // level 0 in compact form
  std::vector<uint64_t> loff = {0};
  lv.reserve(std::max<uint64_t>(2 * (uint64_t)n, 1024), 0, stream);
  TRC_CUDA(cudaMemcpyAsync(c + 1, &nact, 4, cudaMemcpyHostToDevice, stream));
  TRC_LAUNCH(prof, stream, "mbc_store", ceil_div(nact, MT), MT, 0, k_mbc_store, L[cur], c + 1,
             front, lv.o32(), lv.o64());
  loff.push_back(nact);
  uint64_t live = k == 64 ? ~0ull : ((1ull << k) - 1);
  const uint64_t dense_at = n / push_pull_divisor();
  const unsigned pgrid = (unsigned)std::max(1, num_sms() * 8);
  DevView G = view();
  uint32_t level = 0;
  while (nact > 0) {
    level++;
    TRC_CUDA(cudaMemsetAsync(c, 0, 16, stream));
    TRC_CUDA(cudaMemsetAsync(any, 0, 8, stream));
    MSState s{seen, front, next, nullptr, k, live, level};
    uint32_t *nl = L[cur ^ 1];
    const uint64_t base = loff.back();
    lv.reserve(base + n, base, stream);
    if ((uint64_t)nact >= dense_at && dense_at > 0) {
      TRC_LAUNCH(prof, stream, "ms_pull_S", ceil_div(lists.nS, MT), MT, 0, k_ms_pull_S, G,
                 lists.S.get(), lists.nS, s);
      TRC_LAUNCH(prof, stream, "ms_pull_M8", ceil_div(lists.nM1 * 8, MT), MT, 0, k_ms_pull_G8, G,
                 lists.M1.get(), lists.nM1, s);
      TRC_LAUNCH(prof, stream, "ms_pull_M", ceil_div(lists.nM2 * 32, MT), MT, 0, k_ms_pull_W, G,
                 lists.M2.get(), lists.nM2, s);
      TRC_LAUNCH(prof, stream, "ms_pull_H", ceil_div(lists.nH * 32, MT), MT, 0, k_ms_pull_W, G,
                 lists.Hv.get(), lists.nH, s);
      TRC_LAUNCH(prof, stream, "ms_collect", ceil_div(n, MT), MT, 0, k_ms_collect, n, next, nl,
                 c + 1, any);
    } else {
      ms_push_level(L[cur], nact, front, seen, acc, T, c + 2, pbufs);
      TRC_LAUNCH(prof, stream, "ms_commit", pgrid, MT, 0, k_ms_commit_list, s, T, c + 2, acc, nl,
                 c + 1, any);
    }
    TRC_LAUNCH(prof, stream, "mbc_sigma", pgrid, MT, 0, k_mbc_sigma, G, nl, c + 1, front, next,
               sigma, k);
    TRC_LAUNCH(prof, stream, "mbc_store", pgrid, MT, 0, k_mbc_store, nl, c + 1, next,
               lv.o32() + base, lv.o64() + base);
    TRC_LAUNCH(prof, stream, "ms_clear", ceil_div(nact, MT), MT, 0, k_ms_clear, front, L[cur], nact);
    uint32_t hc[2];
    uint64_t hany = 0;
    TRC_CUDA(cudaMemcpyAsync(hc, c, 8, cudaMemcpyDeviceToHost, stream));
    TRC_CUDA(cudaMemcpyAsync(&hany, any, 8, cudaMemcpyDeviceToHost, stream));
    sync();
    nact = hc[1];
    live = hany;
    loff.push_back(base + nact);
    std::swap(front, next);
    cur ^= 1;
  }
  // levels 0..D with entries; loff has D + 2 offsets (the last level empty)
  const int64_t D = (int64_t)loff.size() - 3;
  // dense masks of level L+1 for the backward step (front is all-zero now)
  uint64_t *fnext = front;
  for (int64_t Lv = D; Lv >= 0; Lv--) {
    const uint64_t a = loff[Lv], b = loff[Lv + 1];
    const uint64_t a1 = loff[Lv + 1], b1 = loff[Lv + 2];
    if (b1 > a1)
      TRC_LAUNCH(prof, stream, "mbc_scatter", ceil_div(b1 - a1, MT), MT, 0, k_mbc_scatter,
                 lv.o32() + a1, lv.o64() + a1, (uint32_t)(b1 - a1), fnext);
    TRC_LAUNCH(prof, stream, "mbc_back", ceil_div((b - a) * 32, MT), MT, 0, k_mbc_back, G,
               lv.o32() + a, lv.o64() + a, (uint32_t)(b - a), fnext, sigma, dep, k);
    if (b1 > a1)
      TRC_LAUNCH(prof, stream, "mbc_clear", ceil_div(b1 - a1, MT), MT, 0, k_ms_clear, fnext,
                 lv.o32() + a1, (uint32_t)(b1 - a1));
  }
  bool dev = flags & TRC_DEVICE_PTR;
  double *out = dev ? out_user : outb.alloc_exact((uint64_t)n * k);
  dim3 grid((unsigned)ceil_div(n, 32), (unsigned)ceil_div(k, 32));
  dim3 block(32, 8);
  k_mbc_final<<<grid, block, 0, stream>>>(dep, sigma, n, k, out);
  prof.launches++;
  TRC_CUDA(cudaGetLastError());
  if (!dev)
    TRC_CUDA(cudaMemcpyAsync(out_user, out, (uint64_t)n * k * 8, cudaMemcpyDeviceToHost, stream));
  sync();
}

}  // namespace trc
