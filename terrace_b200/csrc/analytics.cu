// analytics.cu -- edgeMap-style traversals over the three tiers.
//
// Replaces the Ligra layer of the reference: edgeMap / vertexMap with the
// sparse (push) and dense (pull) directions (include/Map.cpp:7-108,
// include/graph.h:1287-1613) and the algorithms on top of it: BFS
// (include/BFS.h:27-84), PageRank PR_S (include/Pagerank.h:105-184), CC
// (include/Components.h:92-120), BC (include/BC.h:99-157) and TC
// (include/TC.h:33-87).
//
// Work is split by vertex class so that every lane does useful loads:
//   S  (1..16 neighbours, all in the 64-byte inline row): 4 lanes per
//      vertex, one 128-bit load each;
//   M  (more than 16, PMA segment): one warp per vertex, the 16 inline
//      neighbours then the contiguous segment in 128-byte chunks;
//   H  (hubs, blocked tier): one CTA per hub, warps over its blocks.
// Direction switching follows the reference rule: dense (pull) when the
// frontier holds at least n/divisor vertices (include/Map.cpp:65-74).
#include <algorithm>
#include <cstring>
#include <vector>

#include "graph.cuh"

namespace trc {

constexpr int AT = 256;  // threads per CTA in the analytics kernels

// ---------------------------------------------------------------------------
// Class lists

struct ClassPred {
  const uint32_t *deg;
  const int32_t *hub_of;
  int cls;  // 0 = S, 1 = M, 2 = H, 3 = S and M (non-hub, degree >= 1),
            // 4 = M with 17..cut neighbours, 5 = M with more than cut
  uint32_t cut;
  __device__ bool operator()(uint64_t i) const {
    bool hub = hub_of[i] >= 0;
    uint32_t d = deg[i];
    if (cls == 2) return hub;
    if (hub) return false;
    if (cls == 3) return d >= 1;
    if (cls == 4) return d > K_INLINE && d <= cut;
    if (cls == 5) return d > cut;
    return cls == 0 ? (d >= 1 && d <= K_INLINE) : d > K_INLINE;
  }
};

struct IdxVal32 {
  __device__ uint32_t operator()(uint64_t i) const { return (uint32_t)i; }
};

void Graph::ensure_lists() {
  if (lists.version == version) return;
  uint64_t *cnt = s_cnt.get() + 24;
  uint64_t *t = tmp(select_tmp_elems(n) + 4);
  uint32_t *bufs[6] = {lists.S.ensure(n), lists.M.ensure(n), lists.Hv.ensure(H ? H : 1),
                       lists.SM.ensure(n), lists.M1.ensure(n), lists.M2.ensure(n)};
  uint64_t lens[6];
  for (int c = 0; c < 6; c++) {
    select_if(ClassPred{deg.get(), hub_of.get(), c, tuned.pr_group_cut}, IdxVal32{}, n, bufs[c],
              cnt + c, t, stream,
              prof);
  }
  TRC_CUDA(cudaMemcpyAsync(lens, cnt, 48, cudaMemcpyDeviceToHost, stream));
  sync();
  lists.nS = lens[0];
  lists.nM = lens[1];
  lists.nH = lens[2];
  lists.nSM = lens[3];
  lists.nM1 = lens[4];
  lists.nM2 = lens[5];
  lists.version = version;
}

// ---------------------------------------------------------------------------
// Warp helpers

__device__ __forceinline__ uint32_t warp_append(bool win, uint32_t *counter) {
  uint32_t m = __ballot_sync(0xFFFFFFFFu, win);
  uint32_t base = 0;
  uint32_t lane = threadIdx.x & 31;
  if (m) {
    uint32_t leader = __ffs(m) - 1;
    if (lane == leader) base = atomicAdd(counter, __popc(m));
    base = __shfl_sync(0xFFFFFFFFu, base, leader);
  }
  return base + __popc(m & lanemask_lt());
}

// Per-warp staging of list appends from many chunks: the warp's winners of
// a chunk are written to `cap` shared slots (a multiple of 32) and go out
// with one atomic when the slots fill (and at the end, flush), instead of
// one atomic per chunk on the list's counter, which every warp of the grid
// hits.  Calls are warp-uniform.
constexpr uint32_t WS_BIG = 128;  // slots of the stages of the busiest lists
struct WarpStage {
  uint32_t *slot;  // `cap` shared words of this warp
  uint32_t cnt;
  uint32_t cap = 32;
  __device__ void flush(uint32_t *list, uint32_t *counter, uint32_t lane) {
    __syncwarp();
    if (cnt) {
      uint32_t base = 0;
      if (lane == 0) base = atomicAdd(counter, cnt);
      base = __shfl_sync(0xFFFFFFFFu, base, 0);
      for (uint32_t i = lane; i < cnt; i += 32) list[base + i] = slot[i];
    }
    __syncwarp();
    cnt = 0;
  }
  __device__ void add(bool win, uint32_t v, uint32_t *list, uint32_t *counter, uint32_t lane) {
    const uint32_t m = __ballot_sync(0xFFFFFFFFu, win);
    if (!m) return;
    const uint32_t k = __popc(m);
    if (cnt + k > cap) flush(list, counter, lane);
    if (win) slot[cnt + __popc(m & lanemask_lt())] = v;
    cnt += k;
    if (cnt == cap) flush(list, counter, lane);
  }
};

// Appends each thread's `cnt` items to a global list with ONE atomic per
// CTA (a per-level frontier counter is one address: a warp-level atomic per
// warp serialises there).  Every thread of the CTA must call it; returns the
// thread's first slot.  sh: AT/32 + 2 words of shared memory.
__device__ __forceinline__ uint32_t block_append(uint32_t cnt, uint32_t *counter, uint32_t *sh) {
  const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const uint32_t incl = warp_incl_scan(cnt);
  if (lane == 31) sh[w] = incl;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t t = 0;
    for (uint32_t k = 0; k < (blockDim.x >> 5); k++) {
      const uint32_t c = sh[k];
      sh[k] = t;
      t += c;
    }
    sh[AT / 32] = t ? atomicAdd(counter, t) : 0u;
  }
  __syncthreads();
  const uint32_t pos = sh[AT / 32] + sh[w] + incl - cnt;
  __syncthreads();
  return pos;
}

template <typename T>
__device__ __forceinline__ T block_sum(T v, T *sh) {
  v = warp_sum(v);
  int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) sh[w] = v;
  __syncthreads();
  T r = 0;
  if (w == 0) {
    r = lane < (int)(blockDim.x >> 5) ? sh[lane] : T(0);
    r = warp_sum(r);
  }
  __syncthreads();
  return r;  // valid in thread 0
}

// ---------------------------------------------------------------------------
// PageRank: per iteration p_next[u] = sum over N(u) of p[v]/deg(v)
// (PR_Vertex then the dense PR_F pull).  The kernels read pdiv = p/deg of
// the previous iteration and write both the new pdiv and, on the last
// iteration, the undivided value.

// Neighbour ids are read with streaming (evict-first) loads so the list
// stream does not push the gathered rank vector out of L2.
struct PRArgs {
  const double *pc;
  double *pn;
  double *out;
  double damping, base;
  int last;
};

__device__ __forceinline__ void pr_range(const PRArgs &, uint32_t, uint32_t d, uint32_t &lo,
                                         uint32_t &hi) {
  lo = 0;
  hi = d;
}

__device__ __forceinline__ void pr_store(const PRArgs &a, uint32_t u, uint32_t d, double sum) {
  double val = a.damping > 0.0 ? a.base + a.damping * sum : sum;
  a.pn[u] = val / (double)d;
  if (a.last) a.out[u] = val;
}

// One thread per vertex of at most 16 neighbours: the 64-byte row as four
// 16-byte loads, then all of its gathers in flight.
__global__ void __launch_bounds__(AT) k_pr_S(DevView G, const uint32_t *S, uint64_t nS, PRArgs a) {
  const uint64_t vi = (uint64_t)blockIdx.x * AT + threadIdx.x;
  if (vi >= nS) return;
  const uint32_t u = S[vi];
  const uint32_t d = G.deg[u];
  const uint4 *row = reinterpret_cast<const uint4 *>(G.inl + (uint64_t)u * K_INLINE);
  uint32_t x[K_INLINE];
#pragma unroll
  for (uint32_t q = 0; q < K_INLINE / 4; q++) {
    const uint4 t = q * 4 < d ? __ldcs(row + q) : make_uint4(0, 0, 0, 0);
    x[4 * q] = t.x;
    x[4 * q + 1] = t.y;
    x[4 * q + 2] = t.z;
    x[4 * q + 3] = t.w;
  }
  double g[K_INLINE];
#pragma unroll
  for (uint32_t e = 0; e < K_INLINE; e++) g[e] = e < d ? __ldg(a.pc + x[e]) : 0.0;
  double sum = 0.0;
#pragma unroll
  for (uint32_t e = 0; e < K_INLINE; e++) sum += g[e];
  pr_store(a, u, d, sum);
}

// Load-balanced pull.  Warp w takes list entries [32w, 32w+32); their
// neighbour lists (inline row, then PMA segment or hub blocks) are flattened
// and walked 64 elements per step: each lane finds the owner of its element
// with a shuffle binary search over the lanes' start offsets, loads the
// neighbour id and applies Op::gather; a segmented warp scan sums per owner
// and the segment's last lane adds into the owner's slot in shared memory.
// Every load of a step is independent of the others, so a warp keeps 64
// index loads and 64 gathers in flight instead of one vertex's chain.
struct FlatWarp {
  uint32_t u, d, start, total;
  int32_t hub;  // hub index, or -1
  const uint32_t *seg;
  bool valid;
};

template <class Op>
__device__ __forceinline__ FlatWarp flat_setup(const DevView &G, const uint32_t *V, uint64_t nV,
                                               uint64_t base, const Op &op) {
  FlatWarp f;
  uint32_t lane = threadIdx.x & 31;
  uint64_t idx = base + lane;
  f.valid = idx < nV;
  f.u = f.valid ? V[idx] : 0;
  f.d = 0;
  f.hub = -1;
  f.seg = G.pma;
  if (f.valid && !op.skip(f.u)) {
    f.d = G.deg[f.u];
    if (f.d > K_INLINE) {
      f.hub = G.hub_of[f.u];
      if (f.hub < 0) f.seg = G.pma + G.pbeg[f.u];
    }
  }
  uint32_t incl = warp_incl_scan(f.d);
  f.start = incl - f.d;
  f.total = __shfl_sync(0xFFFFFFFFu, incl, 31);
  return f;
}

// owner lane of flattened element e (largest lane v with start_v <= e)
__device__ __forceinline__ int flat_owner(const FlatWarp &f, uint32_t e) {
  int v = 0;
#pragma unroll
  for (int step = 16; step > 0; step >>= 1) {
    uint32_t sv = __shfl_sync(0xFFFFFFFFu, f.start, v + step);
    if (sv <= e) v += step;
  }
  return v;
}

// element of flattened index e (owner v): its rank r = e - start_v
__device__ __forceinline__ uint32_t flat_fetch(const DevView &G, const FlatWarp &f, int v,
                                               uint32_t e, bool act) {
  uint32_t uo = __shfl_sync(0xFFFFFFFFu, f.u, v);
  uint32_t so = __shfl_sync(0xFFFFFFFFu, f.start, v);
  int32_t ho = __shfl_sync(0xFFFFFFFFu, f.hub, v);
  uint32_t dh = __shfl_sync(0xFFFFFFFFu, f.d, v);
  const uint32_t *sg = (const uint32_t *)__shfl_sync(0xFFFFFFFFu, (unsigned long long)f.seg, v);
  if (!act) return 0;
  uint32_t r = e - so;
  if (r < K_INLINE) return __ldg(G.inl + (uint64_t)uo * K_INLINE + r);
  r -= K_INLINE;
  if (ho < 0) return __ldg(sg + r);
  // a hub: the directory entry of hub rank r
  const uint64_t e0 = G.hub_dir0[ho];
  const uint32_t i = hub_entry_of_rank(G.hpre + e0, G.hub_nblk[ho], dh - K_INLINE, r);
  return __ldg(G.hslot + (uint64_t)G.hdir[e0 + i] * HUB_BLOCK + (r - G.hpre[e0 + i]));
}

// segmented inclusive sum over lanes (segments = equal owner), tail lanes
// add the segment total into acc[owner]
__device__ __forceinline__ void flat_seg_add(double val, int v, double *acc) {
  uint32_t lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    double t = __shfl_up_sync(0xFFFFFFFFu, val, o);
    int vo = __shfl_up_sync(0xFFFFFFFFu, v, o);
    if ((int)lane >= o && vo == v) val += t;
  }
  int vn = __shfl_down_sync(0xFFFFFFFFu, v, 1);
  if (lane == 31 || vn != v) acc[v] += val;
}

template <class Op>
__global__ void __launch_bounds__(AT) k_flat(DevView G, const uint32_t *V, uint64_t nV, Op op) {
  __shared__ double acc_all[AT];
  const uint32_t lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const uint64_t base = ((uint64_t)blockIdx.x * (AT / 32) + wib) * 32;
  // warps past the end keep going with no entries: Op::store may be
  // CTA-collective
  double *acc = acc_all + wib * 32;
  FlatWarp f = flat_setup(G, V, nV, base, op);
  acc[lane] = 0.0;
  __syncwarp();
  for (uint32_t e0 = 0; e0 < f.total; e0 += 64) {
    uint32_t e1 = e0 + lane, e2 = e0 + 32 + lane;
    bool a1 = e1 < f.total, a2 = e2 < f.total;
    int v1 = flat_owner(f, a1 ? e1 : f.total - 1);
    int v2 = flat_owner(f, a2 ? e2 : f.total - 1);
    uint32_t x1 = flat_fetch(G, f, v1, e1, a1);
    uint32_t x2 = flat_fetch(G, f, v2, e2, a2);
    double g1 = a1 ? op.gather(x1) : 0.0;
    double g2 = a2 ? op.gather(x2) : 0.0;
    flat_seg_add(g1, v1, acc);
    __syncwarp();
    flat_seg_add(g2, v2, acc);
    __syncwarp();
  }
  op.store(f.valid, f.u, f.d, acc[lane]);  // (d == 0: nothing gathered, sum 0)
}

struct PROp {
  PRArgs a;
  __device__ bool skip(uint32_t) const { return false; }
  __device__ double gather(uint32_t x) const { return __ldg(a.pc + x); }
  __device__ void store(bool ok, uint32_t u, uint32_t d, double sum) const {
    if (ok) pr_store(a, u, d, sum);
  }
};

// Group pull for PMA vertices: GS lanes per vertex (8 for 17..64 neighbours,
// 32 above), each lane issuing up to 8 independent index loads and then 8
// gathers before using any of them; a shuffle reduction within the group.
template <int GS>
__global__ void __launch_bounds__(AT) k_pr_group(DevView G, const uint32_t *V, uint64_t nV, PRArgs a) {
  constexpr int U = 8;
  uint64_t gt = (uint64_t)blockIdx.x * AT + threadIdx.x;
  uint64_t vi = gt / GS;
  uint32_t q = gt % GS;
  double sum = 0.0;
  uint32_t u = 0, d = 0;
  if (vi < nV) {
    u = V[vi];
    d = G.deg[u];
    uint32_t lo, hi;
    pr_range(a, u, d, lo, hi);
    const uint32_t *row = G.inl + (uint64_t)u * K_INLINE;
    const uint32_t *seg = G.pma + G.pbeg[u] - K_INLINE;  // index by rank
    for (uint32_t j0 = lo + q; j0 < hi; j0 += GS * U) {
      uint32_t x[U];
#pragma unroll
      for (int k = 0; k < U; k++) {
        uint32_t j = j0 + k * GS;
        x[k] = j < hi ? (j < K_INLINE ? __ldcs(row + j) : __ldcs(seg + j)) : 0u;
      }
#pragma unroll
      for (int k = 0; k < U; k++) {
        uint32_t j = j0 + k * GS;
        if (j < hi) sum += __ldg(a.pc + x[k]);
      }
    }
  }
#pragma unroll
  for (int o = GS / 2; o > 0; o >>= 1) sum += __shfl_xor_sync(0xFFFFFFFFu, sum, o);
  if (vi < nV && q == 0) pr_store(a, u, d, sum);
}

__global__ void __launch_bounds__(AT) k_pr_H(DevView G, const uint32_t *Hv, PRArgs a) {
  __shared__ double sh[AT / 32];
  uint32_t u = Hv[blockIdx.x];
  int32_t h = G.hub_of[u];
  uint32_t d = G.deg[u];
  uint32_t ni = d < K_INLINE ? d : K_INLINE;
  double sum = 0.0;
  if (threadIdx.x < ni) sum = __ldg(a.pc + G.inl[(uint64_t)u * K_INLINE + threadIdx.x]);
  const uint64_t e0 = G.hub_dir0[h];
  const uint32_t nb = d > K_INLINE ? G.hub_nblk[h] : 0;
  uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (uint32_t b = warp; b < nb; b += AT / 32) {
    const uint32_t id = G.hdir[e0 + b];
    const uint32_t c = G.bcnt[id];
    const uint32_t *blk = G.hslot + (uint64_t)id * HUB_BLOCK;
    for (uint32_t s = lane; s < c; s += 32) sum += __ldg(a.pc + blk[s]);
  }
  sum = block_sum(sum, sh);
  if (threadIdx.x == 0) pr_store(a, u, d, sum);
}

__global__ void k_pr_init(const uint32_t *deg, uint32_t n, double p0, double iso, double *pdiv,
                          double *out) {
  uint64_t u = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= n) return;
  uint32_t d = deg[u];
  pdiv[u] = p0 / (double)d;
  if (d == 0) out[u] = iso;
}

void Graph::pagerank(uint32_t iters, double damping, double *ranks, uint32_t flags) {
  if (!ranks) throw_error(TRC_ERR_INVALID, "null output");
  if (damping < 0.0 || damping >= 1.0) throw_error(TRC_ERR_INVALID, "damping must be in [0,1)");
  ensure_lists();
  bool dev = flags & TRC_DEVICE_PTR;
  DBuf<double> pa, pb, ob;
  pa.bind(&budget);
  pb.bind(&budget);
  ob.bind(&budget);
  double *p0 = pa.alloc_exact(n), *p1 = pb.alloc_exact(n);
  double *out = dev ? ranks : ob.alloc_exact(n);
  if (iters == 0) {
    // the reference returns the initial vector 1/n (include/Pagerank.h:137-141)
    std::vector<double> h(n, 1.0 / (double)n);
    TRC_CUDA(cudaMemcpyAsync(out, h.data(), (uint64_t)n * 8, cudaMemcpyHostToDevice, stream));
    sync();
  } else {
    pagerank_launch(iters, damping, p0, p1, out, stream);
  }
  if (!dev) TRC_CUDA(cudaMemcpyAsync(ranks, out, (uint64_t)n * 8, cudaMemcpyDeviceToHost, stream));
  sync();
}

void Graph::pr_kernels(uint32_t iters, double damping, double *p0, double *p1, double *out,
                       cudaStream_t s) {
  const double one_over_n = 1.0 / (double)n;
  const double base = (1.0 - damping) / (double)n;
  TRC_LAUNCH(prof, s, "pr_init", ceil_div(n, AT), AT, 0, k_pr_init, deg.get(), n, one_over_n,
             damping > 0.0 ? base : 0.0, p0, out);
  DevView G = view();
  for (uint32_t it = 0; it < iters; it++) {
    PRArgs a{p0, p1, out, damping, base, it + 1 == iters};
    TRC_LAUNCH(prof, s, "pr_S", ceil_div(lists.nS, AT), AT, 0, k_pr_S, G, lists.S.get(),
               lists.nS, a);
    switch (tuned.pr_group_lanes) {
      case 4:
        TRC_LAUNCH(prof, s, "pr_M4", ceil_div(lists.nM1 * 4, AT), AT, 0, k_pr_group<4>, G,
                   lists.M1.get(), lists.nM1, a);
        break;
      case 16:
        TRC_LAUNCH(prof, s, "pr_M16", ceil_div(lists.nM1 * 16, AT), AT, 0, k_pr_group<16>, G,
                   lists.M1.get(), lists.nM1, a);
        break;
      default:
        TRC_LAUNCH(prof, s, "pr_M8", ceil_div(lists.nM1 * 8, AT), AT, 0, k_pr_group<8>, G,
                   lists.M1.get(), lists.nM1, a);
    }
    TRC_LAUNCH(prof, s, "pr_M32", ceil_div(lists.nM2 * 32, AT), AT, 0, k_pr_group<32>, G,
               lists.M2.get(), lists.nM2, a);
    TRC_LAUNCH(prof, s, "pr_H", lists.nH, AT, 0, k_pr_H, G, lists.Hv.get(), a);
    std::swap(p0, p1);
  }
}

// The iteration loop (iters x 4 launches) is replayed from a CUDA graph:
// captured once per (iteration count, buffers, class lists) and patched with
// cudaGraphExecUpdate when only kernel arguments changed.  With the
// per-kernel profiler on, kernels are launched directly so that each gets
// its own events.  Requires the class lists (ensure_lists) and iters >= 1;
// nothing is allocated or synchronised, so it may run on a second stream.
void Graph::pagerank_launch(uint32_t iters, double damping, double *p0, double *p1, double *out,
                            cudaStream_t s) {
  if (prof.on || !use_graphs || iters < 2) {
    pr_kernels(iters, damping, p0, p1, out, s);
    return;
  }
  uint64_t dbits;
  memcpy(&dbits, &damping, 8);
  const uint64_t key[PRGraphCache::KEY] = {iters, dbits, (uint64_t)p0, (uint64_t)p1, (uint64_t)out,
                                           lists.version, (uint64_t)lists.S.get(), lists.nS,
                                           lists.nM1, lists.nM2, lists.nH, (uint64_t)s,
                                           tuned.pr_group_lanes};
  bool same = prg.exec != nullptr;
  for (int i = 0; same && i < PRGraphCache::KEY; i++) same = prg.key[i] == key[i];
  if (!same) {
    const uint64_t before = prof.launches;
    cudaGraph_t gr = nullptr;
    TRC_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    try {
      pr_kernels(iters, damping, p0, p1, out, s);
    } catch (...) {
      cudaStreamEndCapture(s, &gr);
      if (gr) cudaGraphDestroy(gr);
      prof.launches = before;
      throw;
    }
    TRC_CUDA(cudaStreamEndCapture(s, &gr));
    prg.kernels = prof.launches - before;
    prof.launches = before;
    bool updated = false;
    if (prg.exec) {
      cudaGraphExecUpdateResultInfo info;
      updated = cudaGraphExecUpdate(prg.exec, gr, &info) == cudaSuccess;
      if (!updated) {
        cudaGetLastError();
        cudaGraphExecDestroy(prg.exec);
        prg.exec = nullptr;
      }
    }
    if (!updated) {
      cudaError_t e = cudaGraphInstantiate(&prg.exec, gr, 0);
      if (e != cudaSuccess) {
        cudaGraphDestroy(gr);
        prg.exec = nullptr;
        TRC_CUDA(e);
      }
    }
    cudaGraphDestroy(gr);
    memcpy(prg.key, key, sizeof(key));
    prg.replays_built++;
  }
  TRC_CUDA(cudaGraphLaunch(prg.exec, s));
  prof.launches += prg.kernels;
  prg.replays++;
}

// ---------------------------------------------------------------------------
// BFS (direction-optimising).  Levels are unique; parents follow the
// reference: push claims a vertex with CAS (any frontier parent, BFS_F::
// updateAtomic, include/BFS.h:34-36); pull takes the first frontier
// neighbour in sorted order (map_dense_vs_not_all breaks on cond,
// include/graph.h:1489-1613).

struct BFSState {
  uint32_t *lv;
  int32_t *par;
  const uint32_t *bits;  // frontier bitmap (pull)
  uint32_t *next;        // next-frontier queue
  uint32_t *next_cnt;
  uint32_t d;            // current level
  // dense steps: vertices left unvisited by the inline pass that have a
  // PMA segment (seg: at most BFS_SHORT neighbours, seg2: more), and
  // vertices left unvisited by the step (cand, the next dense step's
  // candidates)
  uint32_t *seg, *seg_cnt;
  uint32_t *cand, *cand_cnt;
  uint32_t *seg2, *seg2_cnt;
  // dense steps: the next level's frontier bitmap (zeroed before the step;
  // every vertex claimed by the step sets its bit), so that a dense step
  // after a dense step needs no pass over the levels
  uint32_t *nbits;
};

// Degree bound of the short segment list (8 lanes per vertex).
constexpr uint32_t BFS_SHORT = 64;

__device__ __forceinline__ bool bit_test(const uint32_t *b, uint32_t v) {
  return (__ldg(b + (v >> 5)) >> (v & 31)) & 1u;
}

// A piece (list_piece) of frontier vertex u's list: claim its unvisited
// neighbours by CAS on the parent (any frontier parent, as BFS_F::
// updateAtomic).
__device__ __forceinline__ void bfs_push_span(const uint32_t *p, uint32_t len, uint32_t u,
                                              const BFSState &s, uint32_t lane, WarpStage &st) {
  bool win = false;
  uint32_t v = 0;
  if (lane < len) {
    v = p[lane];
    // (every visited vertex has its parent set, and a parent is claimed
    // before the level is written: one load filters both the visited and
    // the just-claimed neighbours before a contended CAS)
    if (s.par[v] == -1 && atomicCAS(&s.par[v], -1, (int32_t)u) == -1) {
      s.lv[v] = s.d + 1;
      win = true;
    }
  }
  st.add(win, v, s.next, s.next_cnt, lane);
}

// Edge-balanced push (the frontier's lists cut into list_piece()s; off =
// exclusive prefix of the piece counts, off[nf] = the total T): warp w of W
// takes pieces [T*w/W, T*(w+1)/W), whatever vertices they belong to, so one
// long list is spread over many warps and many short lists share one warp.
// With skip_small, lists of at most K_INLINE elements outside the hub tier
// count no pieces (their vertices are pushed one thread each by
// k_bfs_push_small); off may then repeat values, and a piece's owner is the
// last vertex whose offset is at most the piece's index.
__device__ __forceinline__ uint32_t push_pieces(const DevView &G, uint32_t u, int skip_small) {
  const NbrList L = nbr_list(G, u);
  if (skip_small && L.deg <= K_INLINE && G.hub_of[u] < 0) return 0;
  return list_pieces(L);
}

__global__ void k_list_pieces(DevView G, const uint32_t *F, uint32_t nf, uint32_t *cnt,
                              int skip_small) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nf) cnt[i] = push_pieces(G, F[i], skip_small);
}

// The same and the exclusive prefix in one CTA, for frontiers of at most
// PIECES_ONE_CTA vertices: off[0..nf], off[nf] = the total.
constexpr uint32_t PIECES_ONE_CTA = 1024;
__global__ void __launch_bounds__(PIECES_ONE_CTA)
    k_list_pieces_scan(DevView G, const uint32_t *F, uint32_t nf, uint64_t *off, int skip_small) {
  __shared__ uint64_t ws[PIECES_ONE_CTA / 32 + 1];
  const uint32_t i = threadIdx.x;
  const uint64_t c = i < nf ? push_pieces(G, F[i], skip_small) : 0;
  uint64_t tot;
  const uint64_t ex = block_excl_scan<uint64_t, PIECES_ONE_CTA>(c, ws, tot);
  if (i < nf) off[i] = ex;
  if (i == 0) off[nf] = tot;
}

// The frontier vertex of piece t: the last i with off[i] <= t (vertices
// with no pieces share their successor's offset and are passed over).
__device__ __forceinline__ uint32_t piece_owner(const uint64_t *off, uint32_t nf, uint64_t t) {
  uint32_t a = 0, b = nf;
  while (b - a > 1) {
    const uint32_t m = (a + b) >> 1;
    if (off[m] <= t) a = m;
    else b = m;
  }
  return a;
}

// Push of the frontier's short lists (at most K_INLINE elements, outside the
// hub tier; the edge-balanced push skips them): one thread per frontier
// vertex, its row as four 16-byte loads and all of its parent probes in
// flight, then the claims.
__global__ void __launch_bounds__(AT) k_bfs_push_small(DevView G, const uint32_t *F, uint32_t nf,
                                                       BFSState s) {
  const uint32_t lane = threadIdx.x & 31;
  __shared__ uint32_t stg[AT / 32][WS_BIG];
  WarpStage st{stg[threadIdx.x >> 5], 0, WS_BIG};
  const uint64_t i = (uint64_t)blockIdx.x * AT + threadIdx.x;
  uint32_t u = 0, d = 0;
  if (i < nf) {
    u = F[i];
    d = G.deg[u];
    if (d > K_INLINE || G.hub_of[u] >= 0) d = 0;  // (an edge-balanced push's)
  }
  const uint4 *row = reinterpret_cast<const uint4 *>(G.inl + (uint64_t)u * K_INLINE);
  uint32_t x[K_INLINE];
#pragma unroll
  for (uint32_t q = 0; q < K_INLINE / 4; q++) {
    const uint4 t = q * 4 < d ? __ldcs(row + q) : make_uint4(0, 0, 0, 0);
    x[4 * q] = t.x;
    x[4 * q + 1] = t.y;
    x[4 * q + 2] = t.z;
    x[4 * q + 3] = t.w;
  }
  int32_t pv[K_INLINE];
#pragma unroll
  for (uint32_t e = 0; e < K_INLINE; e++) pv[e] = e < d ? s.par[x[e]] : 0;
#pragma unroll
  for (uint32_t e = 0; e < K_INLINE; e++) {
    bool win = false;
    if (e < d && pv[e] == -1 && atomicCAS(&s.par[x[e]], -1, (int32_t)u) == -1) {
      s.lv[x[e]] = s.d + 1;
      win = true;
    }
    st.add(win, x[e], s.next, s.next_cnt, lane);
  }
  st.flush(s.next, s.next_cnt, lane);
}

__global__ void __launch_bounds__(AT) k_bfs_push_lb(DevView G, const uint32_t *F, uint32_t nf,
                                                    const uint64_t *off, BFSState s) {
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t W = ((uint64_t)gridDim.x * AT) >> 5;
  const uint64_t w = ((uint64_t)blockIdx.x * AT + threadIdx.x) >> 5;
  const uint64_t T = off[nf];
  const uint64_t lo = T * w / W, hi = T * (w + 1) / W;
  __shared__ uint32_t stg[AT / 32][WS_BIG];
  WarpStage st{stg[threadIdx.x >> 5], 0, WS_BIG};
  if (lo < hi) {
    uint32_t i = piece_owner(off, nf, lo);
    uint32_t u = F[i];
    NbrList L = nbr_list(G, u);
    uint64_t vbeg = off[i], vend = off[i + 1];
    for (uint64_t t = lo; t < hi; t++) {
      while (t >= vend) {  // (t < T = off[nf], so i + 1 < nf here)
        i++;
        u = F[i];
        L = nbr_list(G, u);
        vbeg = vend;
        vend = off[i + 1];
      }
      const uint32_t *p;
      uint32_t len;
      list_piece(L, (uint32_t)(t - vbeg), p, len);
      if (len) bfs_push_span(p, len, u, s, lane, st);  // (warp-uniform)
    }
  }
  st.flush(s.next, s.next_cnt, lane);
}

// List entries that are still unvisited (and have more than min_deg
// neighbours).
struct UnvisitedPred {
  const uint32_t *L, *lv, *deg;
  uint32_t min_deg;
  __device__ bool operator()(uint64_t i) const {
    uint32_t u = L[i];
    return lv[u] == TRC_UNREACHED && deg[u] > min_deg;
  }
};

struct ListVal {
  const uint32_t *L;
  __device__ uint32_t operator()(uint64_t i) const { return L[i]; }
};

// frontier bitmap of level d from the levels: one ballot per 32 vertices
// (no atomics, no clearing pass); grid-stride, so the grid is what fits on
// the GPU rather than one tiny CTA per 256 vertices
__global__ void k_level_bits(const uint32_t *lv, uint32_t n, uint32_t d, uint32_t *bits) {
  constexpr uint32_t U = 4;  // level loads in flight per thread
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t W = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t v0 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v0 - lane < n; v0 += U * W) {
    uint32_t x[U];
#pragma unroll
    for (uint32_t j = 0; j < U; j++) x[j] = v0 + j * W < n ? lv[v0 + j * W] : TRC_UNREACHED;
#pragma unroll
    for (uint32_t j = 0; j < U; j++) {
      const uint64_t v = v0 + j * W;
      const uint32_t b = __ballot_sync(0xFFFFFFFFu, x[j] == d);
      if (lane == 0 && v < n) bits[v >> 5] = b;
    }
  }
}

// Inline pass of a dense step: one thread per vertex (grid-stride; a warp
// takes 32 consecutive list entries).  Each thread reads its vertex's
// 64-byte inline row in 16-byte streaming loads (evict-first, so the rows
// streaming through L2 do not push the frontier bitmap out; the warp's rows
// are one contiguous 2 KB block when the entries are consecutive ids), the
// first one and then the other three only on a miss, and its
// frontier-bitmap words (the first four, then the rest on a miss), every
// load of a round issued before any is used; the first frontier neighbour
// in sorted order is the parent.
// Vertices left unvisited go to the short or long segment list (PMA
// vertices) or to the next dense step's candidates.  S == null: the entries
// are the vertex ids 0 .. nS-1 themselves (hubs left to their own pass).
__global__ void __launch_bounds__(AT) k_bfs_pull_S(DevView G, const uint32_t *S, uint64_t nS,
                                                   BFSState s) {
  const uint32_t lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  __shared__ uint32_t stg[3][AT / 32][32], stn[AT / 32][WS_BIG];
  WarpStage sn{stn[wib], 0, WS_BIG}, ss{stg[0][wib], 0}, sc{stg[1][wib], 0}, sl{stg[2][wib], 0};
  const uint64_t step = (uint64_t)gridDim.x * AT;
  for (uint64_t base = (uint64_t)blockIdx.x * AT + (threadIdx.x & ~31u); base < nS; base += step) {
    const uint64_t vi = base + lane;
    bool act = vi < nS;
    const uint32_t u = act ? (S ? S[vi] : (uint32_t)vi) : 0u;
    uint32_t d = act ? G.deg[u] : 0u;
    if (!S && act && G.hub_of[u] >= 0) d = 0;
    act = act && d > 0 && s.lv[u] == TRC_UNREACHED;
    const uint4 *row = reinterpret_cast<const uint4 *>(G.inl + (uint64_t)u * K_INLINE);
    uint32_t x[K_INLINE];
    // the first four neighbours and their bitmap probes; the rest of the row
    // and the other twelve probes only for vertices with no frontier
    // neighbour among those four (on power-law graphs most have one there:
    // the second half of their row is never read)
    {
      const uint4 t = act ? __ldcs(row) : make_uint4(0, 0, 0, 0);
      x[0] = t.x;
      x[1] = t.y;
      x[2] = t.z;
      x[3] = t.w;
    }
    uint32_t wb[K_INLINE];
#pragma unroll
    for (uint32_t e = 0; e < 4; e++) wb[e] = act && e < d ? __ldg(s.bits + (x[e] >> 5)) : 0u;
    uint32_t p = NONE32;
#pragma unroll
    for (int e = 3; e >= 0; e--)
      if ((wb[e] >> (x[e] & 31)) & 1u) p = x[e];
    if (act && p == NONE32 && d > 4) {
#pragma unroll
      for (uint32_t q = 1; q < K_INLINE / 4; q++) {
        const uint4 t = q * 4 < d ? __ldcs(row + q) : make_uint4(0, 0, 0, 0);
        x[4 * q] = t.x;
        x[4 * q + 1] = t.y;
        x[4 * q + 2] = t.z;
        x[4 * q + 3] = t.w;
      }
#pragma unroll
      for (uint32_t e = 4; e < K_INLINE; e++) wb[e] = e < d ? __ldg(s.bits + (x[e] >> 5)) : 0u;
#pragma unroll
      for (int e = K_INLINE - 1; e >= 4; e--)
        if ((wb[e] >> (x[e] & 31)) & 1u) p = x[e];
    }
    const bool win = p != NONE32;
    if (win) {
      s.par[u] = (int32_t)p;
      s.lv[u] = s.d + 1;
    }
    if (S) {
      if (win) atomicOr(s.nbits + (u >> 5), 1u << (u & 31));
    } else {
      // (ids in order: the warp's 32 vertices are one bitmap word, and this
      // pass is the step's first writer)
      const uint32_t b = __ballot_sync(0xFFFFFFFFu, win);
      if (lane == 0) s.nbits[base >> 5] = b;
    }
    const bool left = act && !win;
    sn.add(win, u, s.next, s.next_cnt, lane);
    ss.add(left && d > K_INLINE && d <= BFS_SHORT, u, s.seg, s.seg_cnt, lane);
    sl.add(left && d > BFS_SHORT, u, s.seg2, s.seg2_cnt, lane);
    sc.add(left && d <= K_INLINE, u, s.cand, s.cand_cnt, lane);
  }
  sn.flush(s.next, s.next_cnt, lane);
  ss.flush(s.seg, s.seg_cnt, lane);
  sl.flush(s.seg2, s.seg2_cnt, lane);
  sc.flush(s.cand, s.cand_cnt, lane);
}

// One warp scans the neighbours of vertex u of rank >= j_first for a
// frontier member, 64 per step from the largest id down (two independent
// loads per lane), and returns the smallest frontier neighbour of the first
// step that has one, or NONE32 (warp-uniform).  Any frontier neighbour is a
// valid parent (the levels do not depend on the choice); scanning from the
// top finds one sooner on graphs whose high-degree vertices have large ids
// (RMAT with its d quadrant heaviest).
__device__ __forceinline__ uint32_t warp_any_in_frontier(const NbrList &L, const uint32_t *bits,
                                                         uint32_t j_first) {
  const uint32_t lane = threadIdx.x & 31;
  for (uint32_t e = L.deg; e > j_first;) {
    const uint32_t s0 = e - j_first > 64 ? e - 64 : j_first;
    const uint32_t ja = s0 + lane, jb = s0 + 32 + lane;
    const bool va = ja < e, vb = jb < e;
    const uint32_t xa = va ? L.at(ja) : 0u, xb = vb ? L.at(jb) : 0u;
    const bool ha = va && bit_test(bits, xa), hb = vb && bit_test(bits, xb);
    const uint32_t ma = __ballot_sync(0xFFFFFFFFu, ha), mb = __ballot_sync(0xFFFFFFFFu, hb);
    if (ma) return __shfl_sync(0xFFFFFFFFu, xa, __ffs(ma) - 1);
    if (mb) return __shfl_sync(0xFFFFFFFFu, xb, __ffs(mb) - 1);
    e = s0;
  }
  return NONE32;
}

// Warp per vertex of a list (M or H class), scanning ranks >= j_first (the
// inline pass has already checked ranks below it for M vertices).
// Per-warp staging of list appends: entries collect in 32 shared slots and
// go out 32 at a time with one atomic (no CTA-wide synchronisation, so the
// warps of a CTA never wait for each other's scans).
struct WarpBuf {
  uint32_t *slot;  // 32 shared words of this warp
  uint32_t cnt = 0;
  __device__ void push(bool has, uint32_t v, uint32_t *list, uint32_t *counter, uint32_t lane) {
    if (!has) return;  // warp-uniform
    if (lane == 0) slot[cnt] = v;
    if (++cnt == 32) flush(list, counter, lane);
  }
  __device__ void flush(uint32_t *list, uint32_t *counter, uint32_t lane) {
    __syncwarp();
    if (cnt) {
      uint32_t base = 0;
      if (lane == 0) base = atomicAdd(counter, cnt);
      base = __shfl_sync(0xFFFFFFFFu, base, 0);
      if (lane < cnt) list[base + lane] = slot[lane];
    }
    __syncwarp();
    cnt = 0;
  }
};

// Warp per list entry (nL_dev: count on the device, else nL), grid-stride;
// with `keep`, entries left unvisited join the candidates.
__global__ void __launch_bounds__(AT) k_bfs_pull_W(DevView G, const uint32_t *Lst, uint64_t nL,
                                                   const uint32_t *nL_dev, BFSState s,
                                                   uint32_t j_first, int keep) {
  const uint32_t lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const uint64_t n_l = nL_dev ? *nL_dev : nL;
  __shared__ uint32_t sw[AT / 32][32], sl[AT / 32][32];
  WarpBuf bw{sw[wib]}, bl{sl[wib]};
  const uint64_t stride = ((uint64_t)gridDim.x * AT) >> 5;
  for (uint64_t w = ((uint64_t)blockIdx.x * AT + threadIdx.x) >> 5; w < n_l; w += stride) {
    const uint32_t u = Lst[w];
    uint32_t p = NONE32;
    const bool unvisited = s.lv[u] == TRC_UNREACHED;
    if (unvisited) {
      NbrList L = nbr_list(G, u);
      p = warp_any_in_frontier(L, s.bits, j_first);
      if (p != NONE32 && lane == 0) {
        s.par[u] = (int32_t)p;
        s.lv[u] = s.d + 1;
        atomicOr(s.nbits + (u >> 5), 1u << (u & 31));
      }
    }
    bw.push(unvisited && p != NONE32, u, s.next, s.next_cnt, lane);
    if (keep) bl.push(unvisited && p == NONE32, u, s.cand, s.cand_cnt, lane);
  }
  bw.flush(s.next, s.next_cnt, lane);
  if (keep) bl.flush(s.cand, s.cand_cnt, lane);
}

// Segment pass for the short list (K_INLINE < degree <= BFS_SHORT, no
// hubs): 8 lanes per vertex, 4 vertices per warp step; lane q checks ranks
// 16 + q + 8t (t < 6), every segment load and then every bitmap load issued
// before any is used.  The lowest lane of the group with a frontier
// neighbour sets the parent; vertices without one join the candidates.
__global__ void __launch_bounds__(AT) k_bfs_pull_G8(DevView G, const uint32_t *Lst,
                                                    const uint32_t *nL_dev, BFSState s) {
  constexpr uint32_t R = (BFS_SHORT - K_INLINE) / 8;
  const uint32_t lane = threadIdx.x & 31, q = lane & 7, grp = lane >> 3, wib = threadIdx.x >> 5;
  __shared__ uint32_t stg[AT / 32][32], stn[AT / 32][WS_BIG];
  WarpStage sn{stn[wib], 0, WS_BIG}, sc{stg[wib], 0};
  const uint64_t nL = *nL_dev;
  const uint64_t step = (((uint64_t)gridDim.x * AT) >> 5) * 4;
  for (uint64_t base = (((uint64_t)blockIdx.x * AT + threadIdx.x) >> 5) * 4; base < nL;
       base += step) {
    const uint64_t vi = base + grp;
    const bool act = vi < nL;
    const uint32_t u = act ? Lst[vi] : 0u;
    const uint32_t d = act ? G.deg[u] : 0u;
    const uint32_t *seg = G.pma + (act ? G.pbeg[u] : 0) - K_INLINE;  // indexed by rank
    uint32_t x[R], w[R];
#pragma unroll
    for (uint32_t t = 0; t < R; t++) {
      const uint32_t j = K_INLINE + q + 8 * t;
      x[t] = j < d ? __ldcs(seg + j) : NONE32;
    }
#pragma unroll
    for (uint32_t t = 0; t < R; t++) w[t] = x[t] != NONE32 ? __ldg(s.bits + (x[t] >> 5)) : 0u;
    uint32_t p = NONE32;
#pragma unroll
    for (uint32_t t = 0; t < R; t++)
      if (p == NONE32 && x[t] != NONE32 && ((w[t] >> (x[t] & 31)) & 1u)) p = x[t];
    const uint32_t m = (__ballot_sync(0xFFFFFFFFu, p != NONE32) >> (grp * 8)) & 0xFFu;
    const bool win = m && (uint32_t)(__ffs(m) - 1) == q;
    if (win) {
      s.par[u] = (int32_t)p;
      s.lv[u] = s.d + 1;
      atomicOr(s.nbits + (u >> 5), 1u << (u & 31));
    }
    sn.add(win, u, s.next, s.next_cnt, lane);
    sc.add(act && q == 0 && m == 0, u, s.cand, s.cand_cnt, lane);
  }
  sn.flush(s.next, s.next_cnt, lane);
  sc.flush(s.cand, s.cand_cnt, lane);
}

// (16-byte stores, 4 vertices per thread and step, when both arrays are
// 16-byte aligned; caller arrays may not be)
__global__ void k_bfs_init(uint32_t *lv, int32_t *par, uint32_t n, int vec) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t n4 = vec ? n / 4 : 0;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += stride) {
    reinterpret_cast<uint4 *>(lv)[i] = make_uint4(TRC_UNREACHED, TRC_UNREACHED, TRC_UNREACHED,
                                                  TRC_UNREACHED);
    reinterpret_cast<int4 *>(par)[i] = make_int4(-1, -1, -1, -1);
  }
  for (uint64_t u = n4 * 4 + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; u < n; u += stride) {
    lv[u] = TRC_UNREACHED;
    par[u] = -1;
  }
}

__global__ void k_bfs_source(uint32_t *lv, int32_t *par, uint32_t src, uint32_t *q) {
  lv[src] = 0;
  par[src] = (int32_t)src;
  q[0] = src;
}

const uint64_t *Graph::piece_offsets(const uint32_t *F, uint32_t nf, PieceBufs &pb,
                                     const char *tag, bool skip_small) {
  uint64_t *off = pb.off.ensure((uint64_t)nf + 1);
  if (nf <= PIECES_ONE_CTA) {
    TRC_LAUNCH(prof, stream, "list_pieces", 1, PIECES_ONE_CTA, 0, k_list_pieces_scan, view(), F, nf,
               off, (int)skip_small);
    return off;
  }
  uint32_t *cnt = pb.cnt.ensure(nf);
  uint64_t *st = pb.scan.ensure(scan_tmp_elems(nf) + 4);
  TRC_LAUNCH(prof, stream, "list_pieces", ceil_div(nf, AT), AT, 0, k_list_pieces, view(), F, nf,
             cnt, (int)skip_small);
  exclusive_scan(LoadU32{cnt}, nf, off, st, stream, prof, tag);  // (off[nf] = the total)
  return off;
}

void Graph::bfs(uint32_t src, int32_t *parents, uint32_t *levels, uint32_t flags) {
  if (src >= n) throw_error(TRC_ERR_INVALID, "source vertex out of range");
  if (!parents) throw_error(TRC_ERR_INVALID, "null output");
  ensure_lists();
  bool dev = flags & TRC_DEVICE_PTR;
  DBuf<uint32_t> lvb, qa, qb, bits, bits2, cnt;
  DBuf<int32_t> parb;
  for (auto *b : {&lvb, &qa, &qb, &bits, &bits2, &cnt}) b->bind(&budget);
  parb.bind(&budget);
  uint32_t *lv = (dev && levels) ? levels : lvb.alloc_exact(n);
  int32_t *par = dev ? parents : parb.alloc_exact(n);
  uint32_t *F = qa.alloc_exact(n), *Nx = qb.alloc_exact(n);
  uint64_t words = ceil_div(n, 32);
  uint32_t *bm = bits.alloc_exact(words), *bm2 = bits2.alloc_exact(words);
  bool bm_valid = false;  // bm holds level d's frontier (a dense step wrote it)
  uint32_t *c = cnt.alloc_exact(4);
  TRC_LAUNCH(prof, stream, "bfs_init",
             std::min<uint64_t>(ceil_div(n, 4 * AT), resident_grid(k_bfs_init, AT)), AT, 0,
             k_bfs_init, lv, par, n, (int)((((uintptr_t)lv | (uintptr_t)par) & 15) == 0));
  TRC_LAUNCH(prof, stream, "bfs_source", 1, 1, 0, k_bfs_source, lv, par, src, F);
  DevView G = view();
  uint32_t nf = 1, d = 0;
  const uint64_t dense_at = n / push_pull_divisor();
  // candidates of the dense steps: non-hub vertices not yet visited,
  // compacted after every dense step
  DBuf<uint32_t> cbuf[2], segb, seg2b;  // candidate ping-pong, segment-pass lists
  PieceBufs pbufs(&budget);  // push steps: piece counts, prefix, scan scratch
  cbuf[0].bind(&budget);
  cbuf[1].bind(&budget);
  segb.bind(&budget);
  seg2b.bind(&budget);
  // (the first dense step reads every vertex id in order, no list: its
  // candidates are all non-hub vertices, and the loads stay contiguous)
  const uint32_t *cand = nullptr;
  uint64_t ncand = n;
  int cnext = 0;
  uint32_t *sg = segb.ensure(n), *sg2 = seg2b.ensure(n);
  const unsigned pgrid = (unsigned)num_sms() * 8;
  while (nf > 0) {
    TRC_CUDA(cudaMemsetAsync(c, 0, 16, stream));  // next, seg, cand counts
    BFSState s{lv, par, bm, Nx, c, d, sg, c + 1, nullptr, c + 2, sg2, c + 3, bm2};
    uint32_t hc[3] = {0, 0, 0};
    if ((uint64_t)nf >= dense_at && dense_at > 0) {
      if (!bm_valid)
        TRC_LAUNCH(prof, stream, "bfs_bits",
                   std::min<uint64_t>(ceil_div(n, AT), resident_grid(k_level_bits, AT)), AT, 0,
                   k_level_bits, lv, n, d, bm);
      TRC_CUDA(cudaMemsetAsync(bm2, 0, words * 4, stream));
      // candidates left for the next dense step (never the list being read)
      s.cand = cbuf[cnext].ensure(ncand ? ncand : 1);
      // pass A: the 16 inline neighbours of every unvisited non-hub vertex;
      // those left unvisited go to a segment list (PMA vertices: short or
      // long) or the next candidates
      TRC_LAUNCH(prof, stream, "bfs_pull_inline",
                 std::min<uint64_t>(ceil_div(ncand, (uint64_t)AT), resident_grid(k_bfs_pull_S, AT)),
                 AT, 0, k_bfs_pull_S, G, cand, ncand, s);
      // pass B: the PMA segments of the segment lists (counts on the
      // device; short lists 8 lanes per vertex, long ones a warp); hubs
      // from rank 0
      TRC_LAUNCH(prof, stream, "bfs_pull_M8", resident_grid(k_bfs_pull_G8, AT), AT, 0,
                 k_bfs_pull_G8, G, sg, c + 1, s);
      TRC_LAUNCH(prof, stream, "bfs_pull_M", pgrid, AT, 0, k_bfs_pull_W, G, sg2, 0, c + 3, s,
                 K_INLINE, 1);
      TRC_LAUNCH(prof, stream, "bfs_pull_H", ceil_div(lists.nH * 32, AT), AT, 0, k_bfs_pull_W, G,
                 lists.Hv.get(), lists.nH, (const uint32_t *)nullptr, s, 0u, 0);
      TRC_CUDA(cudaMemcpyAsync(hc, c, 12, cudaMemcpyDeviceToHost, stream));
      sync();
      ncand = hc[2];
      cand = s.cand;
      cnext ^= 1;
      std::swap(bm, bm2);  // the step's claims: level d+1's frontier
      bm_valid = true;
    } else {
      bm_valid = false;
      // edge-balanced push: piece counts scanned, then every warp of the
      // grid takes an equal share of the frontier's pieces
      const uint64_t *off = piece_offsets(F, nf, pbufs, "bfs_push_scan", true);
      TRC_LAUNCH(prof, stream, "bfs_push_small", ceil_div(nf, AT), AT, 0, k_bfs_push_small, G, F,
                 nf, s);
      TRC_LAUNCH(prof, stream, "bfs_push", pgrid, AT, 0, k_bfs_push_lb, G, F, nf, off, s);
      TRC_CUDA(cudaMemcpyAsync(hc, c, 4, cudaMemcpyDeviceToHost, stream));
      sync();
    }
    nf = hc[0];
    std::swap(F, Nx);
    d++;
  }
  if (!dev) {
    TRC_CUDA(cudaMemcpyAsync(parents, par, (uint64_t)n * 4, cudaMemcpyDeviceToHost, stream));
    if (levels) TRC_CUDA(cudaMemcpyAsync(levels, lv, (uint64_t)n * 4, cudaMemcpyDeviceToHost, stream));
  }
  sync();
}

// ---------------------------------------------------------------------------
// CC.  The reference propagates labels with writeMin until no label changes
// (include/Components.h:92-120); on a symmetric graph that fixed point is the
// smallest vertex id of each component.  The same fixed point is reached here
// with lock-free union-find (a root is always hooked under a smaller root, so
// the final root of a component is its smallest id) in the order of the
// published Afforest algorithm (Sutton, Ben-Nun, Barak, IPDPS 2018): link
// every vertex to its first two neighbours, compress, take the most frequent
// root of 1024 sampled vertices as the giant component, then link every
// edge of every vertex outside it; vertices inside it are skipped (an edge
// with an endpoint outside is linked from that endpoint, and an edge inside
// joins vertices already joined).  On power-law graphs the giant component
// holds almost every edge, so most of the adjacency is never read.

__device__ __forceinline__ uint32_t uf_find(uint32_t *p, uint32_t x) {
  uint32_t px = p[x];
  while (px != x) {
    uint32_t gp = p[px];
    if (gp != px) p[x] = gp;  // path halving (monotone: ids only decrease)
    x = px;
    px = p[x];
  }
  return x;
}

__device__ __forceinline__ void uf_unite(uint32_t *p, uint32_t a, uint32_t b) {
  while (true) {
    a = uf_find(p, a);
    b = uf_find(p, b);
    if (a == b) return;
    if (a < b) {
      uint32_t t = a;
      a = b;
      b = t;
    }
    if (atomicCAS(p + a, a, b) == a) return;
  }
}

constexpr uint32_t CC_SAMPLE_NB = 2;   // neighbours linked before the sample
constexpr uint32_t CC_SAMPLES = 1024;  // vertices sampled for the giant component

// thread per vertex: link to its r-th neighbour (inline: r < 16)
__global__ void k_cc_link(DevView G, uint32_t *p, uint32_t r) {
  const uint64_t u = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= G.n || G.deg[u] <= r) return;
  uf_unite(p, (uint32_t)u, G.inl[u * K_INLINE + r]);
}

// roots of pseudo-random vertices (hash of the sample index)
__global__ void k_cc_sample(const uint32_t *p, uint32_t n, uint32_t *out) {
  const uint32_t i = threadIdx.x + blockIdx.x * blockDim.x;
  if (i >= CC_SAMPLES) return;
  uint32_t h = i * 0x9E3779B1u;
  h ^= h >> 15;
  h *= 0x2C1B3C6Du;
  h ^= h >> 12;
  out[i] = p[h % n];
}

// the rest of the edges (rank >= CC_SAMPLE_NB) of vertices outside the giant
// component c: four lanes per vertex of at most 16 neighbours
__global__ void __launch_bounds__(AT) k_cc_S(DevView G, const uint32_t *S, uint64_t nS,
                                             uint32_t *p, uint32_t c) {
  uint64_t gt = (uint64_t)blockIdx.x * AT + threadIdx.x;
  uint64_t vi = gt >> 2;
  uint32_t q = gt & 3;
  if (vi >= nS) return;
  uint32_t u = S[vi];
  uint32_t d = G.deg[u];
  if (q * 4 >= d || d <= CC_SAMPLE_NB || uf_find(p, u) == c) return;
  uint4 v = reinterpret_cast<const uint4 *>(G.inl + (uint64_t)u * K_INLINE)[q];
  uint32_t e[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
  for (int i = 0; i < 4; i++)
    if (q * 4 + i < d && q * 4 + i >= CC_SAMPLE_NB) uf_unite(p, u, e[i]);
}

// ... and a warp per vertex of more: a warp takes 32 list entries, finds
// with one test per lane those outside the giant component, and walks their
// lists one after the other
__global__ void __launch_bounds__(AT) k_cc_W(DevView G, const uint32_t *Lst, uint64_t nL,
                                             uint32_t *p, uint32_t c) {
  const uint64_t i = (uint64_t)blockIdx.x * AT + threadIdx.x;  // 32 entries per warp
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t ul = i < nL ? Lst[i] : 0u;
  uint32_t todo = __ballot_sync(0xFFFFFFFFu, i < nL && uf_find(p, ul) != c);
  while (todo) {
    const uint32_t k = __ffs(todo) - 1;
    todo &= todo - 1;
    const uint32_t u = __shfl_sync(0xFFFFFFFFu, ul, k);
    NbrList L = nbr_list(G, u);
    for (uint32_t j = CC_SAMPLE_NB + lane; j < L.deg; j += 32) uf_unite(p, u, L.at(j));
  }
}

__global__ void k_cc_init(uint32_t *p, uint32_t n) {
  uint64_t u = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (u < n) p[u] = (uint32_t)u;
}

__global__ void k_cc_final(uint32_t *p, uint32_t n) {
  uint64_t u = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= n) return;
  uint32_t x = (uint32_t)u;
  while (p[x] != x) x = p[x];
  p[u] = x;
}

void Graph::cc(uint32_t *labels, uint32_t flags) {
  if (!labels) throw_error(TRC_ERR_INVALID, "null output");
  ensure_lists();
  bool dev = flags & TRC_DEVICE_PTR;
  DBuf<uint32_t> lb, sb;
  lb.bind(&budget);
  sb.bind(&budget);
  uint32_t *p = dev ? labels : lb.alloc_exact(n);
  uint32_t *smp = sb.alloc_exact(CC_SAMPLES);
  DevView G = view();
  TRC_LAUNCH(prof, stream, "cc_init", ceil_div(n, AT), AT, 0, k_cc_init, p, n);
  for (uint32_t r = 0; r < CC_SAMPLE_NB; r++)
    TRC_LAUNCH(prof, stream, "cc_link", ceil_div(n, AT), AT, 0, k_cc_link, G, p, r);
  TRC_LAUNCH(prof, stream, "cc_compress", ceil_div(n, AT), AT, 0, k_cc_final, p, n);
  // the giant component: the most frequent root among the samples
  uint32_t c = NONE32;
  if (n) {
    std::vector<uint32_t> h(CC_SAMPLES);
    TRC_LAUNCH(prof, stream, "cc_sample", ceil_div(CC_SAMPLES, AT), AT, 0, k_cc_sample, p, n, smp);
    TRC_CUDA(cudaMemcpyAsync(h.data(), smp, CC_SAMPLES * 4, cudaMemcpyDeviceToHost, stream));
    sync();
    std::sort(h.begin(), h.end());
    uint32_t best = 0;
    for (size_t i = 0; i < h.size();) {
      size_t j = i;
      while (j < h.size() && h[j] == h[i]) j++;
      if (j - i > best) {
        best = (uint32_t)(j - i);
        c = h[i];
      }
      i = j;
    }
  }
  TRC_LAUNCH(prof, stream, "cc_S", ceil_div(lists.nS * 4, AT), AT, 0, k_cc_S, G, lists.S.get(),
             lists.nS, p, c);
  TRC_LAUNCH(prof, stream, "cc_M", ceil_div(lists.nM, AT), AT, 0, k_cc_W, G, lists.M.get(),
             lists.nM, p, c);
  TRC_LAUNCH(prof, stream, "cc_H", ceil_div(lists.nH, AT), AT, 0, k_cc_W, G, lists.Hv.get(),
             lists.nH, p, c);
  TRC_LAUNCH(prof, stream, "cc_final", ceil_div(n, AT), AT, 0, k_cc_final, p, n);
  if (!dev) TRC_CUDA(cudaMemcpyAsync(labels, p, (uint64_t)n * 4, cudaMemcpyDeviceToHost, stream));
  sync();
}

// ---------------------------------------------------------------------------
// BC from one source (Brandes, as the reference's BC: forward path counts
// over BFS levels, backward dependency sums, final (Dep - 1/sigma)/(1/sigma)).

struct BCFwd {
  uint32_t *lv;
  double *sigma;
  double *sigma_out;    // pull steps write here (committed after the step)
  uint32_t *order;      // order[base ..] receives the next level
  uint32_t *next_cnt;
  uint32_t d;
};

// A piece (list_piece) of a frontier vertex u's list (sigma su): claim
// unvisited neighbours for level d+1 and add su to the path count of every
// neighbour on level d+1 (BC_F::updateAtomic's CAS-add, include/BC.h:44-58).
__device__ __forceinline__ void bc_push_span(const uint32_t *p, uint32_t len, double su,
                                             const BCFwd &s, uint32_t lane, WarpStage &st) {
  bool win = false;
  uint32_t v = 0;
  if (lane < len) {
    v = p[lane];
    uint32_t lvv = s.lv[v];
    if (lvv == TRC_UNREACHED) {
      uint32_t old = atomicCAS(&s.lv[v], TRC_UNREACHED, s.d + 1);
      win = old == TRC_UNREACHED;
      lvv = win ? s.d + 1 : old;
    }
    if (lvv == s.d + 1) atomicAdd(&s.sigma[v], su);
  }
  st.add(win, v, s.order, s.next_cnt, lane);
}

// Edge-balanced push of a BC level (as k_bfs_push_lb).
__global__ void __launch_bounds__(AT) k_bc_push_lb(DevView G, const uint32_t *F, uint32_t nf,
                                                   const uint64_t *off, BCFwd s) {
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t W = ((uint64_t)gridDim.x * AT) >> 5;
  const uint64_t w = ((uint64_t)blockIdx.x * AT + threadIdx.x) >> 5;
  const uint64_t T = off[nf];
  const uint64_t lo = T * w / W, hi = T * (w + 1) / W;
  __shared__ uint32_t stg[AT / 32][WS_BIG];
  WarpStage st{stg[threadIdx.x >> 5], 0, WS_BIG};
  if (lo < hi) {
    uint32_t i = piece_owner(off, nf, lo);
    uint32_t u = F[i];
    double su = s.sigma[u];
    NbrList L = nbr_list(G, u);
    uint64_t vbeg = off[i], vend = off[i + 1];
    for (uint64_t t = lo; t < hi; t++) {
      while (t >= vend) {
        i++;
        u = F[i];
        su = s.sigma[u];
        L = nbr_list(G, u);
        vbeg = vend;
        vend = off[i + 1];
      }
      const uint32_t *p;
      uint32_t len;
      list_piece(L, (uint32_t)(t - vbeg), p, len);
      if (len) bc_push_span(p, len, su, s, lane, st);
    }
  }
  st.flush(s.order, s.next_cnt, lane);
}

// Pull for an unvisited vertex: sigma = sum of sigma over neighbours on level d.
__global__ void __launch_bounds__(AT) k_bc_pull_W(DevView G, const uint32_t *Lst, uint64_t nL,
                                                  BCFwd s) {
  uint64_t w = ((uint64_t)blockIdx.x * AT + threadIdx.x) >> 5;
  uint32_t lane = threadIdx.x & 31;
  if (w >= nL) return;
  uint32_t u = Lst[w];
  bool win = false;
  if (s.lv[u] == TRC_UNREACHED) {
    NbrList L = nbr_list(G, u);
    double sum = 0.0;
    for (uint32_t j = lane; j < L.deg; j += 32) sum += __ldg(s.sigma + L.at(j));
    sum = warp_sum(sum);
    if (sum > 0.0 && lane == 0) {
      s.sigma_out[u] = sum;
      s.lv[u] = s.d + 1;
      win = true;
    }
  }
  uint32_t pos = warp_append(win, s.next_cnt);
  if (win) s.order[pos] = u;
}

__global__ void __launch_bounds__(AT) k_bc_pull_S(DevView G, const uint32_t *S, uint64_t nS,
                                                  BCFwd s) {
  uint64_t gt = (uint64_t)blockIdx.x * AT + threadIdx.x;
  uint64_t vi = gt >> 2;
  uint32_t q = gt & 3;
  double sum = 0.0;
  uint32_t u = 0;
  bool cand = false;
  if (vi < nS) {
    u = S[vi];
    uint32_t d = G.deg[u];
    cand = s.lv[u] == TRC_UNREACHED;
    if (cand && q * 4 < d) {
      uint4 v = reinterpret_cast<const uint4 *>(G.inl + (uint64_t)u * K_INLINE)[q];
      uint32_t e[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
      for (int i = 0; i < 4; i++)
        if (q * 4 + i < d && s.lv[e[i]] == s.d) sum += s.sigma[e[i]];
    }
  }
  sum += __shfl_xor_sync(0xFFFFFFFFu, sum, 1);
  sum += __shfl_xor_sync(0xFFFFFFFFu, sum, 2);
  bool win = cand && q == 0 && sum > 0.0;
  if (win) {
    s.sigma[u] = sum;
    s.lv[u] = s.d + 1;
  }
  uint32_t pos = warp_append(win, s.next_cnt);
  if (win) s.order[pos] = u;
}

// Dense forward step with the load-balanced pull: an unvisited vertex sums
// sigma over its neighbours on level d; a positive sum puts it on level d+1.
// Dense forward step (pull) for the unvisited vertices: sigma = sum of sigma
// over the neighbours on level d.  An unvisited vertex has no neighbour above
// level d (it would have been reached), and every neighbour not on level d
// is unvisited with sigma 0 (the step writes its results to sigma_out,
// committed after it), so the gather needs no level test.
struct BCPullOp {
  BCFwd s;
  __device__ bool skip(uint32_t u) const { return s.lv[u] != TRC_UNREACHED; }
  __device__ double gather(uint32_t x) const { return __ldg(s.sigma + x); }
  __device__ void store(bool ok, uint32_t u, uint32_t, double sum) const {
    bool win = ok && sum > 0.0;  // (a vertex with no neighbour on level d sums 0)
    if (win) {
      s.sigma_out[u] = sum;
      s.lv[u] = s.d + 1;
    }
    __shared__ uint32_t sh[AT / 32 + 2];
    uint32_t pos = block_append(win ? 1u : 0u, s.next_cnt, sh);  // every thread of the CTA
    if (win) s.order[pos] = u;
  }
};

// Backward step with the load-balanced pull over the vertices of level d:
// dep[v] = sum of dep[w] over neighbours on level d+1, plus 1/sigma[v].
// Neighbours of a level-d vertex are on levels d-1..d+1; dep holds only the
// finished levels above d (levels d-1 and d are still 0: this step writes
// to dep_out, committed after it), so the gather needs no level test.
struct BCBackOp {
  const double *inv;
  const double *dep;
  double *dep_out;
  __device__ bool skip(uint32_t) const { return false; }
  __device__ double gather(uint32_t x) const { return __ldg(dep + x); }
  __device__ void store(bool ok, uint32_t u, uint32_t, double sum) const {
    if (ok) dep_out[u] = sum + inv[u];  // every vertex of the level, isolated source included
  }
};

// Backward step over the degree classes instead of the level's list: the
// class lists are scanned whole and every vertex not on level L skipped (one
// lv load each), so each vertex of the level is summed by a lane group sized
// to its degree (four lanes below 17, a group of GS lanes up to the
// lane-group cut, a warp above, a CTA for a hub), every load of a step issued
// before any is used, as the PageRank pull does.
struct BCBackClassOp {
  const uint32_t *lv;
  uint32_t L;
  const double *inv;
  const double *dep;
  double *dep_out;
  __device__ bool skip(uint32_t u) const { return lv[u] != L; }
  __device__ double gather(uint32_t x) const { return __ldg(dep + x); }
  __device__ void store(uint32_t u, double sum) const { dep_out[u] = sum + inv[u]; }
};

// One thread per vertex of at most 16 neighbours: the 64-byte row as four
// 16-byte loads, then every gather in flight.
template <class Op>
__global__ void __launch_bounds__(AT) k_cls_S(DevView G, const uint32_t *S, uint64_t nS, Op op) {
  const uint64_t vi = (uint64_t)blockIdx.x * AT + threadIdx.x;
  if (vi >= nS) return;
  const uint32_t u = S[vi];
  if (op.skip(u)) return;
  const uint32_t d = G.deg[u];
  const uint4 *row = reinterpret_cast<const uint4 *>(G.inl + (uint64_t)u * K_INLINE);
  uint32_t x[K_INLINE];
#pragma unroll
  for (uint32_t q = 0; q < K_INLINE / 4; q++) {
    const uint4 t = q * 4 < d ? __ldcs(row + q) : make_uint4(0, 0, 0, 0);
    x[4 * q] = t.x;
    x[4 * q + 1] = t.y;
    x[4 * q + 2] = t.z;
    x[4 * q + 3] = t.w;
  }
  double g[K_INLINE];
#pragma unroll
  for (uint32_t e = 0; e < K_INLINE; e++) g[e] = e < d ? op.gather(x[e]) : 0.0;
  double sum = 0.0;
#pragma unroll
  for (uint32_t e = 0; e < K_INLINE; e++) sum += g[e];
  op.store(u, sum);
}

template <int GS, class Op>
__global__ void __launch_bounds__(AT) k_cls_group(DevView G, const uint32_t *V, uint64_t nV, Op op) {
  constexpr int U = 8;
  const uint64_t gt = (uint64_t)blockIdx.x * AT + threadIdx.x;
  const uint64_t vi = gt / GS;
  const uint32_t q = gt % GS;
  const uint32_t u = vi < nV ? V[vi] : 0u;
  const bool act = vi < nV && !op.skip(u);
  double sum = 0.0;
  if (act) {
    const uint32_t d = G.deg[u];
    const uint32_t *row = G.inl + (uint64_t)u * K_INLINE;
    const uint32_t *seg = G.pma + G.pbeg[u] - K_INLINE;  // index by rank
    for (uint32_t j0 = q; j0 < d; j0 += GS * U) {
      uint32_t x[U];
#pragma unroll
      for (int k = 0; k < U; k++) {
        const uint32_t j = j0 + k * GS;
        x[k] = j < d ? (j < K_INLINE ? __ldcs(row + j) : __ldcs(seg + j)) : 0u;
      }
#pragma unroll
      for (int k = 0; k < U; k++)
        if (j0 + k * GS < d) sum += op.gather(x[k]);
    }
  }
#pragma unroll
  for (int o = GS / 2; o > 0; o >>= 1) sum += __shfl_xor_sync(0xFFFFFFFFu, sum, o);
  if (act && q == 0) op.store(u, sum);
}

template <class Op>
__global__ void __launch_bounds__(AT) k_cls_H(DevView G, const uint32_t *Hv, Op op) {
  __shared__ double sh[AT / 32];
  const uint32_t u = Hv[blockIdx.x];
  if (op.skip(u)) return;  // CTA-uniform
  NbrList L = nbr_list(G, u);
  double sum = 0.0;
  if (threadIdx.x < L.ni) sum = op.gather(L.inl[threadIdx.x]);
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (uint32_t e = warp; e < L.nb; e += AT / 32) {
    const uint32_t *blk = L.seg + (uint64_t)L.dir[e] * HUB_BLOCK;
    const uint32_t c = (e + 1 < L.nb ? L.pre[e + 1] : L.rest) - L.pre[e];
    for (uint32_t k = lane; k < c; k += 32) sum += op.gather(blk[k]);
  }
  sum = block_sum(sum, sh);
  if (threadIdx.x == 0) op.store(u, sum);
}

// After a step that wrote to a side array: copy the values of the level's
// vertices (order[0 .. *cnt or cnt)) into the main array.
__global__ void k_bc_commit(const uint32_t *order, const uint32_t *cnt_dev, uint64_t cnt,
                            const double *from, double *to) {
  const uint64_t nv = cnt_dev ? *cnt_dev : cnt;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nv;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t v = order[i];
    to[v] = from[v];
  }
}

// Backward, one warp per vertex of level d:
// dep[v] = sum of dep[w] over neighbours on level d+1, plus 1/sigma[v].
__global__ void k_bc_back(DevView G, const uint32_t *Lv, uint32_t nv, const uint32_t *lv,
                          const double *inv, double *dep, uint32_t d) {
  uint64_t w = ((uint64_t)blockIdx.x * AT + threadIdx.x) >> 5;
  uint32_t lane = threadIdx.x & 31;
  if (w >= nv) return;
  uint32_t u = Lv[w];
  NbrList L = nbr_list(G, u);
  double sum = 0.0;
  for (uint32_t j = lane; j < L.deg; j += 32) {
    uint32_t v = L.at(j);
    if (lv[v] == d + 1) sum += dep[v];
  }
  sum = warp_sum(sum);
  if (lane == 0) dep[u] = sum + inv[u];
}

__global__ void k_bc_init(uint32_t *lv, double *sigma, double *dep, uint32_t n, uint32_t src,
                          uint32_t *order) {
  uint64_t u = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= n) return;
  lv[u] = u == src ? 0 : TRC_UNREACHED;
  sigma[u] = u == src ? 1.0 : 0.0;
  dep[u] = 0.0;
  if (u == src) order[0] = src;
}

__global__ void k_bc_inv(const double *sigma, double *inv, uint32_t n) {
  uint64_t u = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (u < n) inv[u] = 1.0 / sigma[u];
}

__global__ void k_bc_final(const double *dep, const double *inv, double *out, uint32_t n) {
  uint64_t u = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (u < n) out[u] = (dep[u] - inv[u]) / inv[u];
}

void Graph::bc(uint32_t src, double *out_user, uint32_t flags) {
  if (src >= n) throw_error(TRC_ERR_INVALID, "source vertex out of range");
  if (!out_user) throw_error(TRC_ERR_INVALID, "null output");
  ensure_lists();
  bool dev = flags & TRC_DEVICE_PTR;
  DBuf<uint32_t> lvb, ordb, cntb;
  DBuf<double> sig, invb, depb, outb, sideb;
  for (auto *b : {&lvb, &ordb, &cntb}) b->bind(&budget);
  for (auto *b : {&sig, &invb, &depb, &outb, &sideb}) b->bind(&budget);
  double *side = sideb.alloc_exact(n);  // a dense step's results before their commit
  uint32_t *lv = lvb.alloc_exact(n), *order = ordb.alloc_exact(n), *c = cntb.alloc_exact(4);
  PieceBufs pbufs(&budget);  // push steps: piece counts, prefix, scan scratch
  double *sigma = sig.alloc_exact(n), *inv = invb.alloc_exact(n), *dep = depb.alloc_exact(n);
  double *out = dev ? out_user : outb.alloc_exact(n);
  TRC_LAUNCH(prof, stream, "bc_init", ceil_div(n, AT), AT, 0, k_bc_init, lv, sigma, dep, n, src,
             order);
  DevView G = view();
  std::vector<uint64_t> loff = {0, 1};
  uint32_t d = 0;
  const uint64_t dense_at = n / push_pull_divisor();
  while (true) {
    uint64_t f0 = loff[d], f1 = loff[d + 1];
    uint32_t nf = (uint32_t)(f1 - f0);
    if (nf == 0) break;
    TRC_CUDA(cudaMemsetAsync(c, 0, 8, stream));
    BCFwd s{lv, sigma, side, order + f1, c, d};
    if ((uint64_t)nf >= dense_at && dense_at > 0) {
      TRC_LAUNCH(prof, stream, "bc_pull_flat", ceil_div(lists.nSM, AT), AT, 0, k_flat<BCPullOp>,
                 G, lists.SM.get(), lists.nSM, BCPullOp{s});
      TRC_LAUNCH(prof, stream, "bc_pull_H", ceil_div(lists.nH * 32, AT), AT, 0, k_bc_pull_W, G,
                 lists.Hv.get(), lists.nH, s);
      TRC_LAUNCH(prof, stream, "bc_commit", (unsigned)num_sms() * 4, AT, 0, k_bc_commit, order + f1,
                 c, 0, side, sigma);
    } else {
      const uint64_t *off = piece_offsets(order + f0, nf, pbufs, "bc_push_scan");
      TRC_LAUNCH(prof, stream, "bc_push", (unsigned)num_sms() * 8, AT, 0, k_bc_push_lb, G,
                 order + f0, nf, off, s);
    }
    uint32_t nn = 0;
    TRC_CUDA(cudaMemcpyAsync(&nn, c, 4, cudaMemcpyDeviceToHost, stream));
    sync();
    loff.push_back(f1 + nn);
    d++;
  }
  // d = number of non-empty levels; the last non-empty one is d-1
  TRC_LAUNCH(prof, stream, "bc_inv", ceil_div(n, AT), AT, 0, k_bc_inv, sigma, inv, n);
  for (int64_t L = (int64_t)d - 1; L >= 0; L--) {
    uint64_t a = loff[L], b = loff[L + 1];
    if (b - a < lists.nSM / 64) {  // a small level: its own list, load-balanced
      TRC_LAUNCH(prof, stream, "bc_back_flat", ceil_div(b - a, AT), AT, 0, k_flat<BCBackOp>, G,
                 order + a, b - a, BCBackOp{inv, dep, side});
    } else {  // a large one: the degree classes
      const BCBackClassOp op{lv, (uint32_t)L, inv, dep, side};
      TRC_LAUNCH(prof, stream, "bc_back_S", ceil_div(lists.nS, AT), AT, 0, k_cls_S<BCBackClassOp>,
                 G, lists.S.get(), lists.nS, op);
      TRC_LAUNCH(prof, stream, "bc_back_M8", ceil_div(lists.nM1 * 8, AT), AT, 0,
                 (k_cls_group<8, BCBackClassOp>), G, lists.M1.get(), lists.nM1, op);
      TRC_LAUNCH(prof, stream, "bc_back_M32", ceil_div(lists.nM2 * 32, AT), AT, 0,
                 (k_cls_group<32, BCBackClassOp>), G, lists.M2.get(), lists.nM2, op);
      TRC_LAUNCH(prof, stream, "bc_back_H", lists.nH, AT, 0, k_cls_H<BCBackClassOp>, G,
                 lists.Hv.get(), op);
    }
    TRC_LAUNCH(prof, stream, "bc_commit", std::min<uint64_t>(ceil_div(b - a, AT), num_sms() * 4), AT,
               0, k_bc_commit, order + a, (const uint32_t *)nullptr, b - a, side, dep);
  }
  TRC_LAUNCH(prof, stream, "bc_final", ceil_div(n, AT), AT, 0, k_bc_final, dep, inv, out, n);
  if (!dev) TRC_CUDA(cudaMemcpyAsync(out_user, out, (uint64_t)n * 8, cudaMemcpyDeviceToHost, stream));
  sync();
}

// ---------------------------------------------------------------------------
// TC.  Every triangle is counted once as w in N+(u) n N+(v) for an oriented
// edge u->v, where N+(x) keeps the neighbours ranked above x by (degree, id).
// The reference counts w < min(s,d) over edges s > d (id order, include/TC.h:
// 51-87); both orders count each triangle exactly once, and the degree order
// bounds the intersection work on skewed graphs.  N+ is materialised once as
// an oriented CSR snapshot, then one warp per vertex intersects sorted lists
// (k_tc_intersect).

__device__ __forceinline__ bool ranked_above(const uint32_t *deg, uint32_t x, uint32_t du,
                                             uint32_t u) {
  uint32_t dx = deg[x];
  return dx > du || (dx == du && x > u);
}

__global__ void k_tc_count_out(DevView G, uint32_t *outdeg) {
  uint64_t w = ((uint64_t)blockIdx.x * AT + threadIdx.x) >> 5;
  uint32_t lane = threadIdx.x & 31;
  if (w >= G.n) return;
  uint32_t u = (uint32_t)w;
  NbrList L = nbr_list(G, u);
  uint32_t c = 0;
  for (uint32_t j = lane; j < L.deg; j += 32) c += ranked_above(G.deg, L.at(j), L.deg, u);
  c = warp_sum(c);
  if (lane == 0) outdeg[u] = c;
}


__global__ void k_tc_fill(DevView G, const uint64_t *off, uint32_t *adj) {
  uint64_t w = ((uint64_t)blockIdx.x * AT + threadIdx.x) >> 5;
  uint32_t lane = threadIdx.x & 31;
  if (w >= G.n) return;
  uint32_t u = (uint32_t)w;
  NbrList L = nbr_list(G, u);
  uint64_t o = off[u];
  for (uint32_t j0 = 0; j0 < L.deg; j0 += 32) {
    uint32_t j = j0 + lane;
    uint32_t v = j < L.deg ? L.at(j) : 0;
    bool keep = j < L.deg && ranked_above(G.deg, v, L.deg, u);
    uint32_t m = __ballot_sync(0xFFFFFFFFu, keep);
    if (keep) adj[o + __popc(m & lanemask_lt())] = v;
    o += __popc(m);
  }
}

// Is x in the sorted list p[0..len)?
__device__ __forceinline__ bool sorted_has(const uint32_t *p, uint32_t len, uint32_t x) {
  uint32_t lo = 0, hi = len;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (p[mid] < x) lo = mid + 1;
    else hi = mid;
  }
  return lo < len && p[lo] == x;
}

// One warp per vertex u.  N+(u) is staged in the warp's shared slice when
// it fits (TC_STAGE ids); the lanes first load the list offsets of 32 of
// u's out-neighbours v at once, then for each v the lanes walk the shorter
// of N+(u) and N+(v) and look each element up in the other: in the staged
// N+(u) by a shared-memory search, in N+(v) by a global binary search.
constexpr uint32_t TC_STAGE = 256;

__global__ void __launch_bounds__(AT) k_tc_intersect(uint32_t n, const uint64_t *off,
                                                     const uint32_t *adj,
                                                     unsigned long long *total) {
  __shared__ uint32_t stage[AT / 32][TC_STAGE];
  const uint32_t lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  uint32_t *As = stage[wib];
  unsigned long long c = 0;
  const uint64_t w = ((uint64_t)blockIdx.x * AT + threadIdx.x) >> 5;
  if (w >= n) return;
  {
    const uint32_t u = (uint32_t)w;
    const uint64_t a0 = off[u];
    const uint32_t na = (uint32_t)(off[u + 1] - a0);
    if (na < 2) return;  // (warp-uniform)
    const uint32_t *A = adj + a0;
    const bool staged = na <= TC_STAGE;
    if (staged) {
      for (uint32_t t = lane; t < na; t += 32) As[t] = A[t];
      __syncwarp();
    }
    const uint32_t *Al = staged ? As : A;
    for (uint32_t i0 = 0; i0 < na; i0 += 32) {
      const uint32_t iv = i0 + lane;
      uint64_t b = 0;
      uint32_t nb = 0;
      if (iv < na) {
        const uint32_t v = A[iv];
        b = off[v];
        nb = (uint32_t)(off[v + 1] - b);
      }
      const uint32_t cnt = na - i0 < 32 ? na - i0 : 32;
      for (uint32_t j = 0; j < cnt; j++) {
        const uint64_t bj = __shfl_sync(0xFFFFFFFFu, b, j);
        const uint32_t nbj = __shfl_sync(0xFFFFFFFFu, nb, j);
        const uint32_t *B = adj + bj;
        if (nbj <= na) {
          for (uint32_t t = lane; t < nbj; t += 32) c += sorted_has(Al, na, B[t]);
        } else {
          for (uint32_t t = lane; t < na; t += 32) c += sorted_has(B, nbj, Al[t]);
        }
      }
    }
  }
  c = warp_sum(c);
  if (lane == 0 && c) atomicAdd(total, c);
}

uint64_t Graph::tc() {
  DBuf<uint32_t> od, adjb;
  DBuf<uint64_t> offb, tot;
  od.bind(&budget);
  adjb.bind(&budget);
  offb.bind(&budget);
  tot.bind(&budget);
  uint32_t *outdeg = od.alloc_exact(n);
  uint64_t *off = offb.alloc_exact((uint64_t)n + 1);
  uint64_t *total = tot.alloc_exact(1);
  DevView G = view();
  TRC_LAUNCH(prof, stream, "tc_count", ceil_div((uint64_t)n * 32, AT), AT, 0, k_tc_count_out, G,
             outdeg);
  uint64_t *t = tmp(scan_tmp_elems(n) + 4);
  exclusive_scan(LoadU32{outdeg}, n, off, t, stream, prof);
  uint64_t mo = read_u64(off + n);
  uint32_t *adj = adjb.alloc_exact(mo ? mo : 1);
  TRC_LAUNCH(prof, stream, "tc_fill", ceil_div((uint64_t)n * 32, AT), AT, 0, k_tc_fill, G, off, adj);
  TRC_CUDA(cudaMemsetAsync(total, 0, 8, stream));
  TRC_LAUNCH(prof, stream, "tc_intersect", ceil_div((uint64_t)n * 32, AT), AT, 0, k_tc_intersect,
             n, off, adj, (unsigned long long *)total);
  return read_u64(total);
}

}  // namespace trc
