// update.cu -- the graph's HBM state and the batch update pipeline.
//
// Replaces Graph::add_edge_batch (include/graph.h:430-502, with add_inplace
// :251-372, add_btree :375-426 and the per-edge PMA inserts of
// src/PMA.cc:2050-2108, :1253-1513) and the per-edge remove loop
// (include/graph.h:675-791, src/PMA.cc:2800-2873).  Instead of per-edge
// inserts under spin locks, a whole batch goes through one device pipeline:
//
//   1  keys (src<<32|dst), symmetrized on request; ids validated
//   2  LSD radix sort + adjacent unique
//   3  existence filter against the tiers (insert keeps new edges, remove
//      keeps present ones) -> the batch B, sorted
//   4  touched vertices (runs of B by source), new degree and tier of each:
//      deg <= 16 inline only, > hub_threshold (or already a hub) blocked
//      tier, otherwise inline + PMA segment
//   5  PMA planning: a vertex whose new segment does not fit its slots
//      triggers the packed-memory-array rule -- climb the implicit tree of
//      aligned vertex ranges until a window's density is within the bound of
//      its level (1.0 at a single vertex down to pma_root_density at the
//      root), rebalance the maximal such windows, or rebuild the whole PMA
//      at pma_build_density when the root overflows (the reference's
//      density bounds, src/PMA.cc:382-394, redistribute :419-655,
//      double_list :659-720)
//   6  rewrite set R = touched vertices + vertices of rebalanced windows
//      (+ every PMA vertex on a rebuild); their old lists are gathered as
//      sorted 64-bit keys, merged with B (insert) or stripped of B (remove)
//      by merge path, and scattered back: first 16 to the inline row, the
//      rest to the PMA segment at its (possibly new) offset or to the hub's
//      blocks (uniformly filled, hub_block_fill).
//
// Set semantics throughout: the reference's duplicate leak (include/graph.h:
// 269-289) and absent-edge remove (include/graph.h:695-716) do not occur.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>

#include "graph.cuh"

namespace trc {

// ---------------------------------------------------------------------------
// Lifetime

Graph::Graph(uint32_t n_, uint64_t budget_bytes, const trc_config &cfg_) : n(n_), cfg(cfg_) {
  budget.limit = budget_bytes;
  TRC_CUDA(cudaGetDevice(&device));
  na_scratch = noalloc_scratch_resolve();
  TRC_CUDA(cudaStreamCreateWithFlags(&own_stream, cudaStreamNonBlocking));
  TRC_CUDA(cudaStreamCreateWithFlags(&side_stream, cudaStreamNonBlocking));
  TRC_CUDA(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
  TRC_CUDA(cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming));
  TRC_CUDA(cudaEventCreateWithFlags(&ev_hub, cudaEventDisableTiming));
  TRC_CUDA(cudaStreamCreateWithFlags(&copy_stream, cudaStreamNonBlocking));
  TRC_CUDA(cudaEventCreateWithFlags(&ev_h2d, cudaEventDisableTiming));
  stream = own_stream;
  budget.stream = stream;
  budget.open_pool(device);
  use_graphs = cfg.cuda_graphs != 0;
  if (cfg.push_pull_divisor) tuned.push_pull_divisor = cfg.push_pull_divisor;
  for (auto *b : {&deg, &inl, &c2, &pma, &err, &hub_vtx, &hub_nblk, &hdir, &hpre, &hkey, &hslot,
                  &bcnt, &bmin, &bown, &bfree, &bfreed, &stamp, &s_in_src, &s_in_dst, &s_tu, &s_tdn,
                  &s_tc2, &s_ovl, &s_hw_u, &s_hw_dn, &s_hw_t, &s_c2n, &s_rlist, &s_pma_next,

                  &lists.S, &lists.M, &lists.Hv, &lists.SM, &lists.M1, &lists.M2,
                  &s_lg, &s_lx, &s_lli, &s_tgq, &s_tgo, &s_tgb, &s_hflag, &s_rwstage})
    b->bind(&budget);
  for (auto *b : {&pbeg, &hub_dir0, &s_A, &s_B, &s_C, &s_tmp, &s_cnt, &s_P, &s_oOff, &s_nOff,
                  &s_wk, &s_wk2, &s_mw, &s_old, &s_new, &s_hwplan, &s_mrec, &s_hplan, &s_hsel})
    b->bind(&budget);
  s_hnbd.bind(&budget);
  hub_of.bind(&budget);
  wstamp.bind(&budget);
  pbeg_alt.bind(&budget);
  s_tix.bind(&budget);
  s_wbits.bind(&budget);
  s_hw_do.bind(&budget);
  bsplits.bind(&budget);
  s_hw_h.bind(&budget);
  s_flags.bind(&budget);

  uint64_t nn = n ? n : 1;
  deg.alloc_exact(nn);
  inl.alloc_exact(nn * K_INLINE);
  c2.alloc_exact(nn);
  pbeg.alloc_exact(nn + 1);
  hub_of.alloc_exact(nn);
  stamp.alloc_exact(nn);
  wstamp.alloc_exact(nn);
  err.alloc_exact(4);
  s_cnt.alloc_exact(32);
  pma.alloc_exact(1);
  N = 0;
  TRC_CUDA(cudaMemsetAsync(deg.get(), 0, nn * 4, stream));
  TRC_CUDA(cudaMemsetAsync(inl.get(), 0, nn * K_INLINE * 4, stream));
  TRC_CUDA(cudaMemsetAsync(c2.get(), 0, nn * 4, stream));
  TRC_CUDA(cudaMemsetAsync(pbeg.get(), 0, (nn + 1) * 8, stream));
  TRC_CUDA(cudaMemsetAsync(hub_of.get(), 0xFF, nn * 4, stream));
  TRC_CUDA(cudaMemsetAsync(stamp.get(), 0, nn * 4, stream));
  TRC_CUDA(cudaMemsetAsync(wstamp.get(), 0, nn * 4, stream));
  TRC_CUDA(cudaMemsetAsync(err.get(), 0, 16, stream));
  hub_init();
  sync();
  // last, so that nothing after it can throw out of the constructor
  TRC_CUDA(cudaMallocHost(&hub_stage_, 256 + 4 * 4 * HUB_SPEC));  // 32 counters, 4 hub arrays
}

Graph::~Graph() {
  if (own_stream) cudaStreamSynchronize(own_stream);
  if (stream && stream != own_stream) cudaStreamSynchronize(stream);
  if (side_stream) cudaStreamSynchronize(side_stream);
  if (copy_stream) cudaStreamSynchronize(copy_stream);
  prof.reset();
  if (prg.exec) cudaGraphExecDestroy(prg.exec);
  // the members free after this body, on the legacy stream (the work on
  // the graph's streams has finished)
  budget.stream = nullptr;
  if (hub_stage_) cudaFreeHost(hub_stage_);
  if (hub_pin_) cudaFreeHost(hub_pin_);
  if (ev_hub) cudaEventDestroy(ev_hub);
  if (ev_fork) cudaEventDestroy(ev_fork);
  if (ev_join) cudaEventDestroy(ev_join);
  if (ev_h2d) cudaEventDestroy(ev_h2d);
  if (copy_stream) cudaStreamDestroy(copy_stream);
  if (side_stream) cudaStreamDestroy(side_stream);
  if (own_stream) cudaStreamDestroy(own_stream);
}

DevView Graph::view() const {
  DevView v;
  v.n = n;
  v.hub_T = cfg.hub_threshold;
  v.deg = deg.get();
  v.inl = inl.get();
  v.pbeg = pbeg.get();
  v.c2 = c2.get();
  v.pma = pma.get();
  v.N = N;
  v.hub_of = hub_of.get();
  v.hub_vtx = hub_vtx.get();
  v.hub_dir0 = hub_dir0.get();
  v.hub_nblk = hub_nblk.get();
  v.hdir = hdir.get();
  v.hpre = hpre.get();
  v.hkey = hkey.get();
  v.hslot = hslot.get();
  v.bcnt = bcnt.get();
  v.bmin = bmin.get();
  v.bown = bown.get();
  v.err = err.get();
  return v;
}

void Graph::release_scratch() {
  sync();
  for (auto *b : {&s_in_src, &s_in_dst, &s_tu, &s_tdn, &s_tc2, &s_ovl, &s_hw_u, &s_hw_dn, &s_hw_t,
                  &s_c2n, &s_rlist, &s_pma_next, &s_tix, &s_hw_do, &s_wbits, &s_lg, &s_lx, &s_lli,

                  &s_tgq, &s_tgo, &s_tgb, &s_hflag, &s_rwstage, &bfreed})
    b->reset();
  for (auto *b : {&s_A, &s_B, &s_C, &s_tmp, &s_P, &s_oOff, &s_nOff, &s_wk, &s_wk2, &s_mw, &s_old,
                  &s_new, &s_hwplan, &pbeg_alt, &s_mrec, &s_hplan, &s_hsel})
    b->reset();
  s_hw_h.reset();
  s_hnbd.reset();
  s_flags.reset();
  lists.version = ~0ull;
  for (auto *b : {&lists.S, &lists.M, &lists.Hv, &lists.SM, &lists.M1, &lists.M2})
    b->reset();
  sync();
  budget.trim();
}

uint32_t Graph::vbits() const {
  uint32_t b = 1;
  while (b < 32 && (1ull << b) < (uint64_t)n) b++;
  return b;
}

void Graph::sync() { TRC_CUDA(cudaStreamSynchronize(stream)); }

void Graph::phase(const char *name) {
  if (!prof.on) return;
  double now = std::chrono::duration<double, std::milli>(
                   std::chrono::steady_clock::now().time_since_epoch())
                   .count();
  if (name) {
    auto &t = prof.totals[std::string("host:") + name];
    t.first += now - phase_t0;
    t.second += 1;
  }
  phase_t0 = now;
}

uint64_t Graph::read_u64(const uint64_t *dptr) {
  uint64_t v = 0;
  TRC_CUDA(cudaMemcpyAsync(&v, dptr, 8, cudaMemcpyDeviceToHost, stream));
  sync();
  return v;
}

// ---------------------------------------------------------------------------
// Kernels of the pipeline

__global__ void k_make_keys(const uint32_t *src, const uint32_t *dst, uint64_t k, uint32_t n,
                            int sym, int drop_self, uint64_t *keys, uint32_t *err) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= k) return;
  uint32_t s = src[i], d = dst[i];
  uint64_t a = KEY_INVALID, b = KEY_INVALID;
  if (s >= n || d >= n) {
    atomicOr(err, ERR_BAD_VERTEX);
  } else if (!(drop_self && s == d)) {
    a = ((uint64_t)s << 32) | d;
    b = ((uint64_t)d << 32) | s;
  }
  if (sym) {
    keys[2 * i] = a;
    keys[2 * i + 1] = b;
  } else {
    keys[i] = a;
  }
}

// Unique test and existence filter in one pass, one tier lookup per key:
// flag[i] = key i is the first of its run and (insert: absent / remove:
// present) in the graph.
__global__ void k_filter_flags(DevView G, const uint64_t *keys, uint64_t k2, int insert,
                               uint8_t *flags) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= k2) return;
  uint64_t x = keys[i];
  // (ids checked against n too: a key that is not a valid edge never passes,
  // whatever an upstream failure left in the buffer)
  bool keep = x != KEY_INVALID && (x >> 32) < G.n && (uint32_t)x < G.n &&
              (i == 0 || keys[i - 1] != x);
  if (keep) {
    bool has = has_edge(G, (uint32_t)(x >> 32), (uint32_t)x);
    keep = insert ? !has : has;
  }
  flags[i] = keep ? 1 : 0;
}

struct FlagPred {
  const uint8_t *f;
  __device__ bool operator()(uint64_t i) const { return f[i] != 0; }
};

struct RunStartPred {
  const uint64_t *keys;
  const uint64_t *count;
  __device__ bool operator()(uint64_t i) const {
    if (i >= *count) return false;
    return i == 0 || (keys[i] >> 32) != (keys[i - 1] >> 32);
  }
};

struct IndexVal {
  __device__ uint64_t operator()(uint64_t i) const { return i; }
};

// Counters in s_cnt (device u64 array)
enum {
  C_KU = 0,
  C_KB,
  C_NT,
  C_NOV,
  C_NH,
  C_ROOT,
  C_NW,
  C_NMW,
  C_NR,
  C_T2DELTA,
  C_MWORK,  // rewrite entries handed out to k_merge_small's warps
  C_COUNT
};

// Warp-aggregated append: one atomic per warp, returns this lane's slot.
__device__ __forceinline__ uint64_t warp_append64(bool take, unsigned long long *counter) {
  uint32_t m = __ballot_sync(0xFFFFFFFFu, take);
  uint64_t base = 0;
  if (m) {
    uint32_t leader = __ffs(m) - 1;
    if ((threadIdx.x & 31) == leader) base = atomicAdd(counter, (unsigned long long)__popc(m));
    base = __shfl_sync(0xFFFFFFFFu, base, leader);
  }
  return base + __popc(m & lanemask_lt());
}

// Classify touched vertices (step 4).
__global__ void k_classify(DevView G, const uint64_t *bkeys, const uint64_t *tpos, int insert,
                           uint32_t *tu, uint32_t *tdn, uint32_t *tc2, uint32_t *ovl,
                           uint32_t *hw_u, uint32_t *hw_dn, uint32_t *hw_t, int32_t *hw_h,
                           uint32_t *hw_do, uint64_t *cnt, uint64_t cap) {
  const uint64_t nt = cnt[C_NT], kb = cnt[C_KB];  // on the device: no synchronisation before
  uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  // t < cap too: cap (the touched tables' size) bounds nt for a sorted batch;
  // after a failed sort (the call fails at the next synchronisation) the
  // run count may be anything
  bool valid = t < nt && t < cap;
  uint32_t u = 0, dn = 0, d = 0;
  int32_t h = -1;
  bool hub = false, over = false;
  long long delta = 0;
  if (valid) {
    uint64_t p0 = tpos[t];
    uint64_t p1 = t + 1 < nt ? tpos[t + 1] : kb;
    u = (uint32_t)(bkeys[p0] >> 32);
    uint32_t c = (uint32_t)(p1 - p0);
    d = G.deg[u];
    dn = insert ? d + c : d - c;
    h = G.hub_of[u];
    hub = h >= 0 || dn > G.hub_T;
    uint32_t nc2 = (!hub && dn > K_INLINE) ? dn - K_INLINE : 0;
    tu[t] = u;
    tdn[t] = dn;
    tc2[t] = nc2;
    delta = (long long)nc2 - (long long)G.c2[u];
    over = !hub && (uint64_t)nc2 > G.pbeg[u + 1] - G.pbeg[u];
  }
  // per-warp delta sum, one atomic per warp
  long long wd = delta;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) wd += __shfl_xor_sync(0xFFFFFFFFu, wd, o);
  if ((threadIdx.x & 31) == 0 && wd)
    atomicAdd((unsigned long long *)&cnt[C_T2DELTA], (unsigned long long)wd);
  uint64_t j = warp_append64(over, (unsigned long long *)&cnt[C_NOV]);
  if (over) ovl[j] = u;
  j = warp_append64(valid && hub, (unsigned long long *)&cnt[C_NH]);
  if (valid && hub) {
    hw_u[j] = u;
    hw_dn[j] = dn;
    hw_t[j] = (uint32_t)t;
    hw_h[j] = h;
    hw_do[j] = d;
  }
}

__global__ void k_scatter_c2(const uint32_t *tu, const uint32_t *tc2, const uint64_t *nt,
                             uint64_t cap, uint32_t *c2n) {
  uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < *nt && t < cap) c2n[tu[t]] = tc2[t];
}

struct LoadC2 {
  const uint32_t *c;
  __device__ uint64_t operator()(uint64_t i) const { return c[i]; }
};

// Per-level bitmaps of the chosen windows: level h has one bit per aligned
// range of 2^h vertices, starting at word base[h].
struct WinBits {
  uint32_t *mark;  // windows chosen by some overflow vertex
  uint32_t *emit;  // maximal windows already listed
  uint64_t base[34];
};

__device__ __forceinline__ bool win_bit(const uint32_t *bits, const WinBits &wb, uint32_t h,
                                        uint64_t idx) {
  return (bits[wb.base[h] + (idx >> 5)] >> (idx & 31)) & 1u;
}

// Window search (step 5): lowest level (from the leaf level, 2^leaf vertex
// segments) whose aligned vertex range has density within its bound; its
// key is (start << 6 | 63 - level) and its bit is set in the level bitmap.
__global__ void k_find_windows(const uint32_t *ovl, const uint64_t *nov, const uint64_t *P,
                               const uint64_t *pbeg, uint32_t n, uint32_t levels, uint32_t leaf,
                               double root_dens, uint64_t *wkeys, uint64_t *cnt, WinBits wb) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= *nov) return;
  uint32_t u = ovl[i];
  for (uint32_t h = leaf; h <= levels; h++) {
    uint64_t a = ((uint64_t)u >> h) << h;
    uint64_t b = a + (1ull << h);
    if (b > n) b = n;
    uint64_t E = P[b] - P[a];
    uint64_t S = pbeg[b] - pbeg[a];
    double tau = 1.0 - (1.0 - root_dens) * (double)h / (double)levels;
    if ((double)E <= tau * (double)S) {
      wkeys[i] = (a << 6) | (uint64_t)(63 - h);
      const uint64_t idx = a >> h;
      atomicOr(wb.mark + wb.base[h] + (idx >> 5), 1u << (idx & 31));
      return;
    }
  }
  wkeys[i] = KEY_INVALID;
  atomicOr((unsigned long long *)&cnt[C_ROOT], 1ull);
}

// Maximal windows without sorting: aligned windows are nested or disjoint,
// so a chosen window is maximal exactly when no enclosing range (the same
// start shifted to every higher level) is chosen; the first overflow vertex
// to claim a maximal window's emit bit lists it (order is irrelevant: the
// windows are laid out independently).
__global__ void k_win_select(const uint64_t *wkeys, const uint64_t *nov, uint32_t levels, WinBits wb,
                             uint64_t *mw, unsigned long long *nmw) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= *nov) return;
  const uint64_t x = wkeys[i];
  if (x == KEY_INVALID) return;
  const uint64_t a = x >> 6;
  const uint32_t h = 63 - (uint32_t)(x & 63);
  for (uint32_t h2 = h + 1; h2 <= levels; h2++)
    if (win_bit(wb.mark, wb, h2, a >> h2)) return;
  const uint64_t idx = a >> h;
  const uint32_t bit = 1u << (idx & 31);
  if (!(atomicOr(wb.emit + wb.base[h] + (idx >> 5), bit) & bit)) mw[atomicAdd(nmw, 1ull)] = x;
}

struct LoadU64Val {
  const uint64_t *p;
  __device__ uint64_t operator()(uint64_t i) const { return p[i]; }
};

// Marks the touched vertices and records u -> touched index (tix), so the
// merge finds a vertex's slice of the batch without a search.  Runs after the
// window / rebuild marking, which resets tix to NONE32 for its vertices.
__global__ void k_mark_touched(const uint32_t *tu, uint64_t nt, uint32_t *stamp, uint32_t *tix,
                               uint32_t epoch) {
  uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < nt) {
    stamp[tu[t]] = epoch;
    tix[tu[t]] = (uint32_t)t;
  }
}

// Slack of a layout is spread in proportion to (elements + PMA_VWEIGHT), so a
// vertex with few or no PMA elements still gets a few free slots: a vertex
// crossing the inline limit then usually fits without a window rebalance.
constexpr uint64_t PMA_VWEIGHT = 4;

__device__ __forceinline__ void window_range(uint64_t x, uint32_t n, uint64_t &a, uint64_t &b) {
  a = x >> 6;
  uint32_t h = 63 - (uint32_t)(x & 63);
  b = a + (1ull << h);
  if (b > n) b = n;
}

// One CTA per maximal window: put its vertices in the rewrite set.
__global__ void k_window_mark(const uint64_t *mw, uint32_t n, uint32_t *stamp, uint32_t epoch) {
  uint64_t a, b;
  window_range(mw[blockIdx.x], n, a, b);
  for (uint64_t u = a + threadIdx.x; u < b; u += blockDim.x) stamp[u] = epoch;
}

// One CTA per maximal window: new segment offsets of its vertices,
// pbeg'[u] = pbeg[a] + (P[u]-P[a]) + floor(gap*Q(u)/Q(b)) with
// Q(u) = (P[u]-P[a]) + PMA_VWEIGHT*(u-a); the window's slot range
// [pbeg[a], pbeg[b]) is unchanged and every vertex keeps >= its elements.
__global__ void k_window_layout(const uint64_t *mw, uint32_t n, const uint64_t *P, uint64_t *pbeg) {
  uint64_t a, b;
  window_range(mw[blockIdx.x], n, a, b);
  uint64_t base = pbeg[a];
  uint64_t S = pbeg[b] - base;
  uint64_t E = P[b] - P[a];
  uint64_t gap = S - E;
  uint64_t QW = E + PMA_VWEIGHT * (b - a);
  __syncthreads();  // every thread has read pbeg[a], pbeg[b] before any write
  for (uint64_t u = a + 1 + threadIdx.x; u < b; u += blockDim.x) {
    uint64_t e = P[u] - P[a];
    uint64_t q = e + PMA_VWEIGHT * (u - a);
    pbeg[u] = base + e + (uint64_t)(((unsigned __int128)gap * q) / QW);
  }
}

// Rebuild layout: every vertex, target density; pbeg'[n] = N'.
__global__ void k_rebuild_layout(const uint64_t *P, uint32_t n, uint64_t Nn, uint64_t *pbeg) {
  uint64_t u = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (u > n) return;
  uint64_t tot = P[n];
  uint64_t gap = Nn > tot ? Nn - tot : 0;
  uint64_t QW = tot + PMA_VWEIGHT * (uint64_t)n;
  uint64_t e = P[u];
  uint64_t q = e + PMA_VWEIGHT * u;
  uint64_t extra = QW ? (uint64_t)(((unsigned __int128)gap * q) / QW) : 0;
  pbeg[u] = (u == n) ? Nn : e + extra;
}

__global__ void k_mark_pma_vertices(const uint32_t *c2n, uint32_t n, uint32_t *stamp,
                                    uint32_t *tix, uint32_t epoch) {
  uint64_t u = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (u < n && c2n[u] > 0) {
    stamp[u] = epoch;
    tix[u] = NONE32;
  }
}

struct StampPred {
  const uint32_t *stamp;
  uint32_t epoch;
  __device__ bool operator()(uint64_t i) const { return stamp[i] == epoch; }
};

struct IndexVal32 {
  __device__ uint32_t operator()(uint64_t i) const { return (uint32_t)i; }
};

struct OldDeg {
  const uint32_t *rlist, *deg;
  __device__ uint64_t operator()(uint64_t i) const { return deg[rlist[i]]; }
};

// New degree of a rewrite-set vertex: from the touched table when touched.
struct NewDeg {
  const uint32_t *rlist, *deg, *tix, *tdn;
  __device__ uint64_t operator()(uint64_t i) const {
    uint32_t u = rlist[i];
    uint32_t t = tix[u];
    return t != NONE32 ? tdn[t] : deg[u];
  }
};

__global__ void k_scatter_c2_final(const uint32_t *tu, const uint32_t *tc2, uint64_t nt,
                                   uint32_t *c2) {
  uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < nt) c2[tu[t]] = tc2[t];
}

// ---------------------------------------------------------------------------
// Fused per-vertex merge for vertices that stay in tiers 1-2 (degree <= the
// hub threshold before and after).  One warp per vertex: the old list is
// staged in shared memory, every old element's output rank is its index plus
// the number of batch keys below it (binary search in the vertex's slice of
// the sorted batch), every inserted key's rank is its index plus the number
// of old elements below it; outputs go straight to the inline row and the
// PMA segment (in place, or to the layout's new position).  About 8 bytes of
// HBM traffic per list element instead of a gather / global merge / scatter.

// Touched vertices handled by the fused merge: non-hubs that stay <= T.
struct TouchedSmallPred {
  const uint32_t *tu, *tdn;
  const int32_t *hub_of;
  uint32_t T;
  __device__ bool operator()(uint64_t t) const { return hub_of[tu[t]] < 0 && tdn[t] <= T; }
};

struct TouchedVal {
  const uint32_t *tu;
  __device__ uint32_t operator()(uint64_t t) const { return tu[t]; }
};

// One CTA per maximal window: appends the window's members that are not
// touched but have PMA elements (their segments move) to the rewrite list
// after the touched ones (count on the device).
__global__ void k_window_members(const uint64_t *mw, uint32_t n, const uint32_t *tix,
                                 const int32_t *hub_of, const uint32_t *c2, uint32_t *rs,
                                 unsigned long long *nrs) {
  __shared__ uint32_t sh[256 / 32 + 2];
  uint64_t a, b;
  window_range(mw[blockIdx.x], n, a, b);
  for (uint64_t base = a; base < b; base += blockDim.x) {
    const uint64_t u = base + threadIdx.x;
    const bool take = u < b && tix[u] == NONE32 && hub_of[u] < 0 && c2[u] > 0;
    // per-CTA append (every thread of the CTA runs the same iterations)
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
      sh[8] = t ? (uint32_t)atomicAdd(nrs, (unsigned long long)t) : 0u;
    }
    __syncthreads();
    if (take) rs[sh[8] + sh[w] + __popc(m & lanemask_lt())] = (uint32_t)u;
    __syncthreads();
  }
}

// Rewrite-set members handled by the fused merge: non-hubs that stay <= T.
struct SmallPred {
  const uint32_t *stamp;
  uint32_t epoch;
  const int32_t *hub_of;
  const uint32_t *deg, *tix, *tdn;
  uint32_t T;
  __device__ bool operator()(uint64_t i) const {
    if (stamp[i] != epoch || hub_of[i] >= 0) return false;
    uint32_t t = tix[i];
    uint32_t dn = t != NONE32 ? tdn[t] : deg[i];
    return dn <= T;
  }
};

struct MergeArgs {
  const uint32_t *rs;
  uint64_t nrs;
  const uint32_t *tix;
  const uint64_t *tpos;
  uint64_t nt, kb;
  const uint64_t *bkeys;
  int insert;
  const uint64_t *pbeg_new;  // segment offsets after this batch
  uint32_t *dst_pma;         // destination of vertices that do not move
  uint32_t *mov_pma;         // destination of vertices inside a rebalanced window
  const uint32_t *wstamp;    // window marks (null: no window moves)
  uint32_t epoch;
  uint32_t T;
  int inplace;               // dst_pma is the live array: unmoved lists keep their prefix
};

// Index of the first element of u's list that is >= x, found by the warp:
// 32 evenly spaced pivots, then 32-element chunks of the bracketed range.
// Every lane returns the same value.
__device__ __forceinline__ uint32_t warp_list_lower_bound(const NbrList &L, uint32_t d, uint32_t x,
                                                         uint32_t lane) {
  const uint32_t step = (d + 31) / 32;
  uint32_t idx = lane * step;
  bool lt = idx < d && L.at(idx) < x;
  uint32_t c = __popc(__ballot_sync(0xFFFFFFFFu, lt));  // pivots below x (a prefix)
  if (step == 1) return c;
  uint32_t lo = c ? (c - 1) * step + 1 : 0;  // pivot c-1 is below x
  uint32_t hi = c * step < d ? c * step : d;  // pivot c (if any) is not
  while (lo < hi) {
    uint32_t j = lo + lane;
    uint32_t k = __popc(__ballot_sync(0xFFFFFFFFu, j < hi && L.at(j) < x));
    if (k < 32 || lo + 32 >= hi) return lo + k;
    lo += 32;
  }
  return lo;
}

__device__ __forceinline__ uint32_t lower_bound_keys(const uint64_t *B, uint32_t nb, uint32_t x) {
  uint32_t lo = 0, hi = nb;
  while (lo < hi) {
    uint32_t mid = (lo + hi) >> 1;
    if ((uint32_t)B[mid] < x) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ uint32_t lower_bound_u32(const uint32_t *A, uint32_t na, uint32_t x) {
  uint32_t lo = 0, hi = na;
  while (lo < hi) {
    uint32_t mid = (lo + hi) >> 1;
    if (A[mid] < x) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// Register variant (no shared memory, so occupancy is set by registers):
// the list is moved in chunks of MF_CH elements held in registers, which is
// safe in place because an insertion only moves elements up (chunks are
// taken from the top down) and a deletion only moves them down (bottom up);
// the loads of a chunk complete (__syncwarp) before its stores.
// Insertion ranks without searching the old list: with c(i) = number of
// batch keys below old element i (c(p-1) = 0, c(d) = nb), key j lands at
// j + i for the i with c(i-1) <= j < c(i); the lane holding element i writes
// those keys while the chunk is in registers, at positions >= i >= the
// chunk's start, so no unread element is overwritten.
constexpr uint32_t MF_R = 4;
constexpr uint32_t MF_CH = 32 * MF_R;

__device__ __forceinline__ void put_rank(uint32_t *row, uint32_t *seg, uint32_t r, uint32_t x) {
  if (r < K_INLINE) row[r] = x;
  else seg[r - K_INLINE] = x;
}

// Per rewrite entry, packed by k_merge_prep (one thread per entry, all its
// loads independent across threads): x = batch slice start << MR_BITS | key
// count, y = old segment offset << MR_BITS | old degree.  The merge's warp
// then reads it next to rs[w] instead of the dependent chains
// rs -> tix -> tpos and rs -> hub_of -> pbeg (about 5 % of the merge's time
// at RMAT scale 22, batch 1e6).  Both counts are at most the hub threshold
// (<= HUB_THRESHOLD_MAX by the configuration check); slice starts and segment offsets
// stay below 2^40 (an 8 TB batch or PMA).
constexpr uint32_t MR_BITS = 24;
constexpr uint64_t MR_MASK = (1ull << MR_BITS) - 1;

// Rewrite entries whose old list has at most MG_D elements are merged by
// MG_G lanes each (k_merge_group), the rest by a warp (k_merge_small); both
// kernels walk the whole rewrite list and take their entries by the old
// degree in the merge record.
constexpr uint32_t MG_G = 8;   // lanes per short list
constexpr uint32_t MG_R = 8;   // elements per lane: MG_G * MG_R covers a short list
constexpr uint32_t MG_D = MG_G * MG_R;

__global__ void k_merge_prep(DevView G, MergeArgs a, const uint64_t *nrs, ulonglong2 *rec) {
  const uint64_t nw = *nrs;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < nw; w += stride) {
    const uint32_t u = a.rs[w];
    const uint32_t t = a.tix[u];
    uint64_t b0 = 0, b1 = 0;
    if (t != NONE32) {
      b0 = a.tpos[t];
      b1 = t + 1 < a.nt ? a.tpos[t + 1] : a.kb;
    }
    rec[w] = make_ulonglong2((b0 << MR_BITS) | (b1 - b0), (G.pbeg[u] << MR_BITS) | G.deg[u]);
  }
}

__device__ __forceinline__ void merge_one(const DevView &G, const MergeArgs &a,
                                          const ulonglong2 *rec, uint64_t w, uint32_t lane) {
  const uint32_t u = a.rs[w];
  const ulonglong2 r = rec[w];
  const uint64_t b0 = r.x >> MR_BITS;
  const uint32_t nb = (uint32_t)(r.x & MR_MASK);
  NbrList L;  // (merge vertices are never hubs)
  L.deg = (uint32_t)(r.y & MR_MASK);
  L.inl = G.inl + (uint64_t)u * K_INLINE;
  L.ni = L.deg < K_INLINE ? L.deg : K_INLINE;
  L.rest = L.deg - L.ni;
  L.seg = G.pma + (r.y >> MR_BITS);
  L.nb = 0;
  L.dir = L.pre = L.key = nullptr;
  const uint32_t d = L.deg;
  const uint64_t *B = a.bkeys + b0;
  uint32_t *row = G.inl + (uint64_t)u * K_INLINE;
  const bool moved = a.wstamp && a.wstamp[u] == a.epoch;
  uint32_t *seg = (moved ? a.mov_pma : a.dst_pma) + a.pbeg_new[u];
  // elements below the first key keep their place (in place, long lists);
  // in place, an element whose rank does not change is not rewritten
  const bool stay = a.inplace && !moved;
  uint32_t p = 0;
  if (a.inplace && !moved && nb > 0 && d > MF_CH)
    p = warp_list_lower_bound(L, d, (uint32_t)B[0], lane);
  if (a.insert) {
    // keys above every old element: ranks j + d
    uint32_t ctop = 0;
    if (d > p) ctop = lower_bound_keys(B, nb, L.at(d - 1));
    for (uint32_t j = ctop + lane; j < nb; j += 32) put_rank(row, seg, j + d, (uint32_t)B[j]);
    // chunks from the top down; kc = keys below the chunk's top element
    uint32_t kc = ctop;
    for (uint32_t e = d; e > p;) {
      const uint32_t s0 = e - p > MF_CH ? e - MF_CH : p;
      uint32_t x[MF_R], c[MF_R];
#pragma unroll
      for (uint32_t k = 0; k < MF_R; k++) {
        uint32_t i = s0 + k * 32 + lane;
        x[k] = i < e ? L.at(i) : 0u;
      }
      // The chunk's keys lie between the element under it and its top
      // element.  They are walked down from kc, 32 at a time from a
      // register window, each broadcast to the lanes, which count the keys
      // above their elements: c = kc - that count (an inserted key never
      // equals a list element).  Work per chunk: its own keys, not a
      // search per element.
      const bool floor = s0 > p;
      const uint32_t xb = floor ? L.at(s0 - 1) : 0u;
      uint32_t gt[MF_R];
#pragma unroll
      for (uint32_t k = 0; k < MF_R; k++) gt[k] = 0;
      int32_t j = (int32_t)kc - 1;
      while (j >= 0) {
        const int32_t jl = j - 31 + (int32_t)lane;
        const uint32_t bl = jl >= 0 ? (uint32_t)B[jl] : 0u;
        // keys ascend with the lane: those above xb are the top lanes
        const uint32_t cnt = __popc(__ballot_sync(0xFFFFFFFFu, jl >= 0 && (!floor || bl > xb)));
        for (uint32_t t = 0; t < cnt; t++) {
          const uint32_t bj = __shfl_sync(0xFFFFFFFFu, bl, 31 - t);
#pragma unroll
          for (uint32_t k = 0; k < MF_R; k++) gt[k] += bj > x[k] ? 1u : 0u;
        }
        j -= (int32_t)cnt;
        if (cnt < 32) break;
      }
      const uint32_t cbelow = (uint32_t)(j + 1);  // keys below the element under the chunk
#pragma unroll
      for (uint32_t k = 0; k < MF_R; k++) c[k] = kc - gt[k];
      __syncwarp();
#pragma unroll
      for (uint32_t k = 0; k < MF_R; k++) {
        uint32_t i = s0 + k * 32 + lane;
        uint32_t cp = __shfl_up_sync(0xFFFFFFFFu, c[k], 1);
        uint32_t last = k > 0 ? __shfl_sync(0xFFFFFFFFu, c[k > 0 ? k - 1 : 0], 31) : cbelow;
        if (lane == 0) cp = last;
        if (i < e) {
          if (c[k] || !stay) put_rank(row, seg, i + c[k], x[k]);
          for (uint32_t j2 = cp; j2 < c[k]; j2++) put_rank(row, seg, j2 + i, (uint32_t)B[j2]);
        }
      }
      __syncwarp();
      kc = cbelow;
      e = s0;
    }
    // list empty above p (d == p): the keys all went above
  } else {
    // chunks from the bottom up; kl = keys below the chunk's first element
    // (0 at p: every key is a list element, and p is the first element
    // not below the smallest key, or 0)
    uint32_t kl = 0;
    for (uint32_t s0 = p; s0 < d; s0 += MF_CH) {
      const uint32_t e = d - s0 > MF_CH ? s0 + MF_CH : d;
      uint32_t x[MF_R];
#pragma unroll
      for (uint32_t k = 0; k < MF_R; k++) {
        uint32_t i = s0 + k * 32 + lane;
        x[k] = i < e ? L.at(i) : 0u;
      }
      // the chunk's keys (up to its top element) walked up from kl, 32 at a
      // time: each lane counts those below its elements and flags a key
      // equal to one
      const uint32_t xt = L.at(e - 1);
      uint32_t lt[MF_R], eq = 0;
#pragma unroll
      for (uint32_t k = 0; k < MF_R; k++) lt[k] = 0;
      uint32_t j = kl;
      while (j < nb) {
        const uint32_t jl = j + lane;
        const uint32_t bl = jl < nb ? (uint32_t)B[jl] : 0u;
        // keys ascend with the lane: those up to xt are the bottom lanes
        const uint32_t cnt = __popc(__ballot_sync(0xFFFFFFFFu, jl < nb && bl <= xt));
        for (uint32_t t = 0; t < cnt; t++) {
          const uint32_t bj = __shfl_sync(0xFFFFFFFFu, bl, t);
#pragma unroll
          for (uint32_t k = 0; k < MF_R; k++) {
            lt[k] += bj < x[k] ? 1u : 0u;
            eq |= bj == x[k] ? 1u << k : 0u;
          }
        }
        j += cnt;
        if (cnt < 32) break;
      }
      __syncwarp();
#pragma unroll
      for (uint32_t k = 0; k < MF_R; k++) {
        uint32_t i = s0 + k * 32 + lane;
        if (i < e) {
          const uint32_t cc = kl + lt[k];
          if (!((eq >> k) & 1u) && (cc || !stay)) put_rank(row, seg, i - cc, x[k]);
        }
      }
      __syncwarp();
      kl = j;
    }
  }
  if (lane == 0) G.deg[u] = a.insert ? d + nb : d - nb;
}

// Persistent over the rewrite list, whose length is read on the device;
// warps take MS_CHUNK entries at a time from a counter, so CTAs that start
// late (behind the hub merge on the side stream) take fewer.  (Long lists
// cluster in the list; per 1e6-pair batch on RMAT-22 the merge took 232 us
// with 4 entries per grab, 252 with 8, 302 with 2, 516 with 1: the counter
// contends below 4, the warps' loads unbalance above.)
constexpr uint32_t MS_CHUNK = 4;

__global__ void __launch_bounds__(256, 8) k_merge_small(DevView G, MergeArgs a,
                                                        const uint64_t *nrs,
                                                        const ulonglong2 *rec,
                                                        unsigned long long *work) {
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t nw = *nrs;
  for (;;) {
    uint64_t w0 = 0;
    if (lane == 0) w0 = atomicAdd(work, (unsigned long long)MS_CHUNK);
    w0 = __shfl_sync(0xFFFFFFFFu, w0, 0);
    if (w0 >= nw) break;
    const uint64_t w1 = w0 + MS_CHUNK < nw ? w0 + MS_CHUNK : nw;
    for (uint64_t w = w0; w < w1; w++)
      if ((rec[w].y & MR_MASK) > MG_D) merge_one(G, a, rec, w, lane);  // (short: k_merge_group)
  }
}

// MG_G lanes per short rewrite entry (old list of at most MG_D elements),
// four entries per warp: the whole old list is loaded into registers (MG_R
// per lane) before anything is written, so in place needs no ordering; each
// element goes to its index plus the keys below it (insert: the lane holding
// element i also writes the keys that land between element i-1 and i) or
// minus the keys below it (remove), as merge_one does for one chunk.
__global__ void __launch_bounds__(256, 4) k_merge_group(DevView G, MergeArgs a,
                                                        const uint64_t *nrs,
                                                        const ulonglong2 *rec) {
  const uint32_t lane = threadIdx.x & 31, g = lane & (MG_G - 1);
  const unsigned mask = ((1u << MG_G) - 1u) << (lane & ~(MG_G - 1));
  const uint64_t nw = *nrs;
  const uint64_t ngroups = ((uint64_t)gridDim.x * blockDim.x) / MG_G;
  for (uint64_t w = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / MG_G; w < nw;
       w += ngroups) {
    const ulonglong2 r = rec[w];
    if ((r.y & MR_MASK) > MG_D) continue;  // (long: k_merge_small; group-uniform)
    const uint32_t u = a.rs[w];
    const uint64_t b0 = r.x >> MR_BITS;
    const uint32_t nb = (uint32_t)(r.x & MR_MASK);
    const uint32_t d = (uint32_t)(r.y & MR_MASK);
    const uint32_t *oseg = G.pma + (r.y >> MR_BITS);  // old tier-2 elements, rank 16 on
    uint32_t *row = G.inl + (uint64_t)u * K_INLINE;
    const uint64_t *B = a.bkeys + b0;
    const bool moved = a.wstamp && a.wstamp[u] == a.epoch;
    uint32_t *seg = (moved ? a.mov_pma : a.dst_pma) + a.pbeg_new[u];
    const bool stay = a.inplace && !moved;
    uint32_t x[MG_R], c[MG_R];
#pragma unroll
    for (uint32_t k = 0; k < MG_R; k++) {
      const uint32_t i = k * MG_G + g;
      x[k] = i < d ? (i < K_INLINE ? row[i] : oseg[i - K_INLINE]) : 0u;
    }
#pragma unroll
    for (uint32_t k = 0; k < MG_R; k++) {
      const uint32_t i = k * MG_G + g;
      c[k] = i < d ? lower_bound_keys(B, nb, x[k]) : 0u;
    }
    __syncwarp(mask);
    if (a.insert) {
      // keys above every old element: ranks j + d
      // (c of the last element counts the keys below it; the others are
      // above it, since inserted keys are absent from the list)
      uint32_t cl = 0;
#pragma unroll
      for (uint32_t k = 0; k < MG_R; k++)
        if (d && k == (d - 1) / MG_G) cl = c[k];
      const uint32_t ctop = d ? __shfl_sync(mask, cl, (d - 1) % MG_G, MG_G) : 0u;
      for (uint32_t j = ctop + g; j < nb; j += MG_G) put_rank(row, seg, j + d, (uint32_t)B[j]);
#pragma unroll
      for (uint32_t k = 0; k < MG_R; k++) {
        const uint32_t i = k * MG_G + g;
        uint32_t cp = __shfl_up_sync(mask, c[k], 1, MG_G);
        const uint32_t last = k > 0 ? __shfl_sync(mask, c[k > 0 ? k - 1 : 0], MG_G - 1, MG_G) : 0u;
        if (g == 0) cp = last;
        if (i < d) {
          if (c[k] || !stay) put_rank(row, seg, i + c[k], x[k]);
          for (uint32_t j = cp; j < c[k]; j++) put_rank(row, seg, j + i, (uint32_t)B[j]);
        }
      }
    } else {
#pragma unroll
      for (uint32_t k = 0; k < MG_R; k++) {
        const uint32_t i = k * MG_G + g;
        if (i < d) {
          const uint32_t cc = c[k];
          if (!(cc < nb && (uint32_t)B[cc] == x[k]) && (cc || !stay)) put_rank(row, seg, i - cc, x[k]);
        }
      }
    }
    if (g == 0) G.deg[u] = a.insert ? d + nb : d - nb;
    __syncwarp(mask);
  }
}

// Moves the segments written to the window buffer to their final slots
// (persistent over the rewrite list, length read on the device).
__global__ void k_window_copy(DevView G, const uint32_t *rs, const uint64_t *nrs,
                              const uint32_t *mov, const uint64_t *pbeg_new, const uint32_t *wstamp,
                              uint32_t epoch) {
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t nw = *nrs;
  const uint64_t stride = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t w = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < nw; w += stride) {
    uint32_t u = rs[w];
    if (wstamp[u] != epoch) continue;
    uint32_t dn = G.deg[u];
    if (dn <= K_INLINE) continue;
    uint64_t o = pbeg_new[u];
    for (uint32_t j = lane; j < dn - K_INLINE; j += 32) G.pma[o + j] = mov[o + j];
  }
}

__global__ void k_window_mark2(const uint64_t *mw, uint32_t n, uint32_t *stamp, uint32_t *wstamp,
                               uint32_t *tix, uint32_t epoch) {
  uint64_t a, b;
  window_range(mw[blockIdx.x], n, a, b);
  for (uint64_t u = a + threadIdx.x; u < b; u += blockDim.x) {
    stamp[u] = epoch;
    wstamp[u] = epoch;
    tix[u] = NONE32;
  }
}

// Batches touching at least this many vertices search PMA windows before
// the classify counts are read (one synchronisation less; the O(n) prefix of
// the tier-2 counts is then computed even when no vertex overflows).
constexpr uint64_t PLAN_SPECULATE = 1u << 16;

// Batches of BUCKET_MIN_KEYS .. BUCKET_MAX_KEYS keys sort with the bucket
// sort (below, both sorts are a handful of launches over a few tiles; above,
// the buckets of skewed batches outgrow the shared-memory sorts).
constexpr uint64_t BUCKET_MIN_KEYS = 1u << 12;
constexpr uint64_t BUCKET_MAX_KEYS = 1u << 24;

// ---------------------------------------------------------------------------
// The pipeline

void Graph::complete_pending() {
  if (!tail_pending) return;
  sync();
  finish_tail();
}

// The pending batch's results that only its last kernels produce: the hub
// pool's free-list size and top (hubs_finish) and the rewrite count.
void Graph::finish_tail() {
  if (!tail_pending) return;
  tail_pending = false;
  hubs_finish();
  uint64_t nrs;
  memcpy(&nrs, hub_stage_ + 62, 8);
  last[3] = nrs + tail_nh;
  last[4] += hub_last[4];
  last[5] += hub_last[5];
}

uint64_t Graph::apply_batch(const uint32_t *src_in, const uint32_t *dst_in, uint64_t k,
                            uint32_t flags, bool insert, bool defer_tail) {
  if (k == 0) return 0;
  if (!src_in || !dst_in) throw_error(TRC_ERR_INVALID, "null edge array");
  const int sym = (flags & TRC_SYMMETRIZE) ? 1 : 0;
  const int drop = (flags & TRC_DROP_SELF_LOOPS) ? 1 : 0;
  phase(nullptr);
  const uint32_t *src, *dst;
  if (tail_pending && !(flags & TRC_DEVICE_PTR) && s_in_src.capacity() >= k &&
      s_in_dst.capacity() >= k) {
    // The previous batch's kernels that still run read neither staging
    // buffer (its key build, their only reader, finished before its first
    // synchronisation), so the copy overlaps them on the copy stream; a
    // buffer that must grow takes the ordered path below instead (its
    // allocation is ordered on the graph's stream).
    src = s_in_src.get();
    dst = s_in_dst.get();
    TRC_CUDA(cudaMemcpyAsync(s_in_src.get(), src_in, k * 4, cudaMemcpyHostToDevice, copy_stream));
    TRC_CUDA(cudaMemcpyAsync(s_in_dst.get(), dst_in, k * 4, cudaMemcpyHostToDevice, copy_stream));
    TRC_CUDA(cudaEventRecord(ev_h2d, copy_stream));
    TRC_CUDA(cudaStreamWaitEvent(stream, ev_h2d, 0));
  } else {
    src = to_device(*this, src_in, k, flags, s_in_src);
    dst = to_device(*this, dst_in, k, flags, s_in_dst);
  }
  const uint64_t k2 = sym ? 2 * k : k;
  DevView G = view();
  uint64_t *cnt = s_cnt.get();
  // the bucket sort unless the radix sort is asked for (or its wait test
  // hook is set); a bucket too large for it sends the batch back here, to
  // the radix sort, before anything is modified
  const bool hooks = sort_wait.withhold_first || sort_wait.spin_limit != SortWait{}.spin_limit;
  bool bucket = sort_mode == 2 ||
                (sort_mode == 0 && k2 >= BUCKET_MIN_KEYS && k2 <= BUCKET_MAX_KEYS && !hooks);
  // small batches: one CTA sorts them all (no radix passes)
  const bool small = sort_mode == 0 && !hooks && k2 <= SORT_SMALL_MAX;
retry_sort:
  TRC_CUDA(cudaMemsetAsync(cnt, 0, 32 * 8, stream));
  TRC_CUDA(cudaMemsetAsync(err.get(), 0, 4, stream));

  // 1-2: keys, sort, unique
  uint64_t *A = s_A.ensure(k2), *B = s_B.ensure(k2);
  TRC_LAUNCH(prof, stream, "upd_make_keys", ceil_div(k, 256), 256, 0, k_make_keys, src, dst, k, n,
             sym, drop, A, err.get());
  const uint32_t *splits = bsplits_ok ? bsplits.get() : nullptr;
  uint64_t *t = tmp(std::max({radix_tmp_elems(k2), select_tmp_elems(k2),
                              bucket ? bucket_tmp_elems(k2, n, splits != nullptr) : (uint64_t)0}));
  uint64_t *sorted = bucket  ? bucket_sort_u64(A, B, k2, n, t, stream, prof, err.get(), splits)
                     : small ? sort_small_u64(A, B, k2, stream, prof)
                             : radix_sort_u64(A, B, k2, vbits(), t, stream, prof, err.get(), sort_wait);
  // the next batches' bucket boundaries: quantiles of this batch's sources
  // (a batch large enough to show the distribution)
  if (k2 >= BUCKET_MIN_KEYS) {
    bucket_learn_splits(sorted, k2, n, bsplits.ensure(BUCKET_SPLITS + 1), stream, prof);
    bsplits_ok = true;
  }
  uint64_t *bkeys = sorted == A ? B : A;
  // 3: unique + existence filter (one lookup per key), compacted
  uint8_t *kflags = s_flags.ensure(k2);
  TRC_LAUNCH(prof, stream, "upd_filter", ceil_div(k2, 256), 256, 0, k_filter_flags, G, sorted, k2,
             insert ? 1 : 0, kflags);
  select_if(FlagPred{kflags}, LoadU64Val{sorted}, k2, bkeys, cnt + C_KB, t, stream, prof,
            "sel_filter");
  // 4: runs by source
  uint64_t *tpos = s_C.ensure(k2);
  select_if(RunStartPred{bkeys, cnt + C_KB}, IndexVal{}, k2, tpos, cnt + C_NT, t, stream, prof,
            "sel_runs");
  phase("sort_filter");
  // ---- classify on the device-side counts (no synchronisation here: the
  // batch's counts, the error word and the plan inputs are read together
  // after it; nothing modifies the graph before that read)
  uint64_t hc[C_COUNT];
  const uint64_t cap = std::min<uint64_t>(k2, n);  // touched vertices <= both
  uint32_t *tu = s_tu.ensure(cap), *tdn = s_tdn.ensure(cap), *tc2 = s_tc2.ensure(cap);
  uint32_t *ovl = s_ovl.ensure(cap);
  uint32_t *hw_u = s_hw_u.ensure(cap), *hw_dn = s_hw_dn.ensure(cap), *hw_t = s_hw_t.ensure(cap);
  int32_t *hw_h = s_hw_h.ensure(cap);
  TRC_LAUNCH(prof, stream, "upd_classify", ceil_div(cap, 256), 256, 0, k_classify, G, bkeys, tpos,
             insert ? 1 : 0, tu, tdn, tc2, ovl, hw_u, hw_dn, hw_t, hw_h, s_hw_do.ensure(cap), cnt,
             cap);
  // ---- PMA planning inputs: the new tier-2 counts c2n, their prefix P, and
  // (large batches) the window search on the device-side overflow count,
  // before the synchronisation that reads the counts; a rebuild decided
  // after it discards the windows
  const uint32_t T_levels = [&] {
    uint32_t l = 1;
    while (l < 32 && (1ull << l) < (uint64_t)n) l++;
    return l;
  }();
  const double root_d = (cfg.pma_root_density > 0 && cfg.pma_root_density < 1) ? cfg.pma_root_density : 0.75;
  uint32_t *c2n = nullptr;
  uint64_t *P = nullptr;
  auto plan_prefix = [&] {
    c2n = s_c2n.ensure(n);
    TRC_CUDA(cudaMemcpyAsync(c2n, c2.get(), (uint64_t)n * 4, cudaMemcpyDeviceToDevice, stream));
    TRC_LAUNCH(prof, stream, "upd_scatter_c2", ceil_div(cap, 256), 256, 0, k_scatter_c2, tu, tc2,
               cnt + C_NT, cap, c2n);
    P = s_P.ensure((uint64_t)n + 1);
    uint64_t *st = tmp(scan_tmp_elems(n) + 4);
    exclusive_scan(LoadC2{c2n}, n, P, st, stream, prof, "scan_c2");
  };
  auto plan_windows = [&](uint64_t cap) {  // cap >= the overflow count on the device
    uint64_t *wk = s_wk.ensure(cap);
    // level bitmaps (mark, emit), cleared per batch
    WinBits wb;
    uint64_t words = 0;
    for (uint32_t h = 0; h <= T_levels && h < 34; h++) {
      wb.base[h] = words;
      words += ceil_div(ceil_div((uint64_t)n, 1ull << h), 32);
    }
    uint32_t *wbits = s_wbits.ensure(2 * words);
    wb.mark = wbits;
    wb.emit = wbits + words;
    TRC_CUDA(cudaMemsetAsync(wbits, 0, 2 * words * 4, stream));
    TRC_LAUNCH(prof, stream, "upd_find_windows", ceil_div(cap, 256), 256, 0, k_find_windows, ovl,
               cnt + C_NOV, P, pbeg.get(), n, T_levels,
               std::min(std::max(tuned.pma_leaf_log, 1u), T_levels), root_d, wk, cnt, wb);
    uint64_t *mw = s_mw.ensure(cap);
    TRC_LAUNCH(prof, stream, "upd_win_select", ceil_div(cap, 256), 256, 0, k_win_select, wk,
               cnt + C_NOV, T_levels, wb, mw, (unsigned long long *)(cnt + C_NMW));
  };
  const bool speculate = k2 >= 2 * PLAN_SPECULATE;
  if (speculate) {
    plan_prefix();
    plan_windows(cap);
  }

  // the counts and (speculatively) the first HUB_SPEC touched-hub records in
  // one copy to pinned staging and one synchronisation; more hubs than that
  // take a second copy
  const uint64_t spec = std::min<uint64_t>(cap, HUB_SPEC);
  uint32_t *sp = hub_stage_ + 64;  // after the 32 counters
  // staging words: the counters 0 .. 2*C_COUNT-1, the error word 60, a
  // deferred batch's rewrite count 62-63, the hub records from 64 on
  static_assert(2 * C_COUNT <= 60, "counter staging");
  TRC_CUDA(cudaMemcpyAsync(hub_stage_, cnt, sizeof(hc), cudaMemcpyDeviceToHost, stream));
  TRC_CUDA(cudaMemcpyAsync(hub_stage_ + 60, err.get(), 4, cudaMemcpyDeviceToHost, stream));
  {
    const uint32_t *src4[4] = {hw_u, hw_dn, (const uint32_t *)hw_h, s_hw_do.get()};
    for (int a = 0; a < 4; a++)
      if (spec)
        TRC_CUDA(cudaMemcpyAsync(sp + a * HUB_SPEC, src4[a], spec * 4, cudaMemcpyDeviceToHost,
                                 stream));
  }
  sync();
  finish_tail();  // a deferred previous batch: its kernels ran before this point
  for (auto &x : hub_last) x = 0;
  memcpy(hc, hub_stage_, sizeof(hc));
  const uint32_t herr = hub_stage_[60];
  if (herr & ERR_BAD_VERTEX) throw_error(TRC_ERR_INVALID, "vertex id out of range [0, n)");
  if (herr & ERR_TIMEOUT) throw_error(TRC_ERR_TIMEOUT, "radix sort look-back wait gave up");
  if (herr & ERR_BIGSEG) {
    bucket = false;
    sort_retries++;
    goto retry_sort;
  }
  const uint64_t kb = hc[C_KB], nt = hc[C_NT];
  if (kb == 0) {
    for (auto &x : last) x = 0;
    last[0] = k2;
    return 0;
  }
  const uint64_t nov = hc[C_NOV], nh = hc[C_NH];
  const int64_t t2delta = (int64_t)hc[C_T2DELTA];
  const uint64_t t2new = (uint64_t)((int64_t)tier2_total + t2delta);

  phase("classify");
  // ---- tier 3: the touched hubs' records, then the first launch phase of
  // the hub update on the side stream (block-local groups located and
  // counted) while the host plans tiers 1-2
  std::vector<uint32_t> hu, hdn, hdo;
  std::vector<int32_t> hh;
  struct HubGuard {  // error path: no hub work may outlive the batch's buffers
    Graph *g;
    bool armed = true;
    ~HubGuard() {
      if (armed && (g->hub_ctx_.active || g->hub_ctx_.readback)) {
        g->hub_ctx_.active = g->hub_ctx_.readback = false;
        cudaStreamSynchronize(g->side_stream);
      }
    }
  } hub_guard{this, true};
  if (nh) {
    hu.resize(nh);
    hdn.resize(nh);
    hdo.resize(nh);
    hh.resize(nh);
    if (nh <= spec) {
      memcpy(hu.data(), sp, nh * 4);
      memcpy(hdn.data(), sp + HUB_SPEC, nh * 4);
      memcpy(hh.data(), sp + 2 * HUB_SPEC, nh * 4);
      memcpy(hdo.data(), sp + 3 * HUB_SPEC, nh * 4);
    } else {
      TRC_CUDA(cudaMemcpyAsync(hu.data(), hw_u, nh * 4, cudaMemcpyDeviceToHost, stream));
      TRC_CUDA(cudaMemcpyAsync(hdn.data(), hw_dn, nh * 4, cudaMemcpyDeviceToHost, stream));
      TRC_CUDA(cudaMemcpyAsync(hh.data(), hw_h, nh * 4, cudaMemcpyDeviceToHost, stream));
      TRC_CUDA(cudaMemcpyAsync(hdo.data(), s_hw_do.get(), nh * 4, cudaMemcpyDeviceToHost, stream));
      sync();
    }
    apply_hubs(nh, hu, hdn, hh, hdo, hw_t, bkeys, tpos, insert);
    G = view();
  }

  phase("hub_plan");
  // ---- PMA planning
  bool rebuild = false;
  uint64_t nmw = 0;
  uint64_t Nn = N;
  const double build_d = (cfg.pma_build_density > 0 && cfg.pma_build_density < 1) ? cfg.pma_build_density : 0.375;
  bool shrink = !insert && N > (1ull << 20) && (double)t2new < 0.125 * (double)N;
  if (nov > 0 || shrink) {
    if (!speculate) plan_prefix();
    if (shrink || (double)t2new > root_d * (double)N) {
      rebuild = true;
    } else if (speculate) {  // windows already searched; their counts came with hc
      if (hc[C_ROOT]) rebuild = true;
      else nmw = hc[C_NMW];
    } else {
      // windows are selected before the root flag is read (one sync for
      // both); a root overflow discards them and rebuilds
      plan_windows(nov);
      uint64_t wc[C_COUNT];
      TRC_CUDA(cudaMemcpyAsync(wc, cnt, sizeof(wc), cudaMemcpyDeviceToHost, stream));
      sync();
      if (wc[C_ROOT]) rebuild = true;
      else nmw = wc[C_NMW];
    }
  }

  phase("pma_plan");
  // ---- rewrite set: touched vertices, window members, (rebuild) all PMA vertices
  epoch++;
  if (epoch == 0) {  // wrapped: clear the marks
    TRC_CUDA(cudaMemsetAsync(stamp.get(), 0, (uint64_t)n * 4, stream));
    TRC_CUDA(cudaMemsetAsync(wstamp.get(), 0, (uint64_t)n * 4, stream));
    epoch = 1;
  }
  uint32_t *tix = s_tix.ensure(n);
  if (nmw)
    TRC_LAUNCH(prof, stream, "upd_window_mark", nmw, 256, 0, k_window_mark2, s_mw.get(), n,
               stamp.get(), wstamp.get(), tix, epoch);
  uint64_t Ptot = 0;
  if (rebuild) {
    Ptot = read_u64(P + n);  // the layout kernel spreads exactly this many
    Nn = std::max<uint64_t>((uint64_t)std::ceil((double)Ptot / build_d), Ptot + 1);
    TRC_LAUNCH(prof, stream, "upd_mark_pma", ceil_div(n, 256), 256, 0, k_mark_pma_vertices, c2n, n,
               stamp.get(), tix, epoch);
  }
  TRC_LAUNCH(prof, stream, "upd_mark", ceil_div(nt, 256), 256, 0, k_mark_touched, tu, nt,
             stamp.get(), tix, epoch);

  // ---- new tier-2 layout (into pbeg_alt; pbeg keeps the old one until the end)
  const bool relayout = rebuild || nmw;
  uint64_t *pbeg_new = pbeg.get();
  uint32_t *dst_pma = pma.get();
  uint32_t *mov_pma = nullptr;
  if (relayout) {
    pbeg_new = pbeg_alt.ensure((uint64_t)n + 1);
    if (rebuild) {
      dst_pma = s_pma_next.alloc_exact(Nn);
      TRC_LAUNCH(prof, stream, "upd_rebuild_layout", ceil_div((uint64_t)n + 1, 256), 256, 0,
                 k_rebuild_layout, P, n, Nn, pbeg_new);
      rebuilds++;
    } else {
      TRC_CUDA(cudaMemcpyAsync(pbeg_new, pbeg.get(), ((uint64_t)n + 1) * 8,
                               cudaMemcpyDeviceToDevice, stream));
      TRC_LAUNCH(prof, stream, "upd_window_layout", nmw, 256, 0, k_window_layout, s_mw.get(), n, P,
                 pbeg_new);
      mov_pma = s_pma_next.ensure(N ? N : 1);
      window_rebalances += nmw;
    }
  }

  phase("layout");
  // ---- fused merge for every rewrite vertex that stays in tiers 1-2
  const uint32_t T = cfg.hub_threshold;
  uint32_t *rs = s_rlist.ensure(n);
  if (rebuild) {  // every PMA vertex moves: one pass over all vertices
    uint64_t *t4 = tmp(select_tmp_elems(n) + 4);
    select_if(SmallPred{stamp.get(), epoch, hub_of.get(), deg.get(), tix, tdn, T}, IndexVal32{},
              n, rs, cnt + C_NR, t4, stream, prof, "sel_rewrite");
  } else {  // touched vertices (in vertex order), then untouched window members
    uint64_t *t4 = tmp(select_tmp_elems(nt) + 4);
    select_if(TouchedSmallPred{tu, tdn, hub_of.get(), T}, TouchedVal{tu}, nt, rs, cnt + C_NR, t4,
              stream, prof, "sel_rewrite");
    if (nmw)
      TRC_LAUNCH(prof, stream, "upd_window_members", nmw, 256, 0, k_window_members, s_mw.get(), n,
                 tix, hub_of.get(), c2.get(), rs, (unsigned long long *)(cnt + C_NR));
  }
  // the rewrite list's length stays on the device (read with the final sync)
  const uint64_t *nrs_dev = cnt + C_NR;
  const unsigned pgrid = (unsigned)num_sms() * 8;  // persistent kernels, 64 warps per SM
  uint64_t nrs = 0;
  uint64_t SO = 0, SN = 0;
  if (prof.on) nrs = read_u64(cnt + C_NR);
  if (prof.on && nrs) {  // element counts for the profiler's byte accounting
    uint64_t *oo = s_oOff.ensure(nrs + 1);
    uint64_t *t5 = tmp(scan_tmp_elems(nrs) + 4);
    exclusive_scan(OldDeg{rs, deg.get()}, nrs, oo, t5, stream, prof, "prof_count");
    SO = read_u64(oo + nrs);
    exclusive_scan(NewDeg{rs, deg.get(), tix, tdn}, nrs, oo, t5, stream, prof, "prof_count");
    SN = read_u64(oo + nrs);
  }
  {
    MergeArgs ma{rs, 0, tix, tpos, nt, kb, bkeys, insert ? 1 : 0, pbeg_new, dst_pma, mov_pma,
                 nmw ? wstamp.get() : nullptr, epoch, T, dst_pma == pma.get() ? 1 : 0};
    static_assert(HUB_THRESHOLD_MAX <= MR_MASK, "merge record counts");
    ulonglong2 *rec = reinterpret_cast<ulonglong2 *>(s_mrec.ensure(2 * (uint64_t)n));
    TRC_LAUNCH(prof, stream, "upd_merge_prep", pgrid, 256, 0, k_merge_prep, G, ma, nrs_dev, rec);
    TRC_LAUNCH(prof, stream, "upd_merge_group", (unsigned)num_sms() * 4, 256, 0, k_merge_group, G,
               ma, nrs_dev, (const ulonglong2 *)rec);
    TRC_LAUNCH(prof, stream, "upd_merge_small", pgrid, 256, 0, k_merge_small, G, ma, nrs_dev,
               (const ulonglong2 *)rec, (unsigned long long *)(cnt + C_MWORK));
  }
  phase("merge_small");
  // ---- tier 3, second phase (the hubs touch vertices disjoint from the
  // small-vertex merge's; the graph's stream waits for it before the window
  // moves)
  if (nh) apply_hubs_finish();

  phase("hub_path");
  // ---- window moves land after every reader of the old segments is done
  if (nmw) {
    DevView GC = view();
    TRC_LAUNCH(prof, stream, "upd_window_copy", pgrid, 256, 0, k_window_copy, GC, rs, nrs_dev,
               mov_pma, pbeg_new, wstamp.get(), epoch);
  }
  TRC_LAUNCH(prof, stream, "upd_c2", ceil_div(nt, 256), 256, 0, k_scatter_c2_final, tu, tc2, nt,
             c2.get());
  if (relayout) pbeg.swap(pbeg_alt);
  if (rebuild) {
    pma.swap(s_pma_next);
    s_pma_next.reset();
    N = Nn;
  }
  m = insert ? m + kb : m - kb;
  if (defer_tail && !prof.on) {
    // the rewrite count lands in pinned staging (clear of the counters and
    // the error word the next batch copies there before reading it)
    TRC_CUDA(cudaMemcpyAsync(hub_stage_ + 62, nrs_dev, 8, cudaMemcpyDeviceToHost, stream));
    hub_guard.armed = false;  // apply_hubs_finish ran: only the readback is left
    tail_pending = true;
    tail_nh = nh;
    tier2_total = rebuild ? Ptot : t2new;
    last[0] = k2;
    last[1] = kb;
    last[2] = nt;
    last[3] = 0;
    last[4] = SO;
    last[5] = SN;
    last[6] = nmw;
    last[7] = rebuild ? 1 : 0;
    version++;
    return kb;
  }
  TRC_CUDA(cudaMemcpyAsync(&nrs, nrs_dev, 8, cudaMemcpyDeviceToHost, stream));
  sync();  // host vectors (the hub records) outlive their copies
  phase("finish");
  hubs_finish();
  const uint64_t nr = nrs + nh;
  SO += hub_last[4];
  SN += hub_last[5];
  tier2_total = rebuild ? Ptot : t2new;
  last[0] = k2;
  last[1] = kb;
  last[2] = nt;
  last[3] = nr;
  last[4] = SO;
  last[5] = SN;
  last[6] = nmw;
  last[7] = rebuild ? 1 : 0;
  version++;
  return kb;
}

}  // namespace trc
