// graph.cuh -- the device-resident three-tier graph (host-side owner of the
// HBM state) and the declarations of its update, query and analytics paths.
#pragma once

#include <vector>

#include "prims.cuh"

namespace trc {

constexpr uint64_t KEY_INVALID = ~0ull;

// Device address of the no-allocation BFS's static scratch array on the
// current device (noalloc.cu).
uint32_t *noalloc_scratch_resolve();

// Lookup of (u, x) in the tiers (used by the update filter and is_edge).
// Is (u, x) an edge?  The inline row is read whole (up to four 16-byte
// loads issued together) and compared at once; only an x above its last
// element searches the rest of the list (the PMA segment, or the hub's
// blocks through the directory).
__device__ __forceinline__ bool has_edge(const DevView &G, uint32_t u, uint32_t x) {
  const uint32_t d = G.deg[u];
  if (d == 0) return false;
  const NbrList L = nbr_list(G, u);
  const uint4 *row = reinterpret_cast<const uint4 *>(L.inl);
  uint32_t v[K_INLINE];
#pragma unroll
  for (uint32_t q = 0; q < K_INLINE / 4; q++) {
    const uint4 t = q * 4 < L.ni ? row[q] : make_uint4(0, 0, 0, 0);
    v[4 * q] = t.x;
    v[4 * q + 1] = t.y;
    v[4 * q + 2] = t.z;
    v[4 * q + 3] = t.w;
  }
  bool found = false;
  uint32_t last = 0;
#pragma unroll
  for (uint32_t e = 0; e < K_INLINE; e++) {
    if (e < L.ni) found |= v[e] == x;
    if (e + 1 == L.ni) last = v[e];
  }
  if (found) return true;
  if (L.ni == L.deg || x < last) return false;
  if (L.nb == 0) {  // the PMA segment, rest elements
    uint32_t lo = 0, hi = L.rest;
    while (lo < hi) {
      const uint32_t mid = (lo + hi) >> 1;
      const uint32_t y = L.seg[mid];
      if (y < x) lo = mid + 1;
      else if (y > x) hi = mid;
      else return true;
    }
    return false;
  }
  return list_has(L, x);  // (a hub: x is above the inline row, so a block search)
}

// Per-vertex class lists for the analytics kernels, rebuilt when the graph
// version changes: S = 1..16 neighbours (inline only), M = more than 16 and
// not a hub (inline + PMA segment), H = hubs, SM = S and M; M1 / M2 = M up
// to / above PageRank's lane-group cut.
struct ClassLists {
  uint64_t version = ~0ull;
  DBuf<uint32_t> S, M, Hv, SM, M1, M2;
  uint64_t nS = 0, nM = 0, nH = 0, nSM = 0, nM1 = 0, nM2 = 0;
};

// Tier-3 work of one batch between its two launch phases (hubs.cu).
struct HubItem {
  uint64_t i;  // index in the batch's touched-hub records
  uint32_t h;  // hub index
};
struct HubCtx {
  bool active = false, readback = false, insert = false;
  uint32_t fill = 192;
  uint64_t NL = 0, QL = 0, F = 0, fresh0 = 0, R = 0;
  std::vector<HubItem> loc, rw;
  std::vector<uint64_t> lp;
  uint64_t *d_lp = nullptr;
  uint32_t *lli = nullptr, *lg = nullptr, *lx = nullptr, *tgq = nullptr, *tgo = nullptr;
  uint32_t *tgb = nullptr, *hflag = nullptr, *stage = nullptr, *freed = nullptr, *pin = nullptr;
  int32_t *hnbd = nullptr;
  const uint32_t *hw_t = nullptr;
  const uint64_t *bkeys = nullptr, *tpos = nullptr;
  const std::vector<uint32_t> *hu = nullptr, *hdn = nullptr, *hdo = nullptr;
};

class Graph {
 public:
  Graph(uint32_t n, uint64_t budget_bytes, const trc_config &cfg);
  ~Graph();

  // ------------------------------------------------------------- state
  uint32_t n;
  trc_config cfg;
  cudaStream_t stream = nullptr;
  cudaStream_t own_stream = nullptr;
  cudaStream_t side_stream = nullptr;  // hub merge, concurrent with the small-vertex merge
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  // A host batch's H2D copy, issued while the previous batch's trailing
  // kernels (merges, window moves) still run on the graph's stream
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t ev_h2d = nullptr;
  Budget budget;
  Profiler prof;

  DBuf<uint32_t> deg, inl, c2, pma, err;
  DBuf<uint64_t> pbeg;
  DBuf<int32_t> hub_of;
  // tier 3 (hubs.cu): hub tables (device) and their host mirrors
  DBuf<uint32_t> hub_vtx, hub_nblk;
  DBuf<uint64_t> hub_dir0;
  std::vector<uint32_t> h_hub_vtx, h_hub_nblk, h_hub_dcap;
  std::vector<uint64_t> h_hub_dbase;  // the hub's directory region: two halves of dcap entries
  std::vector<uint8_t> h_hub_dside;   // the half in use
  uint32_t H = 0;
  // directory pool (entries: block id, elements before the block, first key)
  DBuf<uint32_t> hdir, hpre, hkey;
  uint64_t DP = 0, dir_top = 0;
  // block pool, and the ids of free blocks
  DBuf<uint32_t> hslot, bcnt, bmin, bown;
  DBuf<uint32_t> bfree, bfreed;
  uint64_t NBP = 0;       // pool capacity in blocks
  uint64_t pool_top = 0;  // blocks ever handed out
  uint64_t nfree = 0;     // entries of bfree
  // per-batch statistics of the blocked tier
  uint64_t hub_last[6] = {0, 0, 0, 0, 0, 0};  // touched, local, rewritten, blocks written,
                                              // elements read, elements written
  uint64_t hub_splits = 0, hub_absorbs = 0, hub_rewrites = 0;
  // tier-3 scratch
  DBuf<uint32_t> s_lg, s_lx, s_lli, s_tgq, s_tgo, s_tgb, s_hflag, s_rwstage;
  DBuf<int32_t> s_hnbd;
  DBuf<uint64_t> s_hplan, s_hsel;
  HubCtx hub_ctx_;
  cudaEvent_t ev_hub = nullptr;  // the block-local group counts are on the host

  uint64_t N = 0;          // tier-2 capacity (slots)
  uint64_t m = 0;          // directed edges
  uint64_t tier2_total = 0;
  uint64_t version = 0;
  uint32_t epoch = 0;
  DBuf<uint32_t> stamp;    // per-vertex epoch marks for the rewrite set
  DBuf<uint32_t> wstamp;   // per-vertex epoch marks for rebalanced windows
  DBuf<uint64_t> pbeg_alt; // next tier-2 layout while a batch is applied
  uint64_t rebuilds = 0, window_rebalances = 0;
  uint64_t last[8] = {0, 0, 0, 0, 0, 0, 0, 0};  // sizes of the last batch
  SortWait sort_wait;  // bounded look-back wait of the batch sort (test hook)
  int sort_mode = 0;   // batch sort: 0 by size, 1 radix only, 2 bucket first (test hook)
  DBuf<uint32_t> bsplits;  // bucket sort: source quantiles of the last large batch
  bool bsplits_ok = false;
  uint64_t sort_retries = 0;  // batches the bucket sort handed back to the radix sort

  // ------------------------------------------------------------- scratch
  DBuf<uint32_t> s_in_src, s_in_dst;
  DBuf<uint64_t> s_A, s_B, s_C, s_tmp, s_cnt;
  DBuf<uint64_t> s_mrec;  // merge records, two words per rewrite entry
  DBuf<uint32_t> s_tu, s_tdn, s_tc2, s_ovl, s_hw_u, s_hw_dn, s_hw_t, s_c2n, s_rlist;
  DBuf<int32_t> s_hw_h;
  DBuf<uint64_t> s_P, s_oOff, s_nOff, s_wk, s_wk2, s_mw, s_old, s_new, s_hwplan;
  DBuf<uint8_t> s_flags;
  DBuf<uint32_t> s_pma_next;
  DBuf<uint32_t> s_tix;  // vertex -> index in the touched list (this batch)
  DBuf<uint32_t> s_wbits;  // per-level PMA window bitmaps (this batch)
  DBuf<uint32_t> s_hw_do;  // old degree of each touched hub
  ClassLists lists;

  DevView view() const;
  uint32_t vbits() const;
  void release_scratch();

  // ------------------------------------------------------------- update
  // Applies a batch; returns the number of directed edges changed.
  // With defer_tail the call returns after launching the batch's last
  // kernels: the graph's stream orders every later device use, and
  // complete_pending() (or the next batch, after its first synchronisation)
  // does the host bookkeeping that reads their results.
  uint64_t apply_batch(const uint32_t *src, const uint32_t *dst, uint64_t k, uint32_t flags,
                       bool insert, bool defer_tail = false);
  // Waits for a deferred batch tail and finishes it (no-op without one).
  void complete_pending();
  bool tail_pending = false;
  uint64_t tail_nh = 0;  // the pending batch's touched hubs (its rewrite count)

  // ------------------------------------------------------------- queries
  void is_edge(const uint32_t *src, const uint32_t *dst, uint64_t q, uint8_t *out, uint32_t flags);
  void degree(const uint32_t *v, uint64_t q, uint32_t *out, uint32_t flags);
  uint64_t neighbors(uint32_t v, uint32_t *out, uint64_t cap, uint32_t flags);
  void count_common(const uint32_t *s, const uint32_t *d, uint64_t q, uint32_t *out,
                    uint32_t flags);
  void dump_csr(uint64_t *offsets, uint32_t *targets, uint32_t flags);
  // graph files (io.cu): parse AdjacencyGraph text with m edges and insert
  // them; insert a host CSR; the graph as AdjacencyGraph text
  void load_adj(const uint8_t *bytes, uint64_t len, uint64_t m_file, uint32_t flags);
  void load_csr(const uint64_t *offsets, const uint32_t *targets, uint64_t m_file, uint32_t flags);
  std::vector<uint8_t> format_adj();
  uint64_t check();
  uint64_t size_bytes() const;
  void stats(trc_stats *out);

  // ------------------------------------------------------------- analytics
  void ensure_lists();
  void bfs(uint32_t src, int32_t *parents, uint32_t *levels, uint32_t flags);
  // up to 64 BFS at once, levels[i*n + v] (msbfs.cu)
  void msbfs(const uint32_t *sources, uint32_t k, uint32_t *levels, uint32_t flags);
  // per source: vertices reached and deepest level, without level arrays
  void msbfs_summary(const uint32_t *sources, uint32_t k, uint64_t *reached, uint32_t *ecc);
  void msbfs_run(const uint32_t *sources, uint32_t k, uint32_t *levels, uint32_t flags,
                 uint64_t *reached, uint32_t *ecc);
  // up to 64 BC at once, out[i*n + v] (msbfs.cu)
  void msbc(const uint32_t *sources, uint32_t k, double *out, uint32_t flags);
  // Edge-balanced pushes: the frontier F's lists cut into list_piece()s;
  // returns off[0..nf] = the exclusive prefix of their piece counts (off[nf]
  // = the total), in pb's buffers (analytics.cu)
  struct PieceBufs {
    DBuf<uint32_t> cnt;
    DBuf<uint64_t> off, scan;
    explicit PieceBufs(Budget *b) {
      cnt.bind(b);
      off.bind(b);
      scan.bind(b);
    }
  };
  const uint64_t *piece_offsets(const uint32_t *F, uint32_t nf, PieceBufs &pb, const char *tag,
                                bool skip_small = false);
  void ms_init(uint32_t k, const uint32_t *dsrc, uint64_t *seen, uint64_t *front, uint64_t *next,
               uint32_t *lvrow, unsigned long long *acc);
  // one edge-balanced push level of msbfs / msbc (msbfs.cu)
  void ms_push_level(const uint32_t *F, uint32_t nf, const uint64_t *front, const uint64_t *seen,
                     unsigned long long *acc, uint32_t *T, uint32_t *tcnt, PieceBufs &pb);
  // BFS with scratch in a static device array (no allocation), noalloc.cu
  void bfs_noalloc(uint32_t src, int32_t *parents, uint32_t *levels, uint32_t flags);
  uint32_t *na_scratch = nullptr;  // that array's device address on this graph's device
  int device = 0;  // device the graph was created on
  void pagerank(uint32_t iters, double damping, double *ranks, uint32_t flags);
  // the iterations on stream s into caller buffers (n each); class lists
  // must be current; no allocation or synchronisation
  void pagerank_launch(uint32_t iters, double damping, double *p0, double *p1, double *out,
                       cudaStream_t s);
  void pr_kernels(uint32_t iters, double damping, double *p0, double *p1, double *out,
                  cudaStream_t s);
  struct PRGraphCache {
    static constexpr int KEY = 13;
    cudaGraphExec_t exec = nullptr;
    uint64_t key[KEY] = {};
    uint64_t kernels = 0;       // kernel nodes per replay
    uint64_t replays = 0, replays_built = 0;
  } prg;
  bool use_graphs = true;     // CUDA-graph replay of iteration loops
  void cc(uint32_t *labels, uint32_t flags);
  void bc(uint32_t src, double *dep, uint32_t flags);
  uint64_t tc();

  // helpers
  // Host wall time since the previous phase mark, accumulated under
  // "host:<name>" while profiling (shows syncs and host work per phase).
  void phase(const char *name);
  double phase_t0 = 0.0;
  uint64_t read_u64(const uint64_t *dptr);
  void sync();
  uint32_t push_pull_divisor() const { return tuned.push_pull_divisor; }

  // per-graph choices (config defaults, changed by trc_autotune / trc_set_tuning)
  struct Tuning {
    uint32_t push_pull_divisor = 20;  // dense traversal when |F| >= n / divisor
    uint32_t pr_group_cut = 64;       // PageRank: degree 17..cut use a lane group
    uint32_t pr_group_lanes = 8;      // ... of this many lanes (4, 8 or 16); above: a warp
    uint32_t pma_leaf_log = 1;        // smallest PMA window: 2^x vertex segments
  } tuned;
  void autotune(uint32_t what, const uint32_t *src, const uint32_t *dst, uint64_t k,
                uint32_t flags, double *ms_out);

 private:
  void grow_hub_tables(uint32_t need);
  // pinned staging for the classify counts and the touched hubs' records
  static constexpr uint64_t HUB_SPEC = 4096;
  uint32_t *hub_stage_ = nullptr;
  void grow_pool(uint64_t need_blocks);
  uint64_t *tmp(uint64_t elems) { return s_tmp.ensure(elems); }
  void grow_dir_pool(uint64_t need);
  uint32_t *hub_pin_ = nullptr;  // pinned staging of the tier-3 counts
  uint64_t hub_pin_cap_ = 0;
  uint32_t *hub_pin(uint64_t words);
  uint64_t hub_dir_target(uint32_t h, uint32_t nb);

 public:
  // Tier-3 part of a batch (hubs.cu) on side_stream, in two launch phases
  // around the small-vertex merge: apply_hubs takes the touched hubs' host
  // records (vertex, new degree, hub index or -1, old degree), their device
  // touched indices (hw_t, for each hub's slice of the sorted batch) and
  // launches the block-local location and counting; apply_hubs_finish reads
  // those counts, plans, launches the merges and rewrites and makes the
  // graph's stream wait for them.  The host records must outlive both.
  void apply_hubs(uint64_t nh, const std::vector<uint32_t> &hu, const std::vector<uint32_t> &hdn,
                  const std::vector<int32_t> &hh, const std::vector<uint32_t> &hdo,
                  const uint32_t *hw_t, const uint64_t *bkeys, const uint64_t *tpos, bool insert);
  void apply_hubs_finish();
  void hubs_finish();  // after the batch's final synchronisation
  void finish_tail();  // host part of complete_pending, the stream already synchronised
  void hub_init();
};

// Copies between user buffers and device scratch, honouring TRC_DEVICE_PTR.
template <typename T>
const T *to_device(Graph &g, const T *p, uint64_t count, uint32_t flags, DBuf<T> &stage) {
  if (flags & TRC_DEVICE_PTR) return p;
  T *d = stage.ensure(count ? count : 1);
  if (count) TRC_CUDA(cudaMemcpyAsync(d, p, count * sizeof(T), cudaMemcpyHostToDevice, g.stream));
  return d;
}

}  // namespace trc
