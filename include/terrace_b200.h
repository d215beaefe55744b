/*
 * terrace_b200.h -- C ABI of the B200-native Terrace dynamic-graph hot path.
 *
 * Plain C: opaque handles, plain pointers and sizes, status codes.  No CUDA
 * or torch types appear here; a CUDA stream is passed as `void*`
 * (cudaStream_t).  Every entry point is synchronous: it returns after the
 * device work it launched has finished, except that a batch update returns
 * with its last kernels still queued on the handle's stream (every other
 * entry point waits for them first).  Host buffers may be reused as soon as
 * any call returns.  Unless TRC_DEVICE_PTR is set in `flags`, array arguments are HOST
 * pointers and the library copies them to and from the device itself.
 *
 * Each declaration names the reference interface it replaces
 * (PASSIONLab/terrace, paths inside that tree).  The reference is a
 * header-only C++ library (graphstore::Graph in include/graph.h); this ABI is
 * the flat layer a C++ facade (terrace_b200.hpp) or an FFI binds.
 */
#ifndef TERRACE_B200_H_
#define TERRACE_B200_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct trc_graph trc_graph;

/* Status codes.  The reference exits or aborts on fatal errors
 * (src/PMA.cc:2308-2316, include/io_util.h:117-131) and returns -1/0 from
 * single-edge calls (include/graph.h:505-641, :675-791); here every call
 * returns one of these and trc_last_error() holds a message. */
typedef enum {
  TRC_OK = 0,
  TRC_ERR_INVALID = 1, /* bad argument: null pointer, vertex id >= n, ... */
  TRC_ERR_NOMEM = 2,   /* HBM budget or device allocation exhausted */
  TRC_ERR_CUDA = 3,    /* a CUDA call failed (message has the CUDA error) */
  TRC_ERR_TIMEOUT = 4, /* a bounded device wait ran out (serving loop) */
  TRC_ERR_STATE = 5,   /* call not valid in the handle's current state */
  TRC_ERR_NOT_BUILT = 6, /* the sm_100a kernels are not available */
  TRC_ERR_IO = 7         /* a file could not be opened, read or written */
} trc_status;

/* flags */
#define TRC_DEVICE_PTR 0x1u      /* array arguments are device pointers */
#define TRC_SYMMETRIZE 0x2u      /* apply (u,v) and (v,u) for every pair */
#define TRC_DROP_SELF_LOOPS 0x4u /* ignore pairs with u == v */

#define TRC_UNREACHED 0xFFFFFFFFu /* BFS level of an unreached vertex */

/* Tunables.  Defaults mirror the reference's constants where one exists. */
typedef struct {
  uint32_t hub_threshold;     /* degree above which a vertex moves to the
                                 blocked tier; reference MEDIUM_DEGREE 1024
                                 (include/graph.h:39).  Default 1024; at
                                 most 12288 (a PMA vertex's list is staged
                                 in 48 KB of shared memory when merged). */
  double pma_root_density;    /* upper density bound at the PMA root;
                                 reference 0.75 (src/PMA.cc:382-394). */
  double pma_build_density;   /* density after a full PMA rebuild.  Default
                                 0.375: the reference doubles its array when
                                 the root passes 0.75 (double_list,
                                 src/PMA.cc:659-720). */
  double hub_block_fill;      /* fill of hub blocks after a rewrite or a
                                 split.  Default 0.75. */
  uint32_t push_pull_divisor; /* edgeMap goes dense when |F| >= n/divisor;
                                 reference threshold 20 (include/Map.cpp:65-74).
                                 0 = the autotuned value (default 20). */
  uint32_t hub_stage_limit;   /* most batch edges one hub block merges in
                                 shared memory (capped at 4096); a block
                                 receiving more sends its hub through a
                                 whole-list rewrite.  Default 49152 (the
                                 cap applies). */
  uint32_t cuda_graphs;       /* 1: iteration loops (PageRank) are replayed
                                 from captured CUDA graphs; 0: launched one
                                 by one.  Default 1. */
} trc_config;

/* Fill `cfg` with the defaults listed above. */
void trc_config_default(trc_config *cfg);

const char *trc_status_string(trc_status s);
/* Message of the last failing call on this host thread ("" if none). */
const char *trc_last_error(void);

/* ---- lifetime: replaces graphstore::Graph::Graph(uint32_t) / ~Graph
 *      (include/graph.h:232-239).  hbm_budget_bytes caps the device memory
 *      the handle may hold (0 = no cap beyond the device's free memory). */
trc_status trc_graph_create(uint32_t n, uint64_t hbm_budget_bytes,
                            const trc_config *cfg, trc_graph **out);
trc_status trc_graph_destroy(trc_graph *g);
/* Bind the handle to a CUDA stream (cudaStream_t); NULL = the handle's own
 * stream (so is handle 0, the legacy default stream: bind another stream to
 * order the handle's work with work on it).
 * Batch updates also run their hub merge on a second stream owned by the
 * handle, forked from and joined back to the bound stream with events, so
 * every call's work stays ordered after earlier work on the bound stream. */
trc_status trc_graph_set_stream(trc_graph *g, void *stream);

/* Frees the temporary device buffers kept between calls (sort buffers,
 * merge staging, frontier lists); the next call that needs them allocates
 * them again.  Useful after a bulk load.  No reference counterpart (the
 * reference frees its temporaries per call). */
trc_status trc_release_scratch(trc_graph *g);

/* Test hook for the bounded device wait of the batch sort: the radix sort's
 * scatter passes wait for earlier tiles' counts (decoupled look-back) and
 * give up after spin_limit polls, failing the call with TRC_ERR_TIMEOUT
 * before the graph is modified.  withhold_first_tile != 0 makes no tile 0
 * publish, so every such wait runs out (a flag that nothing sets); 0/0
 * restores the defaults (spin_limit 0 = 2^22 polls).  No reference
 * counterpart (the reference has no device waits). */
trc_status trc_debug_sort_wait(trc_graph *g, uint32_t spin_limit,
                               int withhold_first_tile);

/* Test hook for the choice of batch sort.  Batches of 4,096 to 2^24 keys
 * (after symmetrizing) sort with a bucket sort (buckets are source ranges
 * whose split points are the source quantiles of the previous large batch,
 * or source >> shift before there was one; each bucket sorted whole in
 * registers or shared memory); a batch in which one bucket holds more than
 * 16384 keys is sorted again by the LSD radix sort before anything is
 * modified (trc_stats.sort_retries counts these); batches of at most 2048
 * keys sort in one CTA (a bitonic network in shared memory); other batches,
 * and all batches while the wait hook above is set, use the radix sort.  mode 0
 * restores that choice, 1 forces the radix sort, 2 tries the bucket sort
 * for every batch.  Results are identical.
 * No reference counterpart (the reference's driver sorts each batch with
 * two stable integer sorts, by destination then by source, before the
 * update call: src/graph_bm.cc:354-355). */
trc_status trc_debug_sort_mode(trc_graph *g, int mode);

/* ---- updates: replaces Graph::add_edge_batch (include/graph.h:430-502) and
 *      the per-edge Graph::remove_edge loop of src/graph_bm.cc:375-380 (the
 *      reference declares no remove_edge_batch, include/graph.h:143-150).
 *      Set semantics: duplicates, already-present edges (insert) and absent
 *      edges (remove) are ignored; input need not be sorted and is never
 *      modified.  *applied (may be NULL) receives the number of directed
 *      edges actually inserted / removed.
 *      The call returns once the batch's last kernels (the list merges and
 *      segment moves) are queued on the handle's stream; src and dst may be
 *      reused or freed at once.  Every other entry point on the handle first
 *      waits for those kernels; the next batch call does not, and copies its
 *      host arrays to the device on a second stream while they run. */
trc_status trc_add_edge_batch(trc_graph *g, const uint32_t *src,
                              const uint32_t *dst, uint64_t k, uint32_t flags,
                              uint64_t *applied);
trc_status trc_remove_edge_batch(trc_graph *g, const uint32_t *src,
                                 const uint32_t *dst, uint64_t k,
                                 uint32_t flags, uint64_t *applied);

/* ---- queries: replaces Graph::is_edge, Graph::degree, the NeighborIterator
 *      and Graph::count_common (include/graph.h:643-673, :797-803, :844-899,
 *      :1085-1255), batched over q queries. */
trc_status trc_is_edge(trc_graph *g, const uint32_t *src, const uint32_t *dst,
                       uint64_t q, uint8_t *out, uint32_t flags);
trc_status trc_degree(trc_graph *g, const uint32_t *v, uint64_t q,
                      uint32_t *out, uint32_t flags);
/* Sorted neighbours of v into out[0..cap); *len = degree(v) (may exceed cap,
 * in which case only cap entries are written). */
trc_status trc_neighbors(trc_graph *g, uint32_t v, uint32_t *out, uint64_t cap,
                         uint64_t *len, uint32_t flags);
/* out[i] = |{w in N(s[i]) n N(d[i]) : w < min(s[i],d[i])}| */
trc_status trc_count_common(trc_graph *g, const uint32_t *s, const uint32_t *d,
                            uint64_t q, uint32_t *out, uint32_t flags);
/* Graph::get_num_vertices / get_num_edges / get_size (include/graph.h:805-822) */
trc_status trc_num_vertices(trc_graph *g, uint32_t *n);
trc_status trc_num_edges(trc_graph *g, uint64_t *m);
trc_status trc_get_size(trc_graph *g, uint64_t *bytes);
/* Whole graph as sorted CSR: offsets[n+1], targets[num_edges]. */
trc_status trc_dump_csr(trc_graph *g, uint64_t *offsets, uint32_t *targets,
                        uint32_t flags);

/* ---- graph files: replaces get_edges_from_file_adj_sym (include/io_util.h:
 *      112-145) and the load in src/graph_bm.cc:262-266.  The AdjacencyGraph
 *      text file ("AdjacencyGraph", n, m, n offsets, m targets; vertex i's
 *      edges are targets [offsets[i], offsets[i+1]), the last ending at m) is
 *      parsed on the GPU and its edges inserted as one batch (flags:
 *      TRC_SYMMETRIZE / TRC_DROP_SELF_LOOPS apply to them; the reference
 *      inserts them as given).  TRC_ERR_INVALID for a malformed file
 *      (missing header, wrong word count, a non-number, offsets that do not
 *      rise from 0, a target >= n), TRC_ERR_IO if it cannot be read.
 *      The binary CSR file: "TRCCSR01", n and m (u64), offsets[n+1] (u64),
 *      targets[m] (u32), little-endian. */
trc_status trc_graph_load_adj(const char *path, uint64_t hbm_budget_bytes,
                              const trc_config *cfg, uint32_t flags, trc_graph **out);
/* Writes the graph as an AdjacencyGraph file (sorted lists), formatted on
 * the GPU. */
trc_status trc_graph_save_adj(trc_graph *g, const char *path);
trc_status trc_graph_load_csr(const char *path, uint64_t hbm_budget_bytes,
                              const trc_config *cfg, uint32_t flags, trc_graph **out);
trc_status trc_graph_save_csr(trc_graph *g, const char *path);

/* ---- analytics: replaces BFS_with_edge_map (include/BFS.h:41-84),
 *      PR_S<double> (include/Pagerank.h:105-184), CC (include/Components.h:
 *      92-120), BC (include/BC.h:99-157) and TC (include/TC.h:73-87). */
/* parents: -1 unreached, parents[src]=src; levels (may be NULL):
 * TRC_UNREACHED for unreached vertices. */
trc_status trc_bfs(trc_graph *g, uint32_t src, int32_t *parents,
                   uint32_t *levels, uint32_t flags);
/* Multi-source BFS: k <= 64 sources traversed together, one bit per source
 * in a 64-bit mask per vertex (the reference runs BFS_with_edge_map once per
 * source).  levels[i*n + v] = BFS level of v from sources[i], TRC_UNREACHED
 * if unreached; identical to trc_bfs's levels for each source. */
trc_status trc_msbfs(trc_graph *g, const uint32_t *sources, uint32_t k,
                     uint32_t *levels, uint32_t flags);
/* damping == 0 reproduces the reference (no damping term); 0 < damping < 1
 * computes p' = (1-damping)/n + damping * sum. FP64. */
trc_status trc_pagerank(trc_graph *g, uint32_t iters, double damping,
                        double *ranks, uint32_t flags);
/* labels[v] = smallest vertex id in v's component (symmetric graphs). */
trc_status trc_cc(trc_graph *g, uint32_t *labels, uint32_t flags);
/* Dependencies as the reference returns them; NaN for unreached vertices. */
trc_status trc_bc(trc_graph *g, uint32_t src, double *dep, uint32_t flags);
/* Multi-source BC: k <= 64 sources in one traversal (one bit per source in a
 * 64-bit mask per vertex; the reference runs BC once per source,
 * include/BC.h:99-157).  dep[i*n + v] = trc_bc(sources[i])'s value for v
 * (FP64 sums in the reference's neighbour order; NaN where unreached).
 * Device memory: 16 * k * n bytes for path counts and dependencies. */
trc_status trc_msbc(trc_graph *g, const uint32_t *sources, uint32_t k, double *dep,
                    uint32_t flags);
trc_status trc_tc(trc_graph *g, uint64_t *count);

/* ---- BFS without device allocation.  No counterpart in the reference.
 *      For callers that cannot call cudaMalloc when they traverse: a service
 *      whose device memory is fixed at start-up, an embedding whose
 *      allocator belongs to another component, or a request path that must
 *      not allocate.  Same results as trc_bfs (levels exact, parents a valid
 *      BFS tree), computed with push steps only.  Its scratch (two frontier
 *      queues and a counter, 8 MiB + 256 B) is a static device array: it is
 *      reserved on a GPU, and its device address looked up, when the first
 *      graph is created there (trc_graph_create), and held until exit.  Outputs must be device arrays (TRC_DEVICE_PTR); the
 *      graph may have at most TRC_NOALLOC_MAX_VERTICES vertices
 *      (TRC_ERR_INVALID otherwise).  All calls share the scratch: calls that
 *      overlap on the GPU race. */
#define TRC_NOALLOC_MAX_VERTICES 1048576u
trc_status trc_bfs_noalloc(trc_graph *g, uint32_t src, int32_t *parents,
                           uint32_t *levels, uint32_t flags);

/* ---- device view for user kernels (terrace_b200_edge_map.cuh): raw device
 *      pointers of the tiers, valid until the next update of the graph.  No
 *      reference counterpart (the reference's functors run inside
 *      Graph::map_* on the host, include/graph.h:1287-1613).  Neighbour r of
 *      u: r < min(deg,16): inl[16u + r]; otherwise r' = r - 16 and, when
 *      hub_of[u] < 0, pma[pbeg[u] + r'], else with h = hub_of[u] and
 *      e = hub_dir0[h] + i for the largest i < hub_nblk[h] with
 *      hub_pre[hub_dir0[h] + i] <= r': hslot[hub_dir[e] * hub_block + r' -
 *      hub_pre[e]].  hub_key[e] is the first neighbour in that block (the
 *      directory of a hub is sorted by it). */
typedef struct {
  uint32_t n;
  uint32_t inline_slots; /* 16 */
  uint32_t hub_block;    /* 256 */
  const uint32_t *deg;
  const uint32_t *inl;
  const uint64_t *pbeg;
  const uint32_t *pma;
  const int32_t *hub_of;
  const uint64_t *hub_dir0;
  const uint32_t *hub_nblk;
  const uint32_t *hub_dir;
  const uint32_t *hub_pre;
  const uint32_t *hub_key;
  const uint32_t *hslot;
  void *stream; /* the handle's cudaStream_t */
} trc_device_view;
trc_status trc_get_device_view(trc_graph *g, trc_device_view *out);

/* ---- generator: replaces rMat<uint32_t> (include/rmat_util.h:81-115),
 *      bit-exact, edges first..first+count-1, on the device. */
trc_status trc_rmat_generate(uint32_t n, uint32_t seed, double a, double b,
                             double c, uint64_t first, uint64_t count,
                             uint32_t *src, uint32_t *dst, uint32_t flags,
                             void *stream);

/* ---- autotuner (no reference counterpart: the reference fixes these at
 *      compile time or as constants: the edgeMap threshold 20,
 *      include/Map.cpp:65-74; PMA leaf sizing, src/PMA.cc:2961-2962).
 *      trc_autotune times candidates on this graph and keeps the fastest;
 *      later calls use them.  BFS levels and adjacency stay exact; PageRank
 *      stays within FP64 reordering (1e-9 relative). */
#define TRC_TUNE_PUSH_PULL 1u /* direction threshold: BFS from 4 sources */
#define TRC_TUNE_PAGERANK 2u  /* PageRank lanes per vertex and degree cut */
#define TRC_TUNE_PMA 4u       /* PMA leaf: insert + remove of the sample's
                                 absent edges (the edge set is unchanged) */
typedef struct {
  uint32_t push_pull_divisor; /* dense when |F| >= n / divisor */
  uint32_t pr_group_cut;      /* PageRank: degrees 17..cut use a lane group */
  uint32_t pr_group_lanes;    /* lanes per vertex in that group: 4, 8, 16 */
  uint32_t pma_leaf_log;      /* smallest PMA window: 2^x vertex segments */
  double bfs_ms;              /* best time per BFS (0 if not tuned) */
  double pagerank_iter_ms;    /* best time per PageRank iteration */
  double pma_insert_ms;       /* best insert time of the sample */
} trc_tuning;
/* `what`: TRC_TUNE_* bits.  The sample (src, dst, k; flags TRC_DEVICE_PTR
 * and TRC_SYMMETRIZE apply) is needed by TRC_TUNE_PMA only. */
trc_status trc_autotune(trc_graph *g, uint32_t what, const uint32_t *src, const uint32_t *dst,
                        uint64_t k, uint32_t flags, trc_tuning *out);
trc_status trc_get_tuning(trc_graph *g, trc_tuning *out);
/* Applies saved choices (validated: divisor >= 1, lanes 4/8/16, cut 17..4096,
 * leaf 1..20). */
trc_status trc_set_tuning(trc_graph *g, const trc_tuning *in);

/* ---- serving layer (no reference counterpart: the reference has no serving
 *      mode and forbids updates concurrent with analytics, include/graph.h:
 *      73-230).  A persistent worker thread serves requests on the graph in
 *      rounds.  TRC_SERVE_BATCHED (continuous batching): a round takes every
 *      pending request, runs its queries on the current snapshot (BFS packed
 *      64 per multi-source launch, degree lookups in one launch, PageRank
 *      shared per iteration count), then applies all its updates as one net
 *      change (the last request touching an edge decides).  Requests that
 *      arrive meanwhile join the next round.  TRC_SERVE_FIFO: one request per
 *      round in arrival order (the plain path).  Each request records the
 *      snapshot version it observed (queries) or produced (updates).  While a
 *      server runs, the graph must not be used directly. */
typedef struct trc_server trc_server;
typedef enum {
  TRC_REQ_INSERT = 0,    /* a = src, b = dst, k pairs; result: u64 directed
                            edges inserted by the request's round (FIFO:
                            by the request) */
  TRC_REQ_DELETE = 1,    /* same, removed */
  TRC_REQ_BFS = 2,       /* param = source; result: u32 levels[n] (FULL) or
                            {reached, eccentricity} (SUMMARY) */
  TRC_REQ_DEGREE = 3,    /* a = vertices, k; result: u32 degrees[k] */
  TRC_REQ_NEIGHBORS = 4, /* param = vertex; result: sorted u32 neighbours */
  TRC_REQ_PAGERANK = 5   /* param = iterations; result: f64 ranks[n] (FULL)
                            or {sum, max} (SUMMARY); undamped as PR_S */
} trc_request_kind;
#define TRC_SERVE_FIFO 0u
#define TRC_SERVE_BATCHED 1u
#define TRC_RESULT_FULL 0u
#define TRC_RESULT_SUMMARY 1u
typedef struct {
  uint32_t mode;            /* TRC_SERVE_BATCHED or TRC_SERVE_FIFO */
  uint32_t result_mode;     /* TRC_RESULT_FULL or TRC_RESULT_SUMMARY */
  uint32_t symmetrize;      /* updates apply (u,v) and (v,u) */
  uint32_t max_bfs_group;   /* sources per multi-source BFS launch (<= 64) */
  uint64_t max_round_edges; /* update admission per round (directed keys) */
} trc_server_config;
typedef struct {
  uint64_t completed;
  double elapsed_s;     /* first submit (or reset) to last completion */
  double p50_ms, p99_ms, mean_ms, max_ms; /* completion - arrival */
  uint64_t rounds;
  uint64_t device_calls;
  uint64_t rejected;    /* updates refused by the HBM budget */
  uint64_t version;     /* snapshots produced so far */
  /* the slowest round: duration, its parts, requests, full PMA rebuilds */
  double worst_round_ms, worst_update_ms, worst_bfs_ms, worst_pagerank_ms;
  uint64_t worst_round_requests, worst_round_rebuilds;
  uint64_t pma_rebuilds; /* full tier-2 rebuilds caused by served updates */
} trc_server_stats;
void trc_server_config_default(trc_server_config *cfg);
trc_status trc_server_create(trc_graph *g, const trc_server_config *cfg, trc_server **out);
/* Drains every pending request, then stops the worker. */
trc_status trc_server_destroy(trc_server *s);
/* Copies the inputs; the arrival time is the call time. */
trc_status trc_server_submit(trc_server *s, trc_request_kind kind, const uint32_t *a,
                             const uint32_t *b, uint64_t k, uint32_t param, uint64_t *id);
/* TRC_ERR_TIMEOUT if the request is not done within timeout_ms (< 0: wait). */
trc_status trc_server_wait(trc_server *s, uint64_t id, int64_t timeout_ms);
/* Copies up to cap bytes of the result; *bytes = full size; *latency_ms =
 * completion - arrival; *version = snapshot; *status = the request's own
 * status (e.g. TRC_ERR_INVALID for a bad vertex id). */
trc_status trc_server_result(trc_server *s, uint64_t id, void *out, uint64_t cap,
                             uint64_t *bytes, double *latency_ms, uint64_t *version,
                             trc_status *status);
trc_status trc_server_release(trc_server *s, uint64_t id);
/* kind < 0: every request; otherwise one trc_request_kind. */
trc_status trc_server_get_stats(trc_server *s, int kind, trc_server_stats *out);
trc_status trc_server_reset_stats(trc_server *s);
/* hold != 0: start no new round (requests queue up); hold = 0: the next round
 * takes every pending request, subject to the admission limits.  Lets a
 * caller gather a burst into one round.  Destroy drains a held server. */
trc_status trc_server_hold(trc_server *s, int hold);
/* One record per served round (the last 65536 since creation or reset):
 * where the round's time went and what it held. */
typedef struct {
  double t_start_ms;   /* round start, from the first submit (or reset) */
  double ms;           /* whole round */
  double lookup_ms, update_ms, bfs_ms, pagerank_ms; /* its parts (PageRank:
                          launch + the wait after the BFS part) */
  uint32_t lookups, updates, bfs, pageranks; /* requests of each kind */
  uint64_t update_pairs;                      /* pairs over its updates */
  uint32_t bfs_groups;  /* multi-source BFS launches */
  uint32_t bfs_singles; /* single-source BFS runs */
  uint32_t rebuilds;    /* full tier-2 rebuilds */
  uint32_t pending_after; /* requests left queued when the round started */
} trc_round_record;
/* Copies up to cap records, oldest first; *count = records held. */
trc_status trc_server_rounds(trc_server *s, trc_round_record *out, uint64_t cap,
                             uint64_t *count);

/* ---- diagnostics (no reference counterpart: the reference has only
 *      lock-ownership checks, src/PMA.cc:29-111). */
typedef struct {
  uint32_t n;
  uint64_t num_edges;
  uint64_t inline_edges;   /* tier 1 */
  uint64_t pma_edges;      /* tier 2 */
  uint64_t pma_capacity;   /* tier-2 slots */
  uint64_t hub_edges;      /* tier 3 */
  uint32_t num_hubs;
  uint64_t hub_blocks_used;
  uint64_t device_bytes;   /* bytes held on the device */
  uint64_t pma_rebuilds;   /* full tier-2 rebuilds so far */
  uint64_t pma_window_rebalances; /* local window rebalances so far */
  /* sizes inside the last update batch */
  uint64_t last_keys;      /* keys after symmetrize */
  uint64_t last_applied;   /* edges inserted / removed */
  uint64_t last_touched;   /* source vertices with changes */
  uint64_t last_rewritten; /* vertices whose lists were rewritten */
  uint64_t last_gathered;  /* list elements read (old lists) */
  uint64_t last_written;   /* list elements written (new lists) */
  uint64_t last_windows;   /* PMA windows rebalanced */
  uint64_t last_rebuild;   /* 1 if the PMA was rebuilt */
  /* the blocked tier (hubs) in the last batch */
  uint64_t last_hub_touched;        /* hubs with batch edges */
  uint64_t last_hub_local;          /* of those, updated block by block */
  uint64_t last_hub_rewritten;      /* of those, rewritten whole */
  uint64_t last_hub_blocks_written; /* blocks written (splits included) */
  uint64_t last_hub_read;           /* hub list elements read */
  uint64_t last_hub_written;        /* hub list elements written */
  /* the blocked tier since creation */
  uint64_t hub_splits;              /* blocks added by splits */
  uint64_t hub_rewrites;            /* whole-hub rewrites */
  uint64_t hub_blocks_free;         /* pool blocks on the free list */
  uint64_t hub_absorbs;             /* under-full blocks merged with their successor */
  uint64_t sort_retries;            /* batches re-sorted by the radix sort (a source
                                       with more than 16384 keys in the batch) */
} trc_stats;
trc_status trc_get_stats(trc_graph *g, trc_stats *out);
/* Checks every structural invariant on the device (sorted, duplicate-free
 * lists, degree = list length, tier-2 segments inside their slots, hub
 * blocks packed and ordered).  *violations = number of broken invariants. */
trc_status trc_check(trc_graph *g, uint64_t *violations);

/* Per-kernel device time, recorded with CUDA events on the handle's stream
 * around every launch while enabled.  trc_profile_get returns the summed
 * milliseconds and launch count of the kernel called `name` (of every kernel
 * whose name starts with the prefix when `name` ends in '*'; all kernels
 * when `name` is NULL). */
trc_status trc_profile_enable(trc_graph *g, int on);
trc_status trc_profile_reset(trc_graph *g);
trc_status trc_profile_get(trc_graph *g, const char *name, double *ms,
                           uint64_t *launches);
/* Names of the kernels recorded so far, newline-separated, into buf. */
trc_status trc_profile_names(trc_graph *g, char *buf, uint64_t cap);
/* Kernels this handle has launched since it was created (always counted). */
trc_status trc_launch_count(trc_graph *g, uint64_t *launches);

#ifdef __cplusplus
}
#endif
#endif /* TERRACE_B200_H_ */
