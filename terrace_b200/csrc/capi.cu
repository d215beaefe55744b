// capi.cu -- the extern "C" boundary (include/terrace_b200.h).  Every entry
// point converts internal errors into a trc_status and keeps the message in
// thread-local storage for trc_last_error().
#include <cstring>
#include <string>

#include "graph.cuh"

namespace trc {
void rmat_generate(uint32_t n, uint32_t seed, double a, double b, double c, uint64_t first,
                   uint64_t count, uint32_t *src, uint32_t *dst, cudaStream_t s);
}

struct trc_graph {
  trc::Graph *g;
};

namespace {
thread_local std::string g_last_error;

template <typename F>
trc_status guard(F &&f) {
  try {
    f();
    g_last_error.clear();
    return TRC_OK;
  } catch (const trc::Error &e) {
    g_last_error = e.msg;
    return e.status;
  } catch (const std::bad_alloc &) {
    g_last_error = "host allocation failed";
    return TRC_ERR_NOMEM;
  } catch (const std::exception &e) {
    g_last_error = e.what();
    return TRC_ERR_STATE;
  }
}

// The graph behind a handle, for the batch entry points: a batch may leave
// its last kernels running (the next batch overlaps its input copy with them).
trc::Graph &G_batch(trc_graph *g) {
  if (!g || !g->g) trc::throw_error(TRC_ERR_INVALID, "null graph handle");
  return *g->g;
}

// Every other entry point sees the graph with the last batch finished.
trc::Graph &G(trc_graph *g) {
  trc::Graph &x = G_batch(g);
  x.complete_pending();
  return x;
}
}  // namespace

// Shared with server.cu: the graph behind a handle, and the error slot.
trc::Graph &trc_internal_graph(trc_graph *g) { return G(g); }
extern "C" trc_status trc_internal_set_error(trc_status st, const char *msg) {
  g_last_error = msg ? msg : "";
  return st;
}

extern "C" {

void trc_config_default(trc_config *cfg) {
  if (!cfg) return;
  cfg->hub_threshold = 1024;
  cfg->pma_root_density = 0.75;
  cfg->pma_build_density = 0.375;
  cfg->hub_block_fill = 0.75;
  cfg->push_pull_divisor = 20;
  cfg->hub_stage_limit = 49152;
  cfg->cuda_graphs = 1;
}

const char *trc_status_string(trc_status s) {
  switch (s) {
    case TRC_OK: return "ok";
    case TRC_ERR_INVALID: return "invalid argument";
    case TRC_ERR_NOMEM: return "out of device memory / HBM budget";
    case TRC_ERR_CUDA: return "CUDA error";
    case TRC_ERR_TIMEOUT: return "device wait timed out";
    case TRC_ERR_STATE: return "invalid state";
    case TRC_ERR_NOT_BUILT: return "kernels not available";
    case TRC_ERR_IO: return "file input/output failed";
  }
  return "unknown status";
}

const char *trc_last_error(void) { return g_last_error.c_str(); }

trc_status trc_graph_create(uint32_t n, uint64_t hbm_budget_bytes, const trc_config *cfg,
                            trc_graph **out) {
  return guard([&] {
    if (!out) trc::throw_error(TRC_ERR_INVALID, "null output handle");
    if (n == 0) trc::throw_error(TRC_ERR_INVALID, "n must be positive");
    int dev = 0;
    TRC_CUDA(cudaGetDevice(&dev));
    trc_config c;
    trc_config_default(&c);
    if (cfg) c = *cfg;
    if (c.hub_threshold < trc::K_INLINE || c.hub_threshold > trc::HUB_THRESHOLD_MAX)
      trc::throw_error(TRC_ERR_INVALID, "hub_threshold must be in [16, 12288]");
    if (c.hub_stage_limit > 49152 || c.hub_stage_limit == 0) c.hub_stage_limit = 49152;
    *out = nullptr;
    trc_graph *h = new trc_graph{nullptr};
    try {
      h->g = new trc::Graph(n, hbm_budget_bytes, c);
    } catch (...) {
      delete h;
      throw;
    }
    *out = h;
  });
}

trc_status trc_graph_destroy(trc_graph *g) {
  return guard([&] {
    if (!g) return;
    delete g->g;
    delete g;
  });
}

static void fill_tuning(const trc::Graph &g, trc_tuning *o) {
  o->push_pull_divisor = g.tuned.push_pull_divisor;
  o->pr_group_cut = g.tuned.pr_group_cut;
  o->pr_group_lanes = g.tuned.pr_group_lanes;
  o->pma_leaf_log = g.tuned.pma_leaf_log;
}

trc_status trc_autotune(trc_graph *g, uint32_t what, const uint32_t *src, const uint32_t *dst,
                        uint64_t k, uint32_t flags, trc_tuning *out) {
  return guard([&] {
    trc::Graph &gr = G(g);
    if (what & ~(TRC_TUNE_PUSH_PULL | TRC_TUNE_PAGERANK | TRC_TUNE_PMA))
      trc::throw_error(TRC_ERR_INVALID, "unknown TRC_TUNE_* bit");
    double ms[3];
    gr.autotune(what, src, dst, k, flags, ms);
    if (out) {
      memset(out, 0, sizeof(*out));
      fill_tuning(gr, out);
      out->bfs_ms = ms[0];
      out->pagerank_iter_ms = ms[1];
      out->pma_insert_ms = ms[2];
    }
  });
}

trc_status trc_get_tuning(trc_graph *g, trc_tuning *out) {
  return guard([&] {
    if (!out) trc::throw_error(TRC_ERR_INVALID, "null output");
    memset(out, 0, sizeof(*out));
    fill_tuning(G(g), out);
  });
}

trc_status trc_set_tuning(trc_graph *g, const trc_tuning *in) {
  return guard([&] {
    trc::Graph &gr = G(g);
    if (!in) trc::throw_error(TRC_ERR_INVALID, "null input");
    if (in->push_pull_divisor < 1) trc::throw_error(TRC_ERR_INVALID, "push_pull_divisor >= 1");
    if (in->pr_group_lanes != 4 && in->pr_group_lanes != 8 && in->pr_group_lanes != 16)
      trc::throw_error(TRC_ERR_INVALID, "pr_group_lanes must be 4, 8 or 16");
    if (in->pr_group_cut <= trc::K_INLINE || in->pr_group_cut > 4096)
      trc::throw_error(TRC_ERR_INVALID, "pr_group_cut must be in 17..4096");
    if (in->pma_leaf_log < 1 || in->pma_leaf_log > 20)
      trc::throw_error(TRC_ERR_INVALID, "pma_leaf_log must be in 1..20");
    gr.sync();
    if (in->pr_group_cut != gr.tuned.pr_group_cut) gr.lists.version = ~0ull;
    gr.tuned.push_pull_divisor = in->push_pull_divisor;
    gr.tuned.pr_group_cut = in->pr_group_cut;
    gr.tuned.pr_group_lanes = in->pr_group_lanes;
    gr.tuned.pma_leaf_log = in->pma_leaf_log;
  });
}

trc_status trc_graph_set_stream(trc_graph *g, void *stream) {
  return guard([&] {
    trc::Graph &gr = G(g);
    gr.sync();
    gr.stream = stream ? static_cast<cudaStream_t>(stream) : gr.own_stream;
    gr.budget.stream = gr.stream;
  });
}

trc_status trc_release_scratch(trc_graph *g) {
  return guard([&] { G(g).release_scratch(); });
}

trc_status trc_debug_sort_wait(trc_graph *g, uint32_t spin_limit, int withhold_first_tile) {
  return guard([&] {
    trc::Graph &gr = G(g);
    gr.sort_wait.spin_limit = spin_limit ? spin_limit : trc::SortWait{}.spin_limit;
    gr.sort_wait.withhold_first = withhold_first_tile != 0;
  });
}

trc_status trc_debug_sort_mode(trc_graph *g, int mode) {
  return guard([&] {
    if (mode < 0 || mode > 2) trc::throw_error(TRC_ERR_INVALID, "sort mode must be 0, 1 or 2");
    G(g).sort_mode = mode;
  });
}

trc_status trc_add_edge_batch(trc_graph *g, const uint32_t *src, const uint32_t *dst, uint64_t k,
                              uint32_t flags, uint64_t *applied) {
  return guard([&] {
    uint64_t a = G_batch(g).apply_batch(src, dst, k, flags, true, true);
    if (applied) *applied = a;
  });
}

trc_status trc_remove_edge_batch(trc_graph *g, const uint32_t *src, const uint32_t *dst,
                                 uint64_t k, uint32_t flags, uint64_t *applied) {
  return guard([&] {
    uint64_t a = G_batch(g).apply_batch(src, dst, k, flags, false, true);
    if (applied) *applied = a;
  });
}

trc_status trc_is_edge(trc_graph *g, const uint32_t *src, const uint32_t *dst, uint64_t q,
                       uint8_t *out, uint32_t flags) {
  return guard([&] { G(g).is_edge(src, dst, q, out, flags); });
}

trc_status trc_degree(trc_graph *g, const uint32_t *v, uint64_t q, uint32_t *out, uint32_t flags) {
  return guard([&] { G(g).degree(v, q, out, flags); });
}

trc_status trc_neighbors(trc_graph *g, uint32_t v, uint32_t *out, uint64_t cap, uint64_t *len,
                         uint32_t flags) {
  return guard([&] {
    uint64_t d = G(g).neighbors(v, out, cap, flags);
    if (len) *len = d;
  });
}

trc_status trc_count_common(trc_graph *g, const uint32_t *s, const uint32_t *d, uint64_t q,
                            uint32_t *out, uint32_t flags) {
  return guard([&] { G(g).count_common(s, d, q, out, flags); });
}

trc_status trc_num_vertices(trc_graph *g, uint32_t *n) {
  return guard([&] {
    if (!n) trc::throw_error(TRC_ERR_INVALID, "null output");
    *n = G(g).n;
  });
}

trc_status trc_num_edges(trc_graph *g, uint64_t *m) {
  return guard([&] {
    if (!m) trc::throw_error(TRC_ERR_INVALID, "null output");
    *m = G(g).m;
  });
}

trc_status trc_get_size(trc_graph *g, uint64_t *bytes) {
  return guard([&] {
    if (!bytes) trc::throw_error(TRC_ERR_INVALID, "null output");
    *bytes = G(g).size_bytes();
  });
}

trc_status trc_dump_csr(trc_graph *g, uint64_t *offsets, uint32_t *targets, uint32_t flags) {
  return guard([&] { G(g).dump_csr(offsets, targets, flags); });
}

trc_status trc_bfs(trc_graph *g, uint32_t src, int32_t *parents, uint32_t *levels, uint32_t flags) {
  return guard([&] { G(g).bfs(src, parents, levels, flags); });
}

trc_status trc_msbfs(trc_graph *g, const uint32_t *sources, uint32_t k, uint32_t *levels,
                     uint32_t flags) {
  return guard([&] { G(g).msbfs(sources, k, levels, flags); });
}

trc_status trc_msbc(trc_graph *g, const uint32_t *sources, uint32_t k, double *dep,
                    uint32_t flags) {
  return guard([&] { G(g).msbc(sources, k, dep, flags); });
}

trc_status trc_bfs_noalloc(trc_graph *g, uint32_t src, int32_t *parents, uint32_t *levels,
                           uint32_t flags) {
  return guard([&] { G(g).bfs_noalloc(src, parents, levels, flags); });
}

trc_status trc_pagerank(trc_graph *g, uint32_t iters, double damping, double *ranks,
                        uint32_t flags) {
  return guard([&] { G(g).pagerank(iters, damping, ranks, flags); });
}

trc_status trc_cc(trc_graph *g, uint32_t *labels, uint32_t flags) {
  return guard([&] { G(g).cc(labels, flags); });
}

trc_status trc_bc(trc_graph *g, uint32_t src, double *dep, uint32_t flags) {
  return guard([&] { G(g).bc(src, dep, flags); });
}

trc_status trc_tc(trc_graph *g, uint64_t *count) {
  return guard([&] {
    if (!count) trc::throw_error(TRC_ERR_INVALID, "null output");
    *count = G(g).tc();
  });
}

trc_status trc_rmat_generate(uint32_t n, uint32_t seed, double a, double b, double c,
                             uint64_t first, uint64_t count, uint32_t *src, uint32_t *dst,
                             uint32_t flags, void *stream) {
  return guard([&] {
    if (count && (!src || !dst)) trc::throw_error(TRC_ERR_INVALID, "null output");
    if (n == 0 || (n & (n - 1))) trc::throw_error(TRC_ERR_INVALID, "n must be a power of two");
    if (a + b + c > 1.0) trc::throw_error(TRC_ERR_INVALID, "a + b + c > 1");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (flags & TRC_DEVICE_PTR) {
      trc::rmat_generate(n, seed, a, b, c, first, count, src, dst, s);
      TRC_CUDA(cudaStreamSynchronize(s));
      return;
    }
    uint32_t *ds = nullptr, *dd = nullptr;
    TRC_CUDA(cudaMalloc(&ds, (count ? count : 1) * 4));
    cudaError_t e = cudaMalloc(&dd, (count ? count : 1) * 4);
    if (e != cudaSuccess) {
      cudaFree(ds);
      TRC_CUDA(e);
    }
    try {
      trc::rmat_generate(n, seed, a, b, c, first, count, ds, dd, s);
      TRC_CUDA(cudaMemcpyAsync(src, ds, count * 4, cudaMemcpyDeviceToHost, s));
      TRC_CUDA(cudaMemcpyAsync(dst, dd, count * 4, cudaMemcpyDeviceToHost, s));
      TRC_CUDA(cudaStreamSynchronize(s));
    } catch (...) {
      cudaFree(ds);
      cudaFree(dd);
      throw;
    }
    cudaFree(ds);
    cudaFree(dd);
  });
}

trc_status trc_get_device_view(trc_graph *g, trc_device_view *out) {
  return guard([&] {
    if (!out) trc::throw_error(TRC_ERR_INVALID, "null output");
    trc::Graph &gr = G(g);
    gr.sync();
    trc::DevView v = gr.view();
    out->n = v.n;
    out->inline_slots = trc::K_INLINE;
    out->hub_block = trc::HUB_BLOCK;
    out->deg = v.deg;
    out->inl = v.inl;
    out->pbeg = v.pbeg;
    out->pma = v.pma;
    out->hub_of = v.hub_of;
    out->hub_dir0 = v.hub_dir0;
    out->hub_nblk = v.hub_nblk;
    out->hub_dir = v.hdir;
    out->hub_pre = v.hpre;
    out->hub_key = v.hkey;
    out->hslot = v.hslot;
    out->stream = gr.stream;
  });
}

trc_status trc_get_stats(trc_graph *g, trc_stats *out) {
  return guard([&] {
    if (!out) trc::throw_error(TRC_ERR_INVALID, "null output");
    G(g).stats(out);
  });
}

trc_status trc_check(trc_graph *g, uint64_t *violations) {
  return guard([&] {
    if (!violations) trc::throw_error(TRC_ERR_INVALID, "null output");
    *violations = G(g).check();
  });
}

trc_status trc_profile_enable(trc_graph *g, int on) {
  return guard([&] { G(g).prof.on = on != 0; });
}

trc_status trc_profile_reset(trc_graph *g) {
  return guard([&] { G(g).prof.reset(); });
}

trc_status trc_profile_get(trc_graph *g, const char *name, double *ms, uint64_t *launches) {
  return guard([&] {
    trc::Graph &gr = G(g);
    gr.prof.resolve();
    double t = 0;
    uint64_t c = 0;
    std::string want = name ? name : "";
    bool prefix = !want.empty() && want.back() == '*';
    if (prefix) want.pop_back();
    for (auto &kv : gr.prof.totals) {
      if (!name || (prefix ? kv.first.compare(0, want.size(), want) == 0 : kv.first == want)) {
        t += kv.second.first;
        c += kv.second.second;
      }
    }
    if (ms) *ms = t;
    if (launches) *launches = c;
  });
}

trc_status trc_profile_names(trc_graph *g, char *buf, uint64_t cap) {
  return guard([&] {
    trc::Graph &gr = G(g);
    gr.prof.resolve();
    std::string s;
    for (auto &kv : gr.prof.totals) {
      s += kv.first;
      s += "\n";
    }
    if (buf && cap) {
      uint64_t k = s.size() < cap - 1 ? s.size() : cap - 1;
      memcpy(buf, s.data(), k);
      buf[k] = 0;
    }
  });
}

trc_status trc_launch_count(trc_graph *g, uint64_t *launches) {
  return guard([&] {
    if (!launches) trc::throw_error(TRC_ERR_INVALID, "null output");
    *launches = G(g).prof.launches;
  });
}

}  // extern "C"
