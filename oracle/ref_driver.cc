// ref_driver.cc -- C entry points over the UNMODIFIED reference Terrace
// (graphstore::Graph and its Ligra-style algorithms), compiled from the
// reference's own headers and sources where they lie by oracle/build_ref.sh
// into oracle/_ref/libterrace_ref.so.
//
// Used only as a checker (golden fixtures, oracle pinning) and as the timed
// CPU baseline of bench.py --impl reference.  It mirrors the phases of the
// reference benchmark driver src/graph_bm.cc:231-391.
//
// Preconditions the caller must meet (reference behaviours, see
// src/graph_bm.cc and include/graph.h):
//   * add_edge_batch input sorted by (src,dst) and duplicate-free
//     (include/graph.h:269-289 copies duplicates into the in-place slots);
//   * remove only edges that exist (include/graph.h:695-716 drops the largest
//     in-place neighbour when asked to remove an absent edge).
// Same compile-time configuration as src/graph_bm.cc:12-14: per-vertex
// degree locks on (concurrent add/remove on one vertex are serialised),
// unweighted, no VERIFY dumps.
#define ENABLE_LOCK 1
#define WEIGHTED 0
#define VERIFY 0

#include <stdint.h>
#include <stdio.h>
#include <unistd.h>
#include <fcntl.h>
#include <random>
#include <algorithm>
#include <vector>

#include "graph.h"
#include "BFS.h"
#include "Pagerank.h"
#include "Components.h"
#include "BC.h"
#include "TC.h"
#include "rmat_util.h"
#include "io_util.h"

namespace {

// The reference prints progress lines to stdout inside add_edge_batch
// (include/graph.h:478,500) and PR_S (include/Pagerank.h:122); callers of
// this library expect a clean stdout, so those calls run with fd 1 muted.
struct QuietStdout {
  int saved = -1;
  QuietStdout() {
    fflush(stdout);
    saved = dup(1);
    int devnull = open("/dev/null", O_WRONLY);
    if (devnull >= 0) { dup2(devnull, 1); close(devnull); }
  }
  ~QuietStdout() {
    fflush(stdout);
    if (saved >= 0) { dup2(saved, 1); close(saved); }
  }
};

}  // namespace

extern "C" {

void ref_set_threads(int t) { setWorkers(t); }
int ref_get_threads(void) { return getWorkers(); }

void *ref_graph_new(uint32_t n) { return new Graph(n); }
void ref_graph_free(void *g) { delete static_cast<Graph *>(g); }

// Graph::add_edge_batch (include/graph.h:430-502) with a seeded random
// permutation in place of the time-seeded get_random_permutation
// (src/util.cc:60-78), so runs are repeatable.
void ref_add_edge_batch(void *gp, const uint32_t *src, const uint32_t *dst,
                        uint32_t k, uint32_t perm_seed) {
  if (k == 0) return;
  Graph &g = *static_cast<Graph *>(gp);
  std::vector<uint32_t> s(src, src + k), d(dst, dst + k), perm(k);
  for (uint32_t i = 0; i < k; i++) perm[i] = i;
  std::mt19937 rng(perm_seed);
  std::shuffle(perm.begin(), perm.end(), rng);
  QuietStdout q;
  g.add_edge_batch(s.data(), d.data(), k, perm);
}

// parallel_for over Graph::remove_edge, as src/graph_bm.cc:375-380 does.
// Returns how many removes reported -1.
int64_t ref_remove_edges(void *gp, const uint32_t *src, const uint32_t *dst,
                         uint32_t k) {
  Graph &g = *static_cast<Graph *>(gp);
  int64_t failed = 0;
#pragma omp parallel for reduction(+ : failed)
  for (uint32_t i = 0; i < k; i++) failed += (g.remove_edge(src[i], dst[i]) != 0);
  return failed;
}

uint32_t ref_degree(void *gp, uint32_t v) { return static_cast<Graph *>(gp)->degree(v); }
uint32_t ref_is_edge(void *gp, uint32_t s, uint32_t d) {
  return static_cast<Graph *>(gp)->is_edge(s, d);
}
uint64_t ref_num_vertices(void *gp) { return static_cast<Graph *>(gp)->get_num_vertices(); }

uint64_t ref_num_edges(void *gp) {
  Graph &g = *static_cast<Graph *>(gp);
  uint64_t m = 0;
  for (uint32_t v = 0; v < g.get_num_vertices(); v++) m += g.degree(v);
  return m;
}

// Sorted neighbour lists through Graph::NeighborIterator
// (include/graph.h:844-899).  off has n+1 entries; tgt has ref_num_edges().
void ref_dump_csr(void *gp, uint64_t *off, uint32_t *tgt) {
  Graph &g = *static_cast<Graph *>(gp);
  uint32_t n = g.get_num_vertices();
  off[0] = 0;
  for (uint32_t v = 0; v < n; v++) off[v + 1] = off[v] + g.degree(v);
#pragma omp parallel for schedule(dynamic, 1024)
  for (uint32_t v = 0; v < n; v++) {
    uint64_t o = off[v];
    for (auto it = g.neighbors(v); !it.done(); ++it) tgt[o++] = *it;
  }
}

// BFS_with_edge_map (include/BFS.h:41-84).
void ref_bfs(void *gp, uint32_t src, int32_t *parents) {
  Graph &g = *static_cast<Graph *>(gp);
  int32_t *p = BFS_with_edge_map(g, src);
  memmove(parents, p, sizeof(int32_t) * g.get_num_vertices());
  free(p);
}

// PR_S<double> (include/Pagerank.h:105-184).
void ref_pagerank(void *gp, uint32_t iters, double *out) {
  Graph &g = *static_cast<Graph *>(gp);
  double *p;
  {
    QuietStdout q;
    p = PR_S<double>(g, iters);
  }
  memmove(out, p, sizeof(double) * g.get_num_vertices());
  free(p);
}

// CC (include/Components.h:92-120).
void ref_cc(void *gp, uint32_t *out) {
  Graph &g = *static_cast<Graph *>(gp);
  uint32_t *ids = CC(g);
  memmove(out, ids, sizeof(uint32_t) * g.get_num_vertices());
  free(ids);
}

// BC (include/BC.h:99-157).
void ref_bc(void *gp, uint32_t src, double *out) {
  Graph &g = *static_cast<Graph *>(gp);
  double *dep = BC(g, src);
  memmove(out, dep, sizeof(double) * g.get_num_vertices());
  free(dep);
}

// TC (include/TC.h:73-87).  Known to miscount on some layouts; recorded
// for timing only, never used as the parity value.
uint64_t ref_tc(void *gp) { return TC(*static_cast<Graph *>(gp)); }

// Edges first..first+count-1 of the reference generator rMat<uint32_t>
// (include/rmat_util.h:81-115), used to pin the oracle's generator.
void ref_rmat(uint32_t n, uint32_t seed, double a, double b, double c,
              uint64_t first, uint64_t count, uint32_t *src, uint32_t *dst) {
  rMat<uint32_t> r(n, seed, a, b, c);
  for (uint64_t i = 0; i < count; i++) {
    std::pair<uint32_t, uint32_t> e = r((uint32_t)(first + i));
    src[i] = e.first;
    dst[i] = e.second;
  }
}

// The reference's AdjacencyGraph reader (get_edges_from_file_adj_sym,
// include/io_util.h:112-145) on a well-formed file: returns m and sets *n;
// with src/dst given (capacity cap) copies the edge pairs in file order.
uint64_t ref_read_adj(const char *path, uint32_t *n, uint32_t *src, uint32_t *dst, uint64_t cap) {
  uint64_t m = 0;
  uint32_t nn = 0;
  pair_uint *e = nullptr;
  {
    QuietStdout q;
    e = get_edges_from_file_adj_sym(path, &m, &nn, false);
  }
  *n = nn;
  if (src && dst)
    for (uint64_t i = 0; i < m && i < cap; i++) {
      src[i] = e[i].x;
      dst[i] = e[i].y;
    }
  free(e);
  return m;
}

}  // extern "C"
