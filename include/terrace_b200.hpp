// terrace_b200.hpp -- C++ host facade with the reference's Graph API.
//
// A drop-in for graphstore::Graph (include/graph.h:73-230) and the algorithm
// entry points of the reference (include/BFS.h, Pagerank.h, Components.h,
// BC.h, TC.h), implemented over the C ABI in terrace_b200.h.  Plain C++17,
// no CUDA headers needed; link libterrace_b200.so.  Generic edgeMap /
// vertexMap with user device functors live in terrace_b200_edge_map.cuh
// (nvcc).
//
// Method names and argument meanings follow the reference.  Differences:
// errors throw terrace::Error (the reference exits); add_edge_batch does not
// mutate its inputs and accepts unsorted, duplicated input; the perm argument
// of the reference's add_edge_batch is accepted and ignored (the device
// pipeline has no insertion order).
#pragma once

#include <cstdint>
#include <cstdlib>
#include <stdexcept>
#include <string>
#include <vector>

#include "terrace_b200.h"

namespace terrace {

class Error : public std::runtime_error {
 public:
  Error(trc_status s, const std::string &m) : std::runtime_error(m), status(s) {}
  trc_status status;
};

inline void check(trc_status s) {
  if (s != TRC_OK)
    throw Error(s, std::string(trc_status_string(s)) + ": " + trc_last_error());
}

class Graph {
 public:
  typedef uint32_t vertex;

  explicit Graph(uint32_t size, uint64_t hbm_budget_bytes = 0, const trc_config *cfg = nullptr) {
    check(trc_graph_create(size, hbm_budget_bytes, cfg, &g_));
  }
  ~Graph() {
    if (g_) trc_graph_destroy(g_);
  }
  Graph(const Graph &) = delete;
  Graph &operator=(const Graph &) = delete;

  trc_graph *handle() const { return g_; }

  // Graph::add_edge_batch (include/graph.h:430-502).  perm is ignored.
  void add_edge_batch(vertex *srcs, vertex *dests, uint32_t edge_count,
                      std::vector<uint32_t> & /*perm*/) {
    check(trc_add_edge_batch(g_, srcs, dests, edge_count, 0, nullptr));
  }
  // Batch insert with flags (TRC_SYMMETRIZE, TRC_DROP_SELF_LOOPS,
  // TRC_DEVICE_PTR); returns directed edges inserted.
  uint64_t add_edge_batch(const vertex *srcs, const vertex *dests, uint64_t k,
                          uint32_t flags = 0) {
    uint64_t a = 0;
    check(trc_add_edge_batch(g_, srcs, dests, k, flags, &a));
    return a;
  }
  // Declared but not implemented by the reference (include/graph.h:143-150).
  uint64_t remove_edge_batch(const vertex *srcs, const vertex *dests, uint64_t k,
                             uint32_t flags = 0) {
    uint64_t a = 0;
    check(trc_remove_edge_batch(g_, srcs, dests, k, flags, &a));
    return a;
  }
  // Graph::add_edge / remove_edge: 0 on success, -1 if nothing changed.
  int add_edge(const vertex s, const vertex d) { return add_edge_batch(&s, &d, 1) ? 0 : -1; }
  int remove_edge(const vertex s, const vertex d) {
    return remove_edge_batch(&s, &d, 1) ? 0 : -1;
  }

  uint32_t is_edge(const vertex s, const vertex d) const {
    uint8_t r = 0;
    check(trc_is_edge(g_, &s, &d, 1, &r, 0));
    return r;
  }
  uint32_t degree(const vertex v) const {
    uint32_t r = 0;
    check(trc_degree(g_, &v, 1, &r, 0));
    return r;
  }
  uint32_t count_common(const vertex s, const vertex d) const {
    uint32_t r = 0;
    check(trc_count_common(g_, &s, &d, 1, &r, 0));
    return r;
  }
  uint32_t get_num_vertices() const {
    uint32_t n = 0;
    check(trc_num_vertices(g_, &n));
    return n;
  }
  // The reference returns uint32_t (include/graph.h:817-822); num_edges()
  // gives the full 64-bit count.
  uint32_t get_num_edges() const { return (uint32_t)num_edges(); }
  uint64_t num_edges() const {
    uint64_t m = 0;
    check(trc_num_edges(g_, &m));
    return m;
  }
  uint64_t get_size() const {
    uint64_t b = 0;
    check(trc_get_size(g_, &b));
    return b;
  }

  // Sorted neighbours of v (host copy).
  std::vector<vertex> neighbor_list(const vertex v) const {
    uint64_t len = 0;
    check(trc_neighbors(g_, v, nullptr, 0, &len, 0));
    std::vector<vertex> out(len);
    if (len) check(trc_neighbors(g_, v, out.data(), len, &len, 0));
    return out;
  }

  // Graph::NeighborIterator (include/graph.h:844-899): sorted order.
  class NeighborIterator {
   public:
    NeighborIterator(const Graph *g, vertex v) : list_(g->neighbor_list(v)) {}
    vertex operator*() const { return list_[i_]; }
    void operator++() { ++i_; }
    bool done() const { return i_ >= list_.size(); }

   private:
    std::vector<vertex> list_;
    size_t i_ = 0;
  };
  NeighborIterator neighbors(const vertex v) const { return NeighborIterator(this, v); }

  // Calls f(v, w) for every neighbour w of v in sorted order.
  template <class F>
  void map_neighbors(const vertex v, F f) const {
    for (vertex w : neighbor_list(v)) f(v, w);
  }

 private:
  trc_graph *g_ = nullptr;
};

// ---- algorithm entry points with the reference's names and ownership:
// results are malloc'd host arrays the caller frees (src/graph_bm.cc:99).

// BFS_with_edge_map (include/BFS.h:41-84): parents, -1 unreached.
inline int32_t *BFS_with_edge_map(Graph &G, uint32_t src) {
  int32_t *p = (int32_t *)malloc(sizeof(int32_t) * G.get_num_vertices());
  if (!p) throw std::bad_alloc();
  trc_status s = trc_bfs(G.handle(), src, p, nullptr, 0);
  if (s != TRC_OK) free(p);
  check(s);
  return p;
}

// PR_S<double> (include/Pagerank.h:105-184): undamped, maxIters iterations.
template <typename T>
T *PR_S(Graph &G, long maxIters) {
  static_assert(sizeof(T) == sizeof(double), "PR_S computes in FP64");
  double *p = (double *)malloc(sizeof(double) * G.get_num_vertices());
  if (!p) throw std::bad_alloc();
  trc_status s = trc_pagerank(G.handle(), (uint32_t)maxIters, 0.0, p, 0);
  if (s != TRC_OK) free(p);
  check(s);
  return reinterpret_cast<T *>(p);
}

// CC (include/Components.h:92-120): smallest vertex id per component.
inline uint32_t *CC(Graph &G) {
  uint32_t *l = (uint32_t *)malloc(sizeof(uint32_t) * G.get_num_vertices());
  if (!l) throw std::bad_alloc();
  trc_status s = trc_cc(G.handle(), l, 0);
  if (s != TRC_OK) free(l);
  check(s);
  return l;
}

// BC (include/BC.h:99-157): dependencies, NaN for unreached vertices.
inline double *BC(Graph &G, const uint32_t &start) {
  double *d = (double *)malloc(sizeof(double) * G.get_num_vertices());
  if (!d) throw std::bad_alloc();
  trc_status s = trc_bc(G.handle(), start, d, 0);
  if (s != TRC_OK) free(d);
  check(s);
  return d;
}

// BC of up to 64 sources in one traversal: row i (n doubles) = BC(G, starts[i]).
inline double *BC_multi(Graph &G, const uint32_t *starts, uint32_t k) {
  double *d = (double *)malloc(sizeof(double) * (size_t)k * G.get_num_vertices());
  if (!d) throw std::bad_alloc();
  trc_status s = trc_msbc(G.handle(), starts, k, d, 0);
  if (s != TRC_OK) free(d);
  check(s);
  return d;
}

// TC (include/TC.h:73-87): exact triangle count.
inline uint64_t TC(Graph &G) {
  uint64_t c = 0;
  check(trc_tc(G.handle(), &c));
  return c;
}

}  // namespace terrace
