// cxx_facade_check.cc -- drives the C++ facade (include/terrace_b200.hpp)
// the way src/graph_bm.cc drives graphstore::Graph, and prints the results
// as one line of numbers for tests/test_edge_map.py to compare.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "terrace_b200.hpp"

using namespace terrace;

int main() {
  const uint32_t n = 1u << 12;
  std::vector<uint32_t> s(8 * n), d(8 * n);
  trc_rmat_generate(n, 0, 0.5, 0.1, 0.1, 0, 8 * n, s.data(), d.data(), 0, nullptr);
  Graph g(n);
  g.add_edge_batch(s.data(), d.data(), s.size(), TRC_SYMMETRIZE | TRC_DROP_SELF_LOOPS);
  uint32_t best = 0;
  for (uint32_t v = 0; v < n; v++)
    if (g.degree(v) > g.degree(best)) best = v;
  int32_t *par = BFS_with_edge_map(g, best);
  uint32_t reached = 0;
  for (uint32_t v = 0; v < n; v++) reached += par[v] >= 0;
  double *pr = PR_S<double>(g, 5);
  double prsum = 0;
  for (uint32_t v = 0; v < n; v++) prsum += pr[v];
  uint32_t *cc = CC(g);
  uint32_t comps = 0;
  for (uint32_t v = 0; v < n; v++) comps += cc[v] == v;
  double *bc = BC(g, best);
  uint64_t tri = TC(g);
  uint64_t nb = 0;
  for (auto it = g.neighbors(best); !it.done(); ++it) nb++;
  int dup = g.add_edge(best, *g.neighbors(best));  // existing edge: -1
  std::printf("%u %llu %u %u %.17g %u %llu %llu %d %u\n", n, (unsigned long long)g.num_edges(),
              best, reached, prsum, comps, (unsigned long long)tri, (unsigned long long)nb, dup,
              g.is_edge(best, *g.neighbors(best)));
  free(par);
  free(pr);
  free(cc);
  free(bc);
  return 0;
}
