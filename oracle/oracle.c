/*
 * oracle.c -- CPU restatement of the Terrace hot path, used ONLY as the
 * checker by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg.
 * It is test infrastructure, never the product: nothing in terrace_b200/
 * links, loads or calls it.
 *
 * The graph is modelled as a set of directed (src,dst) pairs; every result
 * is computed from the sorted neighbour lists (CSR: uint64 offsets[n+1],
 * uint32 targets[m]).  Each function cites the reference code it restates
 * (paths inside the PASSIONLab/terrace tree).
 *
 * Parity is pinned against the reference itself: oracle/build_ref.sh
 * compiles the reference's own sources into oracle/_ref/libterrace_ref.so and
 * tests/golden/make_golden.py records its outputs as fixtures.
 *
 * Build: gcc -O2 -std=c11 -fPIC -shared oracle.c -o liboracle.so -lm
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>

#define ORC_UNREACHED 0xFFFFFFFFu

/* ---------------------------------------------------------------------- */
/* Hashes and the RMAT generator: include/rmat_util.h:29-52, :81-115.      */
/* ---------------------------------------------------------------------- */

/* 64-bit hash (numerical recipes), include/rmat_util.h:29-40. */
uint64_t orc_hash64(uint64_t u) {
  uint64_t v = u * 3935559000370003845ull + 2691343689449507681ull;
  v ^= v >> 21;
  v ^= v << 37;
  v ^= v >> 4;
  v *= 4768777513237032717ull;
  v ^= v << 20;
  v ^= v >> 41;
  v ^= v << 5;
  return v;
}

/* 32-bit integer hash, include/rmat_util.h:44-52. */
uint32_t orc_hash32(uint32_t a) {
  a = (a + 0x7ed55d16u) + (a << 12);
  a = (a ^ 0xc761c23cu) ^ (a >> 19);
  a = (a + 0x165667b1u) + (a << 5);
  a = (a + 0xd3a2646cu) ^ (a << 9);
  a = (a + 0xfd7046c5u) + (a << 3);
  a = (a ^ 0xb55a4f09u) ^ (a >> 16);
  return a;
}

/*
 * Edge i of rMat<uint32_t>(n, seed, a, b, c), include/rmat_util.h:81-115.
 * The recursion rMatRec(nn, start, stride) draws r = hash32(start)/INT32_MAX
 * at the top level and recurses with start+stride, so level j (nn = n>>j)
 * uses start + j*stride.  The quadrant offsets add up independently of the
 * order, which gives this loop.  r is divided by INT32_MAX, not UINT32_MAX,
 * so r lies in [0,2): the effective quadrant probabilities are a/2, b/2, c/2.
 */
static inline void rmat_one(uint32_t n, uint32_t h, double a, double ab,
                            double abc, uint32_t i, uint32_t *u, uint32_t *v) {
  uint32_t rs = orc_hash32((uint32_t)(2u * i) * h);
  uint32_t st = orc_hash32((uint32_t)(2u * i + 1u) * h);
  uint32_t x = 0, y = 0;
  for (uint32_t nn = n; nn > 1; nn >>= 1) {
    double r = (double)orc_hash32(rs) / 2147483647.0;
    if (r < a) {
    } else if (r < ab) {
      y += nn / 2;
    } else if (r < abc) {
      x += nn / 2;
    } else {
      x += nn / 2;
      y += nn / 2;
    }
    rs += st;
  }
  *u = x;
  *v = y;
}

void orc_rmat(uint32_t n, uint32_t seed, double a, double b, double c,
              uint64_t first, uint64_t count, uint32_t *src, uint32_t *dst) {
  uint32_t h = orc_hash32(seed);
  double ab = a + b, abc = a + b + c;
  for (uint64_t k = 0; k < count; k++)
    rmat_one(n, h, a, ab, abc, (uint32_t)(first + k), &src[k], &dst[k]);
}

/* ---------------------------------------------------------------------- */
/* Edge-set helpers (64-bit keys src<<32|dst).                            */
/* ---------------------------------------------------------------------- */

/* LSD radix sort on 16-bit digits, only over the digits that vary. */
static void radix_sort_u64(uint64_t *keys, uint64_t k) {
  if (k < 2) return;
  uint64_t all_or = 0, all_and = ~0ull;
  for (uint64_t i = 0; i < k; i++) { all_or |= keys[i]; all_and &= keys[i]; }
  uint64_t diff = all_or ^ all_and;
  uint64_t *tmp = (uint64_t *)malloc(k * sizeof(uint64_t));
  uint64_t *cnt = (uint64_t *)malloc(65536 * sizeof(uint64_t));
  uint64_t *in = keys, *out = tmp;
  for (int shift = 0; shift < 64; shift += 16) {
    if (((diff >> shift) & 0xFFFFull) == 0) continue;
    memset(cnt, 0, 65536 * sizeof(uint64_t));
    for (uint64_t i = 0; i < k; i++) cnt[(in[i] >> shift) & 0xFFFF]++;
    uint64_t s = 0;
    for (int d = 0; d < 65536; d++) { uint64_t c = cnt[d]; cnt[d] = s; s += c; }
    for (uint64_t i = 0; i < k; i++) out[cnt[(in[i] >> shift) & 0xFFFF]++] = in[i];
    uint64_t *t = in; in = out; out = t;
  }
  if (in != keys) memcpy(keys, in, k * sizeof(uint64_t));
  free(tmp);
  free(cnt);
}

/*
 * Turn a batch of pairs into sorted unique keys.  symmetrize adds (v,u) for
 * every (u,v); drop_self removes u==v.  keys_out needs room for 2k keys when
 * symmetrize is set.  Returns the number of unique keys.
 */
uint64_t orc_make_keys(const uint32_t *src, const uint32_t *dst, uint64_t k,
                       int symmetrize, int drop_self, uint64_t *keys_out) {
  uint64_t m = 0;
  for (uint64_t i = 0; i < k; i++) {
    if (drop_self && src[i] == dst[i]) continue;
    keys_out[m++] = ((uint64_t)src[i] << 32) | dst[i];
    if (symmetrize) keys_out[m++] = ((uint64_t)dst[i] << 32) | src[i];
  }
  radix_sort_u64(keys_out, m);
  uint64_t u = 0;
  for (uint64_t i = 0; i < m; i++)
    if (u == 0 || keys_out[u - 1] != keys_out[i]) keys_out[u++] = keys_out[i];
  return u;
}

/* out = A union B (both sorted unique).  Returns |out|. */
uint64_t orc_key_union(const uint64_t *A, uint64_t na, const uint64_t *B,
                       uint64_t nb, uint64_t *out) {
  uint64_t i = 0, j = 0, o = 0;
  while (i < na && j < nb) {
    if (A[i] < B[j]) out[o++] = A[i++];
    else if (B[j] < A[i]) out[o++] = B[j++];
    else { out[o++] = A[i++]; j++; }
  }
  while (i < na) out[o++] = A[i++];
  while (j < nb) out[o++] = B[j++];
  return o;
}

/* out = A minus B (both sorted unique).  Returns |out|. */
uint64_t orc_key_difference(const uint64_t *A, uint64_t na, const uint64_t *B,
                            uint64_t nb, uint64_t *out) {
  uint64_t i = 0, j = 0, o = 0;
  while (i < na) {
    while (j < nb && B[j] < A[i]) j++;
    if (j < nb && B[j] == A[i]) { i++; continue; }
    out[o++] = A[i++];
  }
  return o;
}

/* out = A intersect B (both sorted unique).  Returns |out|. */
uint64_t orc_key_intersection(const uint64_t *A, uint64_t na, const uint64_t *B,
                              uint64_t nb, uint64_t *out) {
  uint64_t i = 0, j = 0, o = 0;
  while (i < na && j < nb) {
    if (A[i] < B[j]) i++;
    else if (B[j] < A[i]) j++;
    else { out[o++] = A[i++]; j++; }
  }
  return o;
}

/* CSR from sorted unique keys.  offsets has n+1 entries, targets k. */
void orc_csr_from_keys(uint32_t n, const uint64_t *keys, uint64_t k,
                       uint64_t *offsets, uint32_t *targets) {
  memset(offsets, 0, (size_t)(n + 1) * sizeof(uint64_t));
  for (uint64_t i = 0; i < k; i++) {
    offsets[(keys[i] >> 32) + 1]++;
    targets[i] = (uint32_t)keys[i];
  }
  for (uint32_t v = 0; v < n; v++) offsets[v + 1] += offsets[v];
}

/* ---------------------------------------------------------------------- */
/* BFS: include/BFS.h:27-84 with include/Map.cpp:65-74.                    */
/* Levels are unique; parents are any frontier neighbour (sparse CAS) or   */
/* the smallest-id frontier neighbour (dense pull), so only levels are     */
/* compared exactly and parents are checked for validity.                  */
/* ---------------------------------------------------------------------- */
void orc_bfs_levels(uint32_t n, const uint64_t *off, const uint32_t *tgt,
                    uint32_t src, uint32_t *level) {
  for (uint32_t v = 0; v < n; v++) level[v] = ORC_UNREACHED;
  if (src >= n) return;
  uint32_t *queue = (uint32_t *)malloc((size_t)n * sizeof(uint32_t));
  uint64_t head = 0, tail = 0;
  level[src] = 0;
  queue[tail++] = src;
  while (head < tail) {
    uint32_t u = queue[head++];
    for (uint64_t e = off[u]; e < off[u + 1]; e++) {
      uint32_t v = tgt[e];
      if (level[v] == ORC_UNREACHED) {
        level[v] = level[u] + 1;
        queue[tail++] = v;
      }
    }
  }
  free(queue);
}

/* Returns how many vertices violate: parent[src]==src; unreached -> -1;
 * otherwise (parent,v) is an edge and level[parent] == level[v]-1. */
uint64_t orc_bfs_check_parents(uint32_t n, const uint64_t *off,
                               const uint32_t *tgt, uint32_t src,
                               const uint32_t *level, const int32_t *parent) {
  uint64_t bad = 0;
  for (uint32_t v = 0; v < n; v++) {
    if (v == src) { bad += (parent[v] != (int32_t)src); continue; }
    if (level[v] == ORC_UNREACHED) { bad += (parent[v] != -1); continue; }
    int32_t p = parent[v];
    if (p < 0 || (uint32_t)p >= n || level[p] + 1 != level[v]) { bad++; continue; }
    /* (p, v) must be an edge: binary search v in N(p). */
    uint64_t lo = off[p], hi = off[p + 1];
    int found = 0;
    while (lo < hi) {
      uint64_t mid = (lo + hi) / 2;
      if (tgt[mid] < v) lo = mid + 1;
      else if (tgt[mid] > v) hi = mid;
      else { found = 1; break; }
    }
    bad += !found;
  }
  return bad;
}

/* ---------------------------------------------------------------------- */
/* PageRank: PR_S<double>, include/Pagerank.h:105-184.                     */
/* p0 = 1/n; per iteration p <- p/deg (PR_Vertex, :60-69), p_next = 0     */
/* (PR_Vertex_Reset, :89-98), then the dense pull map_dense_vs_all        */
/* (include/graph.h:1384-1487) adds p[v] over N(u) in sorted order        */
/* (PR_F::update, :39-44); swap.  There is no damping in the reference:   */
/* damping == 0 selects that.  damping in (0,1) gives                      */
/* p_next = (1-d)/n + d*sum, the textbook form (not in the reference).    */
/* ---------------------------------------------------------------------- */
void orc_pagerank(uint32_t n, const uint64_t *off, const uint32_t *tgt,
                  uint32_t iters, double damping, double *out) {
  double *p = (double *)malloc((size_t)n * sizeof(double));
  double *q = (double *)malloc((size_t)n * sizeof(double));
  double one_over_n = 1.0 / (double)n;
  double base = (1.0 - damping) / (double)n;
  for (uint32_t i = 0; i < n; i++) p[i] = one_over_n;
  for (uint32_t it = 0; it < iters; it++) {
    for (uint32_t i = 0; i < n; i++) p[i] = p[i] / (double)(off[i + 1] - off[i]);
    for (uint32_t u = 0; u < n; u++) {
      double s = 0.0;
      for (uint64_t e = off[u]; e < off[u + 1]; e++) s += p[tgt[e]];
      q[u] = (damping == 0.0) ? s : base + damping * s;
    }
    double *t = p; p = q; q = t;
  }
  memcpy(out, p, (size_t)n * sizeof(double));
  free(p);
  free(q);
}

/* ---------------------------------------------------------------------- */
/* CC: include/Components.h:92-120.  Label propagation with writeMin       */
/* (include/parallel_util.h:18-24) converges, on a symmetric graph, to the */
/* smallest vertex id of each component; that fixed point is computed     */
/* here with union-find.                                                   */
/* ---------------------------------------------------------------------- */
static uint32_t uf_find(uint32_t *par, uint32_t x) {
  while (par[x] != x) { par[x] = par[par[x]]; x = par[x]; }
  return x;
}

void orc_cc(uint32_t n, const uint64_t *off, const uint32_t *tgt,
            uint32_t *labels) {
  for (uint32_t v = 0; v < n; v++) labels[v] = v;
  for (uint32_t u = 0; u < n; u++)
    for (uint64_t e = off[u]; e < off[u + 1]; e++) {
      uint32_t a = uf_find(labels, u), b = uf_find(labels, tgt[e]);
      if (a < b) labels[b] = a;
      else if (b < a) labels[a] = b;
    }
  for (uint32_t v = 0; v < n; v++) labels[v] = uf_find(labels, v);
}

/* ---------------------------------------------------------------------- */
/* BC from one source: include/BC.h:99-157, in the dense (sorted-order)   */
/* form of its edgeMaps.  Forward: NumPaths[s]=1, NumPaths[v] = sum of     */
/* NumPaths over neighbours on the previous level (BC_F, :34-52).         */
/* Backward: inv = 1/NumPaths; Dep[v] = sum over neighbours on the next   */
/* level of Dep[w] (BC_Back_F, :54-73), then Dep[v] += inv[v]              */
/* (BC_Back_Vertex_F, :87-96); finally (Dep - inv)/inv (:140-142).         */
/* Unreached vertices give (0 - inf)/inf = NaN, as in the reference.      */
/* ---------------------------------------------------------------------- */
void orc_bc(uint32_t n, const uint64_t *off, const uint32_t *tgt, uint32_t src,
            double *out) {
  uint32_t *level = (uint32_t *)malloc((size_t)n * sizeof(uint32_t));
  uint32_t *order = (uint32_t *)malloc((size_t)n * sizeof(uint32_t));
  double *sigma = (double *)calloc(n, sizeof(double));
  double *dep = (double *)calloc(n, sizeof(double));
  for (uint32_t v = 0; v < n; v++) level[v] = ORC_UNREACHED;
  uint64_t head = 0, tail = 0;
  level[src] = 0;
  sigma[src] = 1.0;
  order[tail++] = src;
  /* BFS order; sigma of a vertex is final once its level is complete. */
  while (head < tail) {
    uint32_t u = order[head++];
    for (uint64_t e = off[u]; e < off[u + 1]; e++) {
      uint32_t v = tgt[e];
      if (level[v] == ORC_UNREACHED) { level[v] = level[u] + 1; order[tail++] = v; }
    }
  }
  for (uint64_t i = 1; i < tail; i++) {
    uint32_t v = order[i];
    double s = 0.0;
    for (uint64_t e = off[v]; e < off[v + 1]; e++)
      if (level[tgt[e]] + 1 == level[v]) s += sigma[tgt[e]];
    sigma[v] = s;
  }
  double *inv = (double *)malloc((size_t)n * sizeof(double));
  for (uint32_t v = 0; v < n; v++) inv[v] = 1.0 / sigma[v];
  for (uint64_t i = tail; i-- > 0;) {
    uint32_t v = order[i];
    double s = 0.0;
    for (uint64_t e = off[v]; e < off[v + 1]; e++)
      if (level[tgt[e]] == level[v] + 1) s += dep[tgt[e]];
    dep[v] = s + inv[v];
  }
  for (uint32_t v = 0; v < n; v++) out[v] = (dep[v] - inv[v]) / inv[v];
  free(level); free(order); free(sigma); free(dep); free(inv);
}

/* ---------------------------------------------------------------------- */
/* TC: include/TC.h:51-87 with Graph::count_common (include/graph.h:       */
/* 1085-1255): for every edge (s,d) with s > d, count common neighbours    */
/* w < min(s,d).  That is the exact triangle count (each triangle once).  */
/* ---------------------------------------------------------------------- */
uint64_t orc_tc(uint32_t n, const uint64_t *off, const uint32_t *tgt) {
  uint64_t total = 0;
  for (uint32_t s = 0; s < n; s++) {
    for (uint64_t e = off[s]; e < off[s + 1]; e++) {
      uint32_t d = tgt[e];
      if (d >= s) break; /* sorted: the rest are larger */
      uint64_t i = off[s], j = off[d];
      while (i < off[s + 1] && j < off[d + 1]) {
        uint32_t a = tgt[i], b = tgt[j];
        if (a >= d || b >= d) break;
        if (a == b) { total++; i++; j++; }
        else if (a < b) i++;
        else j++;
      }
    }
  }
  return total;
}

/* ---------------------------------------------------------------------- */
/* Triangles that contain at least one edge of a set B, for checking TC   */
/* after a batch without recounting the whole graph (same triangles as    */
/* orc_tc above, include/TC.h:51-87): with B as sorted unique directed    */
/* keys (src<<32|dst) holding both directions of each edge,               */
/*   T(G + B) = T(G) + orc_tc_touching(G + B, B minus G),                 */
/*   T(G - B) = T(G) - orc_tc_touching(G, B within G).                    */
/* A triangle is counted once, at its B edge with the smallest undirected */
/* key max<<32|min.                                                       */
/* ---------------------------------------------------------------------- */
static int key_in(const uint64_t *B, uint64_t nb, uint64_t x) {
  uint64_t lo = 0, hi = nb;
  while (lo < hi) {
    uint64_t mid = (lo + hi) / 2;
    if (B[mid] < x) lo = mid + 1;
    else hi = mid;
  }
  return lo < nb && B[lo] == x;
}

static uint64_t ukey(uint32_t a, uint32_t b) {
  return a > b ? ((uint64_t)a << 32) | b : ((uint64_t)b << 32) | a;
}

uint64_t orc_tc_touching(uint32_t n, const uint64_t *off, const uint32_t *tgt,
                         const uint64_t *bk, uint64_t nb) {
  uint64_t total = 0;
  for (uint64_t i = 0; i < nb; i++) {
    uint32_t u = (uint32_t)(bk[i] >> 32), v = (uint32_t)bk[i];
    if (u <= v || u >= n || v >= n) continue; /* each undirected edge once */
    uint64_t e = bk[i];
    uint64_t a = off[u], ae = off[u + 1], b = off[v], be = off[v + 1];
    while (a < ae && b < be) {
      uint32_t x = tgt[a], y = tgt[b];
      if (x < y) { a++; continue; }
      if (y < x) { b++; continue; }
      /* common neighbour w = x: triangle {u, v, w} */
      uint64_t f1 = ukey(u, x), f2 = ukey(v, x);
      if (!((f1 < e && key_in(bk, nb, f1)) || (f2 < e && key_in(bk, nb, f2)))) total++;
      a++;
      b++;
    }
  }
  return total;
}
