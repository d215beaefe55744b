// query.cu -- point queries over the tiers and the whole-graph dump.
//
// Replaces Graph::is_edge (include/graph.h:643-673), Graph::degree (:797-803),
// the NeighborIterator (:844-899), Graph::count_common (:1085-1255) and
// get_num_edges / get_size (:805-822).  The reference dispatches over six
// tier pairs in count_common; here every list is rank-addressable
// (NbrList::at), so one merge routine covers every pair.
#include "graph.cuh"

namespace trc {

__global__ void k_is_edge(DevView G, const uint32_t *s, const uint32_t *d, uint64_t q,
                          uint8_t *out) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= q) return;
  uint32_t u = s[i], x = d[i];
  if (u >= G.n || x >= G.n) {
    atomicOr(G.err, ERR_BAD_VERTEX);
    out[i] = 0;
    return;
  }
  out[i] = has_edge(G, u, x) ? 1 : 0;
}

__global__ void k_degree(DevView G, const uint32_t *v, uint64_t q, uint32_t *out) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= q) return;
  uint32_t u = v[i];
  if (u >= G.n) {
    atomicOr(G.err, ERR_BAD_VERTEX);
    out[i] = 0;
    return;
  }
  out[i] = G.deg[u];
}

__global__ void k_neighbors(DevView G, uint32_t u, uint32_t *out, uint64_t cap) {
  NbrList L = nbr_list(G, u);
  uint64_t lim = L.deg < cap ? L.deg : cap;
  for (uint64_t j = threadIdx.x + (uint64_t)blockIdx.x * blockDim.x; j < lim;
       j += (uint64_t)blockDim.x * gridDim.x)
    out[j] = L.at((uint32_t)j);
}

// |{w in N(s) n N(d) : w < min(s,d)}|, one thread per query (merge walk).
__global__ void k_count_common(DevView G, const uint32_t *s, const uint32_t *d, uint64_t q,
                               uint32_t *out) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= q) return;
  uint32_t a = s[i], b = d[i];
  if (a >= G.n || b >= G.n) {
    atomicOr(G.err, ERR_BAD_VERTEX);
    out[i] = 0;
    return;
  }
  uint32_t lim = a < b ? a : b;
  NbrList A = nbr_list(G, a), B = nbr_list(G, b);
  uint32_t ia = 0, ib = 0, c = 0;
  while (ia < A.deg && ib < B.deg) {
    uint32_t x = A.at(ia), y = B.at(ib);
    if (x >= lim || y >= lim) break;
    if (x == y) {
      c++;
      ia++;
      ib++;
    } else if (x < y) {
      ia++;
    } else {
      ib++;
    }
  }
  out[i] = c;
}

struct LoadDeg {
  const uint32_t *deg;
  __device__ uint64_t operator()(uint64_t i) const { return deg[i]; }
};

struct LoadMin {
  const uint32_t *d;
  __device__ uint64_t operator()(uint64_t i) const { return d[i] < K_INLINE ? d[i] : K_INLINE; }
};

__global__ void k_dump(DevView G, const uint64_t *off, uint32_t *tgt) {
  uint64_t w = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  uint32_t lane = threadIdx.x & 31;
  if (w >= G.n) return;
  uint32_t u = (uint32_t)w;
  NbrList L = nbr_list(G, u);
  uint64_t base = off[u];
  for (uint32_t j = lane; j < L.deg; j += 32) tgt[base + j] = L.at(j);
}

// Invariant checker: one warp per vertex, counts violations.
//  - list strictly increasing, entries < n
//  - non-hub: c2 == max(deg-16, 0) and segment inside [pbeg[u], pbeg[u+1])
//  - hub: c2 == 0; directory entries in key order with 1..256 elements per
//    block, prefixes and first keys equal to the blocks' counts and first
//    slots, owner u, the counts summing to deg-16 (no blocks when deg <= 16)
//  - pbeg non-decreasing, pbeg[n] == N
__global__ void k_check(DevView G, unsigned long long *bad) {
  uint64_t w = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  uint32_t lane = threadIdx.x & 31;
  if (w > G.n) return;
  uint32_t u = (uint32_t)w;
  if (u == G.n) {
    if (lane == 0 && G.pbeg[G.n] != G.N && G.N != 0) atomicAdd(bad, 1ull);
    return;
  }
  uint32_t nbad = 0;
  NbrList L = nbr_list(G, u);
  for (uint32_t j = lane; j < L.deg; j += 32) {
    uint32_t x = L.at(j);
    if (x >= G.n) nbad++;
    if (j > 0 && L.at(j - 1) >= x) nbad++;
  }
  const int32_t h = G.hub_of[u];
  const uint32_t d = G.deg[u];
  const uint32_t rest = d > K_INLINE ? d - K_INLINE : 0;
  if (h >= 0) {
    const uint64_t e0 = G.hub_dir0[h];
    const uint32_t nb = G.hub_nblk[h];
    uint32_t sum = 0;  // lane-local part of the element total
    for (uint32_t i = lane; i < nb; i += 32) {
      const uint32_t b = G.hdir[e0 + i];
      const uint32_t c = G.bcnt[b];
      const uint32_t next = i + 1 < nb ? G.hpre[e0 + i + 1] : rest;
      if (c == 0 || c > HUB_BLOCK) nbad++;
      if (next - G.hpre[e0 + i] != c) nbad++;
      if (G.bown[b] != u) nbad++;
      if (c && (G.bmin[b] != G.hslot[(uint64_t)b * HUB_BLOCK] || G.hkey[e0 + i] != G.bmin[b])) nbad++;
      sum += c;
    }
    sum = warp_sum(sum);
    if (lane == 0) {
      if (sum != rest) nbad++;
      if (nb && G.hpre[e0] != 0) nbad++;
      if (rest == 0 && nb != 0) nbad++;
      if (G.c2[u] != 0) nbad++;
      if (G.hub_vtx[h] != u) nbad++;
    }
  } else if (lane == 0) {
    if (G.c2[u] != rest) nbad++;
    if (G.pbeg[u] + G.c2[u] > G.pbeg[u + 1]) nbad++;
  }
  if (lane == 0 && G.pbeg[u] > G.pbeg[u + 1]) nbad++;
  nbad = warp_sum(nbad);
  if (lane == 0 && nbad) atomicAdd(bad, (unsigned long long)nbad);
}

void Graph::is_edge(const uint32_t *s_in, const uint32_t *d_in, uint64_t q, uint8_t *out,
                    uint32_t flags) {
  if (q == 0) return;
  if (!s_in || !d_in || !out) throw_error(TRC_ERR_INVALID, "null pointer");
  const uint32_t *s = to_device(*this, s_in, q, flags, s_in_src);
  const uint32_t *d = to_device(*this, d_in, q, flags, s_in_dst);
  uint8_t *o = (flags & TRC_DEVICE_PTR) ? out : s_flags.ensure(q);
  TRC_CUDA(cudaMemsetAsync(err.get(), 0, 4, stream));
  TRC_LAUNCH(prof, stream, "q_is_edge", ceil_div(q, 256), 256, 0, k_is_edge, view(), s, d, q, o);
  if (!(flags & TRC_DEVICE_PTR))
    TRC_CUDA(cudaMemcpyAsync(out, o, q, cudaMemcpyDeviceToHost, stream));
  uint32_t herr = 0;
  TRC_CUDA(cudaMemcpyAsync(&herr, err.get(), 4, cudaMemcpyDeviceToHost, stream));
  sync();
  if (herr) throw_error(TRC_ERR_INVALID, "vertex id out of range [0, n)");
}

void Graph::degree(const uint32_t *v_in, uint64_t q, uint32_t *out, uint32_t flags) {
  if (q == 0) return;
  if (!v_in || !out) throw_error(TRC_ERR_INVALID, "null pointer");
  const uint32_t *v = to_device(*this, v_in, q, flags, s_in_src);
  uint32_t *o = (flags & TRC_DEVICE_PTR) ? out : s_in_dst.ensure(q);
  TRC_CUDA(cudaMemsetAsync(err.get(), 0, 4, stream));
  TRC_LAUNCH(prof, stream, "q_degree", ceil_div(q, 256), 256, 0, k_degree, view(), v, q, o);
  if (!(flags & TRC_DEVICE_PTR))
    TRC_CUDA(cudaMemcpyAsync(out, o, q * 4, cudaMemcpyDeviceToHost, stream));
  uint32_t herr = 0;
  TRC_CUDA(cudaMemcpyAsync(&herr, err.get(), 4, cudaMemcpyDeviceToHost, stream));
  sync();
  if (herr) throw_error(TRC_ERR_INVALID, "vertex id out of range [0, n)");
}

uint64_t Graph::neighbors(uint32_t v, uint32_t *out, uint64_t cap, uint32_t flags) {
  if (v >= n) throw_error(TRC_ERR_INVALID, "vertex id out of range [0, n)");
  uint32_t d = 0;
  TRC_CUDA(cudaMemcpyAsync(&d, deg.get() + v, 4, cudaMemcpyDeviceToHost, stream));
  sync();
  uint64_t lim = d < cap ? d : cap;
  if (lim && !out) throw_error(TRC_ERR_INVALID, "null output");
  if (lim) {
    uint32_t *o = (flags & TRC_DEVICE_PTR) ? out : s_in_dst.ensure(lim);
    TRC_LAUNCH(prof, stream, "q_neighbors", ceil_div(lim, 256) < 1024 ? ceil_div(lim, 256) : 1024,
               256, 0, k_neighbors, view(), v, o, lim);
    if (!(flags & TRC_DEVICE_PTR))
      TRC_CUDA(cudaMemcpyAsync(out, o, lim * 4, cudaMemcpyDeviceToHost, stream));
    sync();
  }
  return d;
}

void Graph::count_common(const uint32_t *s_in, const uint32_t *d_in, uint64_t q, uint32_t *out,
                         uint32_t flags) {
  if (q == 0) return;
  if (!s_in || !d_in || !out) throw_error(TRC_ERR_INVALID, "null pointer");
  const uint32_t *s = to_device(*this, s_in, q, flags, s_in_src);
  const uint32_t *d = to_device(*this, d_in, q, flags, s_in_dst);
  uint32_t *o = (flags & TRC_DEVICE_PTR) ? out : s_tu.ensure(q);
  TRC_CUDA(cudaMemsetAsync(err.get(), 0, 4, stream));
  TRC_LAUNCH(prof, stream, "q_count_common", ceil_div(q, 128), 128, 0, k_count_common, view(), s, d,
             q, o);
  if (!(flags & TRC_DEVICE_PTR))
    TRC_CUDA(cudaMemcpyAsync(out, o, q * 4, cudaMemcpyDeviceToHost, stream));
  uint32_t herr = 0;
  TRC_CUDA(cudaMemcpyAsync(&herr, err.get(), 4, cudaMemcpyDeviceToHost, stream));
  sync();
  if (herr) throw_error(TRC_ERR_INVALID, "vertex id out of range [0, n)");
}

void Graph::dump_csr(uint64_t *offsets, uint32_t *targets, uint32_t flags) {
  if (!offsets || (m && !targets)) throw_error(TRC_ERR_INVALID, "null pointer");
  bool dev = flags & TRC_DEVICE_PTR;
  uint64_t *off = dev ? offsets : s_oOff.ensure((uint64_t)n + 1);
  uint32_t *tgt = dev ? targets : s_pma_next.ensure(m ? m : 1);
  uint64_t *t = tmp(scan_tmp_elems(n) + 4);
  exclusive_scan(LoadDeg{deg.get()}, n, off, t, stream, prof);
  TRC_LAUNCH(prof, stream, "q_dump", ceil_div((uint64_t)n * 32, 256), 256, 0, k_dump, view(), off,
             tgt);
  if (!dev) {
    TRC_CUDA(cudaMemcpyAsync(offsets, off, ((uint64_t)n + 1) * 8, cudaMemcpyDeviceToHost, stream));
    if (m) TRC_CUDA(cudaMemcpyAsync(targets, tgt, m * 4, cudaMemcpyDeviceToHost, stream));
  }
  sync();
  if (!dev) s_pma_next.reset();
}

uint64_t Graph::check() {
  uint64_t *c = s_cnt.get() + 20;
  TRC_CUDA(cudaMemsetAsync(c, 0, 8, stream));
  TRC_LAUNCH(prof, stream, "q_check", ceil_div(((uint64_t)n + 1) * 32, 256), 256, 0, k_check, view(),
             (unsigned long long *)c);
  uint64_t bad = read_u64(c);
  // host-side: directed edge count equals the sum of degrees
  uint64_t *t = tmp(scan_tmp_elems(n) + 4);
  uint64_t *off = s_oOff.ensure((uint64_t)n + 1);
  exclusive_scan(LoadDeg{deg.get()}, n, off, t, stream, prof);
  if (read_u64(off + n) != m) bad++;
  return bad;
}

uint64_t Graph::size_bytes() const {
  return deg.bytes() + inl.bytes() + c2.bytes() + pbeg.bytes() + hub_of.bytes() + pma.bytes() +
         hub_vtx.bytes() + hub_nblk.bytes() + hub_dir0.bytes() + hdir.bytes() + hpre.bytes() +
         hkey.bytes() + hslot.bytes() + bcnt.bytes() + bmin.bytes() + bown.bytes() + bfree.bytes();
}

void Graph::stats(trc_stats *o) {
  o->n = n;
  o->num_edges = m;
  o->pma_edges = tier2_total;
  o->pma_capacity = N;
  o->num_hubs = H;
  o->hub_blocks_used = pool_top - nfree;
  o->device_bytes = budget.used;
  o->pma_rebuilds = rebuilds;
  o->pma_window_rebalances = window_rebalances;
  o->last_keys = last[0];
  o->last_applied = last[1];
  o->last_touched = last[2];
  o->last_rewritten = last[3];
  o->last_gathered = last[4];
  o->last_written = last[5];
  o->last_windows = last[6];
  o->last_rebuild = last[7];
  o->last_hub_touched = hub_last[0];
  o->last_hub_local = hub_last[1];
  o->last_hub_rewritten = hub_last[2];
  o->last_hub_blocks_written = hub_last[3];
  o->last_hub_read = hub_last[4];
  o->last_hub_written = hub_last[5];
  o->hub_splits = hub_splits;
  o->hub_rewrites = hub_rewrites;
  o->hub_blocks_free = nfree;
  o->hub_absorbs = hub_absorbs;
  o->sort_retries = sort_retries;
  // inline = sum(min(deg,16)); hub = m - inline - tier2
  uint64_t *t = tmp(scan_tmp_elems(n) + 4);
  uint64_t *off = s_oOff.ensure((uint64_t)n + 1);
  exclusive_scan(LoadMin{deg.get()}, n, off, t, stream, prof, "stats_scan");
  o->inline_edges = read_u64(off + n);
  o->hub_edges = m - o->inline_edges - o->pma_edges;
}

}  // namespace trc
