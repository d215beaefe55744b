// pagerank.cu -- PR_S over a degree-ordered CSR snapshot.
//
// Replaces PR_S<double> (include/Pagerank.h:105-184): p0 = 1/n; per iteration
// p <- p/deg (PR_Vertex, :60-69), then the dense pull p_next[u] = sum over
// N(u) of p[v] (map_dense_vs_all, include/graph.h:1384-1487, PR_F::update,
// :39-44); damping 0 is the reference, 0 < damping < 1 the textbook form.
//
// Every iteration gathers p[v]/deg(v) (8 bytes) once per edge, at random; on
// a graph whose rank vector exceeds L2 those gathers, one 32-byte sector for
// 8 useful bytes, bound the pull.  So PageRank runs on a snapshot of the
// graph, rebuilt when the graph changes: the non-isolated vertices relabelled
// by degree, highest first, and their lists (neighbour ids relabelled, in the
// original sorted order) as one CSR.  The most gathered values are then the
// first entries of the rank vector, packed into few sectors that stay in L1
// and L2.  The lists are read once per iteration with streaming loads,
// contiguous for every vertex with no tier dispatch, by a lane group sized
// to the degree class: a CTA per vertex above 4096 neighbours, a warp above
// the lane-group cut, a lane group (4, 8 or 16) above 16, four lanes below.
// Classes are contiguous ranges of the relabelled ids.  Results are
// scattered back to the original ids on the last iteration.
#include <algorithm>
#include <cstring>

#include "graph.cuh"

namespace trc {

constexpr int PRT = 256;                 // threads per CTA of the pull kernels
constexpr uint32_t PR_BLOCK_DEG = 4096;  // above: a CTA per vertex

struct PRSArgs {
  const uint64_t *off;
  const uint32_t *adj;
  const uint32_t *perm;  // relabelled id -> original id
  const double *pc;      // p/deg of the previous iteration (relabelled order)
  double *pn;            // p/deg of this iteration
  double *out;           // final ranks (original order), last iteration
  double damping, base;
  int last;
};

__device__ __forceinline__ void prs_store(const PRSArgs &a, uint64_t r, uint32_t d, double sum) {
  const double val = a.damping > 0.0 ? a.base + a.damping * sum : sum;
  a.pn[r] = val / (double)d;
  if (a.last) a.out[a.perm[r]] = val;
}

// GS lanes per vertex over relabelled ids [r0, r1), one group per vertex;
// each lane issues U independent list loads, then U gathers.
template <int GS>
__global__ void __launch_bounds__(PRT) k_prs_group(PRSArgs a, uint64_t r0, uint64_t r1) {
  constexpr int U = 8;
  const uint32_t lg = threadIdx.x & (GS - 1);
  const uint32_t lane = threadIdx.x & 31;
  const unsigned mask = GS == 32 ? 0xFFFFFFFFu : (((1u << GS) - 1u) << (lane & ~(uint32_t)(GS - 1)));
  const uint64_t r = r0 + ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / GS;
  if (r >= r1) return;  // whole groups leave together
  const uint64_t e0 = a.off[r], e1 = a.off[r + 1];
  double sum = 0.0;
  for (uint64_t e = e0 + lg; e < e1; e += (uint64_t)GS * U) {
    uint32_t x[U];
#pragma unroll
    for (int k = 0; k < U; k++) {
      const uint64_t ee = e + (uint64_t)k * GS;
      x[k] = ee < e1 ? __ldcs(a.adj + ee) : NONE32;
    }
#pragma unroll
    for (int k = 0; k < U; k++)
      if (x[k] != NONE32) sum += __ldg(a.pc + x[k]);
  }
#pragma unroll
  for (int o = GS / 2; o > 0; o >>= 1) sum += __shfl_xor_sync(mask, sum, o);
  if (lg == 0) prs_store(a, r, (uint32_t)(e1 - e0), sum);
}

// A CTA per vertex over [r0, r1) (the largest degrees).
__global__ void __launch_bounds__(PRT) k_prs_block(PRSArgs a, uint64_t r0) {
  __shared__ double ws[PRT / 32];
  const uint64_t r = r0 + blockIdx.x;
  const uint64_t e0 = a.off[r], e1 = a.off[r + 1];
  double sum = 0.0;
  for (uint64_t e = e0 + threadIdx.x; e < e1; e += blockDim.x) sum += __ldg(a.pc + __ldcs(a.adj + e));
  sum = warp_sum(sum);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = sum;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < PRT / 32; w++) t += ws[w];
    prs_store(a, r, (uint32_t)(e1 - e0), t);
  }
}

__global__ void k_prs_init(const uint64_t *off, uint64_t na, double p0, double *pdiv) {
  const uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r < na) pdiv[r] = p0 / (double)(off[r + 1] - off[r]);
}

// isolated vertices: never gathered; their final rank is the constant term
__global__ void k_prs_isolated(const uint32_t *deg, uint32_t n, double iso, double *out) {
  const uint64_t u = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (u < n && deg[u] == 0) out[u] = iso;
}

// ---------------------------------------------------------------- snapshot

struct DegKeyPred {
  const uint32_t *deg;
  __device__ bool operator()(uint64_t i) const { return deg[i] > 0; }
};

// (complement of the degree) << 32 | id: ascending = degree descending, ids
// ascending within a degree (the sort is stable on the id order)
struct DegKeyVal {
  const uint32_t *deg;
  __device__ uint64_t operator()(uint64_t i) const {
    return ((uint64_t)(0xFFFFFFFFu - deg[i]) << 32) | (uint32_t)i;
  }
};

__global__ void k_prs_perm(const uint64_t *keys, uint64_t na, uint32_t *perm, uint32_t *inv,
                           uint32_t *dsort) {
  const uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= na) return;
  const uint64_t k = keys[r];
  const uint32_t u = (uint32_t)k;
  perm[r] = u;
  inv[u] = (uint32_t)r;
  dsort[r] = 0xFFFFFFFFu - (uint32_t)(k >> 32);
}

struct LoadDsort {
  const uint32_t *d;
  __device__ uint64_t operator()(uint64_t i) const { return d[i]; }
};

// warp per relabelled vertex: its list with relabelled neighbour ids
__global__ void k_prs_fill(DevView G, const uint32_t *perm, const uint32_t *inv,
                           const uint64_t *off, uint64_t na, uint32_t *adj) {
  const uint64_t w = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t lane = threadIdx.x & 31;
  if (w >= na) return;
  const NbrList L = nbr_list(G, perm[w]);
  uint32_t *dst = adj + off[w];
  for (uint32_t j = lane; j < L.deg; j += 32) dst[j] = inv[L.at(j)];
}

// class boundaries: the number of vertices with degree above each threshold
// (dsort descending)
__global__ void k_prs_bounds(const uint32_t *dsort, uint64_t na, uint32_t t0, uint32_t t1,
                             uint32_t t2, uint64_t *out) {
  const uint32_t t = threadIdx.x == 0 ? t0 : threadIdx.x == 1 ? t1 : t2;
  if (threadIdx.x >= 3) return;
  uint64_t lo = 0, hi = na;  // first index with dsort <= t
  while (lo < hi) {
    const uint64_t mid = (lo + hi) >> 1;
    if (dsort[mid] > t) lo = mid + 1;
    else hi = mid;
  }
  out[threadIdx.x] = lo;
}

void Graph::ensure_pr_snapshot() {
  PRSnap &S = prs;
  if (S.version != version) {
    S.version = ~0ull;
    S.cut = 0;
    DBuf<uint64_t> ka, kb, tb, cb;
    for (auto *b : {&ka, &kb, &tb, &cb}) b->bind(&budget);
    uint64_t *A = ka.alloc_exact(n), *B = kb.alloc_exact(n);
    uint64_t *t = tb.alloc_exact(std::max(radix_tmp_elems(n), select_tmp_elems(n)) + 4);
    uint64_t *c = cb.alloc_exact(4);
    select_if(DegKeyPred{deg.get()}, DegKeyVal{deg.get()}, n, A, c, t, stream, prof, "prs_keys");
    const uint64_t na = read_u64(c);
    const int shifts[4] = {32, 40, 48, 56};
    const uint64_t *sorted = radix_sort_u64_shifts(A, B, na, shifts, 4, t, stream, prof, err.get());
    uint32_t *perm = S.perm.ensure(na + 1), *inv = S.inv.ensure(n), *dsort = S.dsort.ensure(na + 1);
    TRC_LAUNCH(prof, stream, "prs_perm", ceil_div(na, 256), 256, 0, k_prs_perm, sorted, na, perm,
               inv, dsort);
    uint64_t *off = S.off.ensure(na + 1);
    exclusive_scan(LoadDsort{dsort}, na, off, t, stream, prof, "prs_off");
    const uint64_t mm = read_u64(off + na);
    if (mm != m) throw_error(TRC_ERR_STATE, "PageRank snapshot: degree sum differs from the edge count");
    uint32_t *adj = S.adj.ensure(mm + 1);
    TRC_LAUNCH(prof, stream, "prs_fill", ceil_div(na * 32, 256), 256, 0, k_prs_fill, view(), perm,
               inv, off, na, adj);
    S.na = na;
    S.version = version;
  }
  if (S.cut != tuned.pr_group_cut) {
    uint64_t *b = s_cnt.get() + 20;
    TRC_LAUNCH(prof, stream, "prs_bounds", 1, 32, 0, k_prs_bounds, S.dsort.get(), S.na,
               PR_BLOCK_DEG, std::max<uint32_t>(tuned.pr_group_cut, K_INLINE), K_INLINE, b);
    uint64_t h[3];
    TRC_CUDA(cudaMemcpyAsync(h, b, sizeof(h), cudaMemcpyDeviceToHost, stream));
    sync();
    S.rb = h[0];  // [0, rb): CTA per vertex
    S.rw = h[1];  // [rb, rw): a warp
    S.rg = h[2];  // [rw, rg): a lane group; [rg, na): four lanes
    S.cut = tuned.pr_group_cut;
  }
}

// ---------------------------------------------------------------- iterations

void Graph::pagerank(uint32_t iters, double damping, double *ranks, uint32_t flags) {
  if (!ranks) throw_error(TRC_ERR_INVALID, "null output");
  if (damping < 0.0 || damping >= 1.0) throw_error(TRC_ERR_INVALID, "damping must be in [0,1)");
  const bool dev = flags & TRC_DEVICE_PTR;
  DBuf<double> pa, pb, ob;
  pa.bind(&budget);
  pb.bind(&budget);
  ob.bind(&budget);
  double *out = dev ? ranks : ob.alloc_exact(n);
  if (iters == 0) {
    // the reference returns the initial vector 1/n (include/Pagerank.h:137-141)
    std::vector<double> h(n, 1.0 / (double)n);
    TRC_CUDA(cudaMemcpyAsync(out, h.data(), (uint64_t)n * 8, cudaMemcpyHostToDevice, stream));
    sync();
  } else {
    ensure_pr_snapshot();
    double *p0 = pa.alloc_exact(prs.na + 1), *p1 = pb.alloc_exact(prs.na + 1);
    pagerank_launch(iters, damping, p0, p1, out, stream);
  }
  if (!dev) TRC_CUDA(cudaMemcpyAsync(ranks, out, (uint64_t)n * 8, cudaMemcpyDeviceToHost, stream));
  sync();
}

void Graph::pr_kernels(uint32_t iters, double damping, double *p0, double *p1, double *out,
                       cudaStream_t s) {
  const double one_over_n = 1.0 / (double)n;
  const double base = (1.0 - damping) / (double)n;
  const PRSnap &S = prs;
  TRC_LAUNCH(prof, s, "pr_isolated", ceil_div(n, 256), 256, 0, k_prs_isolated, deg.get(), n,
             damping > 0.0 ? base : 0.0, out);
  if (S.na == 0) return;
  TRC_LAUNCH(prof, s, "pr_init", ceil_div(S.na, 256), 256, 0, k_prs_init, S.off.get(), S.na,
             one_over_n, p0);
  for (uint32_t it = 0; it < iters; it++) {
    PRSArgs a{S.off.get(), S.adj.get(), S.perm.get(), p0, p1, out, damping, base,
              it + 1 == iters ? 1 : 0};
    if (S.rb) TRC_LAUNCH(prof, s, "pr_block", S.rb, PRT, 0, k_prs_block, a, 0);
    if (S.rw > S.rb)
      TRC_LAUNCH(prof, s, "pr_warp", ceil_div((S.rw - S.rb) * 32, PRT), PRT, 0, k_prs_group<32>, a,
                 S.rb, S.rw);
    if (S.rg > S.rw) {
      const uint64_t nv = S.rg - S.rw;
      switch (tuned.pr_group_lanes) {
        case 4:
          TRC_LAUNCH(prof, s, "pr_group4", ceil_div(nv * 4, PRT), PRT, 0, k_prs_group<4>, a, S.rw,
                     S.rg);
          break;
        case 16:
          TRC_LAUNCH(prof, s, "pr_group16", ceil_div(nv * 16, PRT), PRT, 0, k_prs_group<16>, a,
                     S.rw, S.rg);
          break;
        default:
          TRC_LAUNCH(prof, s, "pr_group8", ceil_div(nv * 8, PRT), PRT, 0, k_prs_group<8>, a, S.rw,
                     S.rg);
      }
    }
    if (S.na > S.rg)
      TRC_LAUNCH(prof, s, "pr_small", ceil_div((S.na - S.rg) * 4, PRT), PRT, 0, k_prs_group<4>, a,
                 S.rg, S.na);
    std::swap(p0, p1);
  }
}

// The iteration loop is replayed from a CUDA graph: captured once per
// (iteration count, buffers, snapshot) and patched with cudaGraphExecUpdate
// when only kernel arguments changed.  With the per-kernel profiler on,
// kernels are launched directly so that each gets its own events.  Requires
// a current snapshot (ensure_pr_snapshot) and iters >= 1; nothing is
// allocated or synchronised, so it may run on a second stream.
void Graph::pagerank_launch(uint32_t iters, double damping, double *p0, double *p1, double *out,
                            cudaStream_t s) {
  if (prs.version != version) throw_error(TRC_ERR_STATE, "PageRank snapshot is not current");
  if (prof.on || !use_graphs || iters < 2) {
    pr_kernels(iters, damping, p0, p1, out, s);
    return;
  }
  uint64_t dbits;
  memcpy(&dbits, &damping, 8);
  const uint64_t key[PRGraphCache::KEY] = {iters, dbits, (uint64_t)p0, (uint64_t)p1, (uint64_t)out,
                                           prs.version, (uint64_t)prs.adj.get(), prs.na, prs.rb,
                                           prs.rw ^ (prs.rg << 32), (uint64_t)s,
                                           tuned.pr_group_lanes, 0};
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

}  // namespace trc
