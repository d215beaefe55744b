// tune.cu -- per-graph autotuner for the choices the reference fixes at
// compile time or leaves to a constant:
//   * the edgeMap direction threshold |F| >= n / divisor (reference 20,
//     include/Map.cpp:65-74): candidates 4..64, timed on BFS from the
//     maximum-degree vertex and three seeded non-isolated vertices;
//   * the PageRank block shape for degrees 17..cut: lanes per vertex (4, 8,
//     16) and the cut (32, 64, 128) above which a warp takes a vertex,
//     timed on two iterations;
//   * the PMA leaf, the smallest window the rebalancer considers (2^x vertex
//     segments, x in 1..5; the reference sizes its leaves from the capacity,
//     src/PMA.cc:2961-2962), timed by inserting and then removing a sample
//     batch of absent edges, which leaves the edge set unchanged.
// Each choice is kept in the graph (trc_get_tuning / trc_set_tuning) and
// applies to later calls; results stay exact (BFS, PMA) or within FP64
// reordering (PageRank's summation grouping follows the lane count).
#include <algorithm>
#include <chrono>
#include <random>
#include <vector>

#include "graph.cuh"

namespace trc {

namespace {
double wall_ms() {
  return std::chrono::duration<double, std::milli>(
             std::chrono::steady_clock::now().time_since_epoch())
      .count();
}
}  // namespace

void Graph::autotune(uint32_t what, const uint32_t *src, const uint32_t *dst, uint64_t k,
                     uint32_t flags, double *ms_out) {
  const bool prof_was = prof.on;
  prof.on = false;
  ms_out[0] = ms_out[1] = ms_out[2] = 0.0;
  try {
    // -------------------------------------------------- push / pull threshold
    if ((what & TRC_TUNE_PUSH_PULL) && m > 0) {
      std::vector<uint32_t> hdeg(n);
      TRC_CUDA(cudaMemcpyAsync(hdeg.data(), deg.get(), (uint64_t)n * 4, cudaMemcpyDeviceToHost,
                               stream));
      sync();
      std::vector<uint32_t> nz;
      for (uint32_t v = 0; v < n; v++)
        if (hdeg[v]) nz.push_back(v);
      std::vector<uint32_t> srcs;
      srcs.push_back((uint32_t)(std::max_element(hdeg.begin(), hdeg.end()) - hdeg.begin()));
      std::mt19937_64 rng(0x5EED ^ n);
      for (int i = 0; i < 3 && !nz.empty(); i++) srcs.push_back(nz[rng() % nz.size()]);
      DBuf<int32_t> pb;
      DBuf<uint32_t> lb;
      pb.bind(&budget);
      lb.bind(&budget);
      int32_t *par = pb.alloc_exact(n);
      uint32_t *lv = lb.alloc_exact(n);
      const uint32_t cand[] = {4, 8, 12, 16, 20, 32, 64};
      const uint32_t keep = tuned.push_pull_divisor;
      double best = 1e30;
      uint32_t best_d = keep;
      bfs(srcs[0], par, lv, TRC_DEVICE_PTR);  // warm (class lists, scratch)
      for (uint32_t d : cand) {
        tuned.push_pull_divisor = d;
        double t = 1e30;
        for (int rep = 0; rep < 2; rep++) {
          double t0 = wall_ms();
          for (uint32_t s : srcs) bfs(s, par, lv, TRC_DEVICE_PTR);
          t = std::min(t, wall_ms() - t0);
        }
        if (t < best) {
          best = t;
          best_d = d;
        }
      }
      tuned.push_pull_divisor = best_d;
      ms_out[0] = best / (double)srcs.size();
    }
    // -------------------------------------------------- PageRank block shape
    if ((what & TRC_TUNE_PAGERANK) && m > 0) {
      DBuf<double> a, b, o;
      a.bind(&budget);
      b.bind(&budget);
      o.bind(&budget);
      double *p0 = a.alloc_exact(n), *p1 = b.alloc_exact(n), *out = o.alloc_exact(n);
      const Tuning keep = tuned;
      double best = 1e30;
      Tuning best_t = keep;
      cudaEvent_t e0, e1;
      TRC_CUDA(cudaEventCreate(&e0));
      TRC_CUDA(cudaEventCreate(&e1));
      for (uint32_t cut : {32u, 64u, 128u}) {
        tuned.pr_group_cut = cut;
        lists.version = ~0ull;  // the class lists depend on the cut
        ensure_lists();
        for (uint32_t lanes : {4u, 8u, 16u}) {
          tuned.pr_group_lanes = lanes;
          pagerank_launch(1, 0.0, p0, p1, out, stream);  // warm
          float t = 1e30f;
          for (int rep = 0; rep < 2; rep++) {
            TRC_CUDA(cudaEventRecord(e0, stream));
            pagerank_launch(2, 0.0, p0, p1, out, stream);
            TRC_CUDA(cudaEventRecord(e1, stream));
            TRC_CUDA(cudaEventSynchronize(e1));
            float ms = 0;
            TRC_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            t = std::min(t, ms);
          }
          if (t < best) {
            best = t;
            best_t = tuned;
          }
        }
      }
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      tuned.pr_group_cut = best_t.pr_group_cut;
      tuned.pr_group_lanes = best_t.pr_group_lanes;
      lists.version = ~0ull;
      ms_out[1] = best / 2.0;
    }
    // -------------------------------------------------- PMA leaf
    if ((what & TRC_TUNE_PMA) && k > 0 && src && dst) {
      // the sample as directed edges, validated, without self loops and
      // without edges already present, deduplicated
      std::vector<uint32_t> hs(k), hd(k);
      if (flags & TRC_DEVICE_PTR) {
        TRC_CUDA(cudaMemcpyAsync(hs.data(), src, k * 4, cudaMemcpyDeviceToHost, stream));
        TRC_CUDA(cudaMemcpyAsync(hd.data(), dst, k * 4, cudaMemcpyDeviceToHost, stream));
        sync();
      } else {
        std::copy(src, src + k, hs.begin());
        std::copy(dst, dst + k, hd.begin());
      }
      std::vector<uint64_t> keys;
      keys.reserve(2 * k);
      for (uint64_t i = 0; i < k; i++) {
        if (hs[i] >= n || hd[i] >= n) throw_error(TRC_ERR_INVALID, "sample vertex out of range");
        if (hs[i] == hd[i]) continue;
        keys.push_back(((uint64_t)hs[i] << 32) | hd[i]);
        if (flags & TRC_SYMMETRIZE) keys.push_back(((uint64_t)hd[i] << 32) | hs[i]);
      }
      std::sort(keys.begin(), keys.end());
      keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
      std::vector<uint32_t> qs(keys.size()), qd(keys.size());
      for (size_t i = 0; i < keys.size(); i++) {
        qs[i] = (uint32_t)(keys[i] >> 32);
        qd[i] = (uint32_t)keys[i];
      }
      std::vector<uint8_t> present(keys.size());
      if (!keys.empty()) is_edge(qs.data(), qd.data(), keys.size(), present.data(), 0);
      std::vector<uint32_t> as, ad;
      for (size_t i = 0; i < keys.size(); i++)
        if (!present[i]) {
          as.push_back(qs[i]);
          ad.push_back(qd[i]);
        }
      if (!as.empty()) {
        DBuf<uint32_t> ds, dd;
        ds.bind(&budget);
        dd.bind(&budget);
        uint32_t *s_d = ds.alloc_exact(as.size()), *d_d = dd.alloc_exact(as.size());
        TRC_CUDA(cudaMemcpyAsync(s_d, as.data(), as.size() * 4, cudaMemcpyHostToDevice, stream));
        TRC_CUDA(cudaMemcpyAsync(d_d, ad.data(), ad.size() * 4, cudaMemcpyHostToDevice, stream));
        sync();
        const uint32_t keep = tuned.pma_leaf_log;
        double best = 1e30;
        uint32_t best_l = keep;
        for (uint32_t leaf = 1; leaf <= 5; leaf++) {
          tuned.pma_leaf_log = leaf;
          double t = 1e30;
          for (int rep = 0; rep < 2; rep++) {
            double t0 = wall_ms();
            apply_batch(s_d, d_d, as.size(), TRC_DEVICE_PTR, true);
            double t1 = wall_ms();
            apply_batch(s_d, d_d, as.size(), TRC_DEVICE_PTR, false);
            t = std::min(t, t1 - t0);
          }
          if (t < best) {
            best = t;
            best_l = leaf;
          }
        }
        tuned.pma_leaf_log = best_l;
        ms_out[2] = best;
      }
    }
  } catch (...) {
    prof.on = prof_was;
    throw;
  }
  prof.on = prof_was;
}

}  // namespace trc
