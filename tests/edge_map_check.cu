// edge_map_check.cu -- the reference's BFS, CC and PageRank written against
// the generic edgeMap / vertexMap layer (include/terrace_b200_edge_map.cuh)
// with the reference's functors (include/BFS.h:27-39, include/Components.h:
// 24-117, include/Pagerank.h:31-98).  Built by tests/test_edge_map.py into a
// small shared library and compared with the built-in entry points.
#include <cstdint>
#include <vector>

#include "terrace_b200_edge_map.cuh"

using namespace terrace;

namespace {

struct BFS_F {
  int32_t *Parents;
  uint32_t *Level;
  uint32_t cur;
  __device__ bool update(uint32_t s, uint32_t d) {
    if (Parents[d] == -1) {
      Parents[d] = (int32_t)s;
      Level[d] = cur + 1;
      return true;
    }
    return false;
  }
  __device__ bool updateAtomic(uint32_t s, uint32_t d) {
    if (atomicCAS(&Parents[d], -1, (int32_t)s) == -1) {
      Level[d] = cur + 1;
      return true;
    }
    return false;
  }
  __device__ bool cond(uint32_t d) { return Parents[d] == -1; }
};

struct CC_Vertex_F {
  uint32_t *IDs, *prevIDs;
  __device__ bool operator()(uint32_t i) {
    prevIDs[i] = IDs[i];
    return true;
  }
};

struct CC_F {
  uint32_t *IDs, *prevIDs;
  __device__ bool update(uint32_t s, uint32_t d) {
    uint32_t origID = IDs[d];
    if (IDs[s] < origID) {
      IDs[d] = IDs[s];
      if (origID == prevIDs[d]) return true;
    }
    return false;
  }
  __device__ bool updateAtomic(uint32_t s, uint32_t d) {
    uint32_t origID = IDs[d];
    uint32_t v = IDs[s];
    bool wrote = atomicMin(&IDs[d], v) > v;  // writeMin, include/parallel_util.h:18-24
    return wrote && origID == prevIDs[d];
  }
  __device__ bool cond(uint32_t) { return true; }
};

struct PR_F {
  const double *p_curr;
  double *p_next;
  __device__ bool update(uint32_t s, uint32_t d) {
    p_next[d] += p_curr[s];
    return true;
  }
  __device__ bool updateAtomic(uint32_t s, uint32_t d) {
    atomicAdd(&p_next[d], p_curr[s]);
    return true;
  }
  __device__ bool cond(uint32_t) { return true; }
};

struct PR_Vertex {
  double *p_curr;
  const uint32_t *deg;
  __device__ bool operator()(uint32_t i) {
    p_curr[i] = p_curr[i] / deg[i];
    return true;
  }
};

struct PR_Vertex_Reset {
  double *p;
  __device__ bool operator()(uint32_t i) {
    p[i] = 0.0;
    return true;
  }
};

__global__ void fill_u32(uint32_t *a, uint32_t n, uint32_t v, int iota) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) a[i] = iota ? (uint32_t)i : v;
}
__global__ void fill_f64(double *a, uint32_t n, double v) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) a[i] = v;
}

template <typename T>
T *dalloc(uint64_t n) {
  T *p = nullptr;
  cudaMalloc(&p, sizeof(T) * (n ? n : 1));
  return p;
}

}  // namespace

extern "C" int em_bfs(trc_graph *g, uint32_t src, int32_t *parents_h, uint32_t *levels_h) {
  try {
    DeviceGraph dg = device_graph(g);
    uint32_t n = dg.v.n;
    cudaStream_t s = static_cast<cudaStream_t>(dg.v.stream);
    int32_t *par = dalloc<int32_t>(n);
    uint32_t *lv = dalloc<uint32_t>(n);
    fill_u32<<<(n + 255) / 256, 256, 0, s>>>((uint32_t *)par, n, 0xFFFFFFFFu, 0);
    fill_u32<<<(n + 255) / 256, 256, 0, s>>>(lv, n, 0xFFFFFFFFu, 0);
    int32_t ps = (int32_t)src;
    uint32_t zero = 0;
    cudaMemcpyAsync(par + src, &ps, 4, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(lv + src, &zero, 4, cudaMemcpyHostToDevice, s);
    cudaStreamSynchronize(s);
    // BFS_with_edge_map (include/BFS.h:41-84)
    VertexSubset frontier(src, n, s);
    uint32_t level = 0;
    while (frontier.not_empty()) {
      VertexSubset next = edgeMap(g, frontier, BFS_F{par, lv, level}, true);
      frontier = std::move(next);
      level++;
    }
    cudaMemcpy(parents_h, par, 4ull * n, cudaMemcpyDeviceToHost);
    cudaMemcpy(levels_h, lv, 4ull * n, cudaMemcpyDeviceToHost);
    cudaFree(par);
    cudaFree(lv);
    return 0;
  } catch (const std::exception &) {
    return 1;
  }
}

extern "C" int em_cc(trc_graph *g, uint32_t *labels_h) {
  try {
    DeviceGraph dg = device_graph(g);
    uint32_t n = dg.v.n;
    cudaStream_t s = static_cast<cudaStream_t>(dg.v.stream);
    uint32_t *ids = dalloc<uint32_t>(n), *prev = dalloc<uint32_t>(n);
    fill_u32<<<(n + 255) / 256, 256, 0, s>>>(ids, n, 0, 1);
    // CC (include/Components.h:92-120)
    VertexSubset active(0, n, true, s);
    while (active.not_empty()) {
      vertexMap(active, CC_Vertex_F{ids, prev}, false);
      VertexSubset next = edgeMap(g, active, CC_F{ids, prev}, true);
      active = std::move(next);
    }
    cudaMemcpy(labels_h, ids, 4ull * n, cudaMemcpyDeviceToHost);
    cudaFree(ids);
    cudaFree(prev);
    return 0;
  } catch (const std::exception &) {
    return 1;
  }
}

extern "C" int em_pagerank(trc_graph *g, uint32_t iters, double *out_h) {
  try {
    DeviceGraph dg = device_graph(g);
    uint32_t n = dg.v.n;
    cudaStream_t s = static_cast<cudaStream_t>(dg.v.stream);
    double *pc = dalloc<double>(n), *pn = dalloc<double>(n);
    fill_f64<<<(n + 255) / 256, 256, 0, s>>>(pc, n, 1.0 / (double)n);
    // PR_S<double> (include/Pagerank.h:105-184)
    VertexSubset all(0, n, true, s);
    for (uint32_t it = 0; it < iters; it++) {
      vertexMap(all, PR_Vertex{pc, dg.v.deg}, false);
      vertexMap(all, PR_Vertex_Reset{pn}, false);
      edgeMap(g, all, PR_F{pc, pn}, false);
      std::swap(pc, pn);
    }
    cudaMemcpy(out_h, pc, 8ull * n, cudaMemcpyDeviceToHost);
    cudaFree(pc);
    cudaFree(pn);
    return 0;
  } catch (const std::exception &) {
    return 1;
  }
}
