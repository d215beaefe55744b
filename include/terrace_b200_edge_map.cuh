// terrace_b200_edge_map.cuh -- generic edgeMap / vertexMap over VertexSubset
// for user device functors (compile with nvcc, sm_100a).
//
// The reference's traversal layer (include/Map.cpp:7-108,
// include/VertexSubset.cpp:5-248) takes a functor with
//     bool update(uint32_t s, uint32_t d);        // dense (pull), exclusive
//     bool updateAtomic(uint32_t s, uint32_t d);  // sparse (push), concurrent
//     bool cond(uint32_t d);
// and a VertexSubset frontier (sparse queue, dense bitmap or "all").  This
// header keeps that contract with __device__ functors, run over the graph's
// tiers on the GPU:
//   * sparse: one warp per frontier vertex; for every neighbour d with
//     f.cond(d), f.updateAtomic(s, d) == true puts d in the output queue
//     (Graph::map_sparse, include/graph.h:1287-1382);
//   * dense: one thread per vertex d with f.cond(d); neighbours s in sorted
//     order, f.update(s, d) for s in the frontier, stopping as soon as
//     f.cond(d) is false (map_dense_vs_not_all / map_dense_vs_all,
//     include/graph.h:1384-1613);
//   * dense iff n / threshold <= |frontier| (include/Map.cpp:65-74).
// Functors are copied by value into the kernels, as the reference copies F.
// The built-in trc_bfs / trc_pagerank / ... use specialised kernels; this
// layer is for user algorithms.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <utility>

#include "terrace_b200.hpp"

namespace terrace {

namespace detail {
inline void cuda_ok(cudaError_t e, const char *what) {
  if (e != cudaSuccess)
    throw Error(TRC_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}
}  // namespace detail

// Device-side view of the graph: degree and neighbour r of u (sorted order).
struct DeviceGraph {
  trc_device_view v;
  __device__ __forceinline__ uint32_t num_vertices() const { return v.n; }
  __device__ __forceinline__ uint32_t degree(uint32_t u) const { return v.deg[u]; }
  __device__ __forceinline__ uint32_t neighbor(uint32_t u, uint32_t r) const {
    if (r < v.inline_slots) return v.inl[(uint64_t)u * v.inline_slots + r];
    r -= v.inline_slots;
    int32_t h = v.hub_of[u];
    if (h < 0) return v.pma[v.pbeg[u] + r];
    // the hub's directory: the block whose element prefix is the largest <= r
    const uint64_t e0 = v.hub_dir0[h];
    uint32_t lo = 0, hi = v.hub_nblk[h];
    while (hi - lo > 1) {
      uint32_t mid = (lo + hi) >> 1;
      if (v.hub_pre[e0 + mid] <= r) lo = mid;
      else hi = mid;
    }
    return v.hslot[(uint64_t)v.hub_dir[e0 + lo] * v.hub_block + (r - v.hub_pre[e0 + lo])];
  }
};

inline DeviceGraph device_graph(trc_graph *g) {
  trc_device_view dv;
  check(trc_get_device_view(g, &dv));
  return DeviceGraph{dv};
}
inline DeviceGraph device_graph(Graph &G) { return device_graph(G.handle()); }

// Device-side view of a frontier.
struct SubsetView {
  uint32_t n;
  int all, sparse;
  const uint32_t *queue;  // sparse entries
  const uint32_t *bits;   // dense bitmap, n bits
  __device__ __forceinline__ bool has(uint32_t v) const {
    return all || ((bits[v >> 5] >> (v & 31)) & 1u);
  }
};

namespace detail {
__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

template <class F>
__global__ void em_sparse(DeviceGraph G, const uint32_t *q, uint32_t nq, F f, int output,
                          uint32_t *outq, uint32_t *outcnt) {
  uint64_t w = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  uint32_t lane = threadIdx.x & 31;
  if (w >= nq) return;
  uint32_t s = q[w];
  uint32_t deg = G.degree(s);
  for (uint32_t j0 = 0; j0 < deg; j0 += 32) {
    uint32_t j = j0 + lane;
    bool win = false;
    uint32_t d = 0;
    if (j < deg) {
      d = G.neighbor(s, j);
      win = f.cond(d) && f.updateAtomic(s, d);
    }
    if (output) {
      uint32_t m = __ballot_sync(0xFFFFFFFFu, win);
      uint32_t base = 0;
      if (m) {
        uint32_t leader = __ffs(m) - 1;
        if (lane == leader) base = atomicAdd(outcnt, __popc(m));
        base = __shfl_sync(0xFFFFFFFFu, base, leader);
      }
      if (win) outq[base + __popc(m & lanemask_lt())] = d;
    }
  }
}

template <class F>
__global__ void em_dense(DeviceGraph G, SubsetView in, F f, int output, uint32_t *outbits) {
  uint64_t d64 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (d64 >= G.num_vertices()) return;
  uint32_t d = (uint32_t)d64;
  if (!f.cond(d)) return;
  uint32_t deg = G.degree(d);
  for (uint32_t r = 0; r < deg; r++) {
    uint32_t s = G.neighbor(d, r);
    if (in.has(s) && f.update(s, d) && output) atomicOr(outbits + (d >> 5), 1u << (d & 31));
    if (!f.cond(d)) return;
  }
}

template <class F>
__global__ void vm_kernel(SubsetView in, uint32_t count, F f, int output, uint32_t *outq,
                          uint32_t *outcnt, uint32_t *outbits) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  uint32_t v = in.sparse ? in.queue[i] : (uint32_t)i;
  if (!in.sparse && !in.has(v)) return;
  bool r = f(v);
  if (!output || !r) return;
  if (in.sparse) outq[atomicAdd(outcnt, 1u)] = v;
  else atomicOr(outbits + (v >> 5), 1u << (v & 31));
}

static __global__ void bits_to_queue(const uint32_t *bits, uint32_t n, uint32_t *q, uint32_t *cnt) {
  uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (v < n && ((bits[v >> 5] >> (v & 31)) & 1u)) q[atomicAdd(cnt, 1u)] = (uint32_t)v;
}

static __global__ void queue_to_bits(const uint32_t *q, uint32_t nq, uint32_t *bits) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nq) atomicOr(bits + (q[i] >> 5), 1u << (q[i] & 31));
}

static __global__ void popcount_bits(const uint32_t *bits, uint64_t words, uint32_t *cnt) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t c = i < words ? __popc(bits[i]) : 0u;
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xFFFFFFFFu, c, o);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(cnt, c);
}

inline unsigned blocks(uint64_t work, unsigned bs) { return (unsigned)((work + bs - 1) / bs); }
}  // namespace detail

// VertexSubset (include/VertexSubset.cpp): "all", a sparse device queue, or
// a dense device bitmap; move-only.
class VertexSubset {
 public:
  VertexSubset() = default;
  // VertexSubset(e, max_el): the single vertex e, sparse.
  VertexSubset(uint32_t e, uint32_t max_el, cudaStream_t s = 0) : n_(max_el), stream_(s) {
    make_sparse();
    detail::cuda_ok(cudaMemcpyAsync(queue_, &e, 4, cudaMemcpyHostToDevice, s), "subset init");
    uint32_t one = 1;
    detail::cuda_ok(cudaMemcpyAsync(cnt_, &one, 4, cudaMemcpyHostToDevice, s), "subset init");
    detail::cuda_ok(cudaStreamSynchronize(s), "subset init");
  }
  // VertexSubset(0, max_el, true): every vertex.
  VertexSubset(uint32_t, uint32_t max_el, bool all, cudaStream_t s = 0)
      : n_(max_el), stream_(s), all_(all), sparse_(false) {
    if (!all) make_dense();
  }
  static VertexSubset empty_sparse(uint32_t n, cudaStream_t s) {
    VertexSubset v;
    v.n_ = n;
    v.stream_ = s;
    v.make_sparse();
    detail::cuda_ok(cudaMemsetAsync(v.cnt_, 0, 4, s), "subset init");
    return v;
  }
  static VertexSubset empty_dense(uint32_t n, cudaStream_t s) {
    VertexSubset v;
    v.n_ = n;
    v.stream_ = s;
    v.make_dense();
    return v;
  }
  VertexSubset(VertexSubset &&o) noexcept { *this = std::move(o); }
  VertexSubset &operator=(VertexSubset &&o) noexcept {
    if (this != &o) {
      release();
      n_ = o.n_;
      stream_ = o.stream_;
      all_ = o.all_;
      sparse_ = o.sparse_;
      queue_ = o.queue_;
      cnt_ = o.cnt_;
      bits_ = o.bits_;
      o.queue_ = o.cnt_ = o.bits_ = nullptr;
    }
    return *this;
  }
  VertexSubset(const VertexSubset &) = delete;
  VertexSubset &operator=(const VertexSubset &) = delete;
  ~VertexSubset() { release(); }

  bool all() const { return all_; }
  bool is_sparse() const { return sparse_ && !all_; }
  uint32_t max_el() const { return n_; }

  // get_n (include/VertexSubset.cpp:145-156)
  uint64_t get_n() const {
    if (all_) return n_;
    uint32_t c = 0;
    if (sparse_) {
      detail::cuda_ok(cudaMemcpyAsync(&c, cnt_, 4, cudaMemcpyDeviceToHost, stream_), "get_n");
    } else {
      detail::cuda_ok(cudaMemsetAsync(cnt_, 0, 4, stream_), "get_n");
      uint64_t words = (n_ + 31) / 32;
      detail::popcount_bits<<<detail::blocks(words, 256), 256, 0, stream_>>>(bits_, words, cnt_);
      detail::cuda_ok(cudaMemcpyAsync(&c, cnt_, 4, cudaMemcpyDeviceToHost, stream_), "get_n");
    }
    detail::cuda_ok(cudaStreamSynchronize(stream_), "get_n");
    return c;
  }
  bool not_empty() const { return all_ || get_n() > 0; }

  // convert_to_dense / convert_to_sparse (include/VertexSubset.cpp:330-363)
  void convert_to_dense() {
    if (all_ || !sparse_) return;
    uint32_t c = (uint32_t)get_n();
    uint32_t *q = queue_;
    queue_ = nullptr;
    make_dense();
    detail::queue_to_bits<<<detail::blocks(c, 256), 256, 0, stream_>>>(q, c, bits_);
    detail::cuda_ok(cudaStreamSynchronize(stream_), "convert_to_dense");
    cudaFree(q);
  }
  void convert_to_sparse() {
    if (all_ || sparse_) return;
    uint32_t *b = bits_;
    bits_ = nullptr;
    make_sparse();
    detail::cuda_ok(cudaMemsetAsync(cnt_, 0, 4, stream_), "convert_to_sparse");
    detail::bits_to_queue<<<detail::blocks(n_, 256), 256, 0, stream_>>>(b, n_, queue_, cnt_);
    detail::cuda_ok(cudaStreamSynchronize(stream_), "convert_to_sparse");
    cudaFree(b);
  }

  SubsetView view() const {
    return SubsetView{n_, all_ ? 1 : 0, sparse_ && !all_ ? 1 : 0, queue_, bits_};
  }
  uint32_t *queue() const { return queue_; }
  uint32_t *counter() const { return cnt_; }
  uint32_t *bits() const { return bits_; }
  cudaStream_t stream() const { return stream_; }

 private:
  void make_sparse() {
    sparse_ = true;
    if (!cnt_) detail::cuda_ok(cudaMalloc(&cnt_, 4), "subset alloc");
    detail::cuda_ok(cudaMalloc(&queue_, (size_t)(n_ ? n_ : 1) * 4), "subset alloc");
  }
  void make_dense() {
    sparse_ = false;
    if (!cnt_) detail::cuda_ok(cudaMalloc(&cnt_, 4), "subset alloc");
    size_t words = (n_ + 31) / 32;
    detail::cuda_ok(cudaMalloc(&bits_, (words ? words : 1) * 4), "subset alloc");
    detail::cuda_ok(cudaMemsetAsync(bits_, 0, (words ? words : 1) * 4, stream_), "subset alloc");
  }
  void release() {
    if (queue_) cudaFree(queue_);
    if (bits_) cudaFree(bits_);
    if (cnt_) cudaFree(cnt_);
    queue_ = bits_ = cnt_ = nullptr;
  }
  uint32_t n_ = 0;
  cudaStream_t stream_ = 0;
  bool all_ = false, sparse_ = true;
  uint32_t *queue_ = nullptr, *cnt_ = nullptr, *bits_ = nullptr;
};

// edgeMap (include/Map.cpp:65-74).  Returns the output frontier (empty when
// output is false).  Runs on the graph's stream and returns when done.
template <class F>
VertexSubset edgeMap(trc_graph *G, VertexSubset &vs, F f, bool output = true,
                     uint32_t threshold = 20) {
  DeviceGraph dg = device_graph(G);
  cudaStream_t s = static_cast<cudaStream_t>(dg.v.stream);
  const uint32_t n = dg.v.n;
  if ((uint64_t)n / threshold <= vs.get_n()) {
    vs.convert_to_dense();
    VertexSubset out = VertexSubset::empty_dense(n, s);
    detail::em_dense<F><<<detail::blocks(n, 256), 256, 0, s>>>(dg, vs.view(), f, output ? 1 : 0,
                                                                out.bits());
    detail::cuda_ok(cudaGetLastError(), "edgeMap dense");
    detail::cuda_ok(cudaStreamSynchronize(s), "edgeMap dense");
    return out;
  }
  vs.convert_to_sparse();
  uint32_t nq = (uint32_t)vs.get_n();
  VertexSubset out = VertexSubset::empty_sparse(n, s);
  detail::em_sparse<F><<<detail::blocks((uint64_t)nq * 32, 256), 256, 0, s>>>(
      dg, vs.queue(), nq, f, output ? 1 : 0, out.queue(), out.counter());
  detail::cuda_ok(cudaGetLastError(), "edgeMap sparse");
  detail::cuda_ok(cudaStreamSynchronize(s), "edgeMap sparse");
  return out;
}

template <class F>
VertexSubset edgeMap(Graph &G, VertexSubset &vs, F f, bool output = true,
                     uint32_t threshold = 20) {
  return edgeMap(G.handle(), vs, f, output, threshold);
}

// vertexMap (include/Map.cpp:92-108): f(v) for every v in vs; the output
// (same representation, "all" -> dense) holds the v with f(v) == true.
template <class F>
VertexSubset vertexMap(VertexSubset &vs, F f, bool output = true) {
  cudaStream_t s = vs.stream();
  const uint32_t n = vs.max_el();
  SubsetView in = vs.view();
  uint32_t count = in.sparse ? (uint32_t)vs.get_n() : n;
  VertexSubset out = in.sparse ? VertexSubset::empty_sparse(n, s) : VertexSubset::empty_dense(n, s);
  detail::vm_kernel<F><<<detail::blocks(count, 256), 256, 0, s>>>(
      in, count, f, output ? 1 : 0, out.queue(), out.counter(), out.bits());
  detail::cuda_ok(cudaGetLastError(), "vertexMap");
  detail::cuda_ok(cudaStreamSynchronize(s), "vertexMap");
  return out;
}

}  // namespace terrace
