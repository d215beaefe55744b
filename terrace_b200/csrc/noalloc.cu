// noalloc.cu -- trc_bfs_noalloc: BFS that allocates no device memory.
//
// Some callers cannot call cudaMalloc when they need a traversal: a service
// that sizes its device memory once at start-up and must not grow it while
// answering requests, an embedding that has handed the allocator to another
// component, or code that must not risk an allocation failure (or the
// implicit synchronisation cudaMalloc/cudaFree bring) on its request path.
// trc_bfs does allocate (level and frontier buffers, per-class vertex lists),
// so this variant keeps its only scratch -- two frontier queues and a counter
// -- in the file-scope array below.  It uses push steps only, which need no
// per-class lists.
//
// The caller passes the outputs (parents and levels, device arrays of n
// entries).  The array's name in host code is a host-side stand-in, not a
// device address.  Its device address is looked up with cudaGetSymbolAddress
// when a graph is created, with the graph's device current, and kept in the
// graph: that lookup is also what loads this file's module (CUDA loads
// modules lazily), so the array's NOALLOC_BYTES are reserved on the device
// when the first graph is created there, not by the no-allocation call, and
// stay reserved until the process exits.  A graph's copy of the address
// lives no longer than the graph, which a device reset invalidates anyway.
// All calls share the array, so calls that overlap on the GPU (two host
// threads, two streams, two graphs) race on it.
#include "graph.cuh"

namespace trc {

constexpr uint64_t NOALLOC_QUEUE = TRC_NOALLOC_MAX_VERTICES;
// two queues of NOALLOC_QUEUE entries, then a 256-byte slot for the counter
constexpr uint64_t NOALLOC_WORDS = 2 * NOALLOC_QUEUE + 64;
constexpr uint64_t NOALLOC_BYTES = NOALLOC_WORDS * 4;  // 8 MiB + 256 B

static __device__ __align__(256) uint32_t g_noalloc_scratch[NOALLOC_WORDS];

// Device address of g_noalloc_scratch on the current device.
uint32_t *noalloc_scratch_resolve() {
  void *p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || !p) {
    cudaGetLastError();
    throw_error(TRC_ERR_CUDA, std::string("cudaGetSymbolAddress(noalloc scratch) failed: ") +
                                  cudaGetErrorString(e));
  }
  return static_cast<uint32_t *>(p);
}

namespace {
__device__ __forceinline__ uint32_t na_lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

__global__ void k_na_init(uint32_t *lv, int32_t *par, uint32_t n, uint32_t src, uint32_t *queue) {
  uint64_t u = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= n) return;
  lv[u] = u == src ? 0 : TRC_UNREACHED;
  par[u] = u == src ? (int32_t)src : -1;
  if (u == src) queue[0] = src;
}

// One warp per frontier vertex: claim unvisited neighbours with CAS on the
// parent array (BFS_F::updateAtomic, include/BFS.h:34-36) and append them to
// the next queue with one atomic per warp.
__global__ void k_na_push(DevView G, const uint32_t *F, uint32_t nf, uint32_t *lv, int32_t *par,
                          uint32_t *next, uint32_t *next_cnt, uint32_t d) {
  uint64_t w = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  uint32_t lane = threadIdx.x & 31;
  if (w >= nf) return;
  uint32_t u = F[w];
  NbrList L = nbr_list(G, u);
  for (uint32_t j0 = 0; j0 < L.deg; j0 += 32) {
    uint32_t j = j0 + lane;
    bool win = false;
    uint32_t v = 0;
    if (j < L.deg) {
      v = L.at(j);
      if (lv[v] == TRC_UNREACHED && atomicCAS(&par[v], -1, (int32_t)u) == -1) {
        lv[v] = d + 1;
        win = true;
      }
    }
    uint32_t m = __ballot_sync(0xFFFFFFFFu, win);
    uint32_t base = 0;
    if (m) {
      uint32_t leader = __ffs(m) - 1;
      if (lane == leader) base = atomicAdd(next_cnt, __popc(m));
      base = __shfl_sync(0xFFFFFFFFu, base, leader);
    }
    if (win) next[base + __popc(m & na_lanemask_lt())] = v;
  }
}
}  // namespace

void Graph::bfs_noalloc(uint32_t src, int32_t *parents, uint32_t *levels, uint32_t flags) {
  if (!(flags & TRC_DEVICE_PTR))
    throw_error(TRC_ERR_INVALID, "trc_bfs_noalloc needs device output arrays (TRC_DEVICE_PTR)");
  if (!parents || !levels) throw_error(TRC_ERR_INVALID, "null output");
  if (n > TRC_NOALLOC_MAX_VERTICES)
    throw_error(TRC_ERR_INVALID, "trc_bfs_noalloc supports at most TRC_NOALLOC_MAX_VERTICES "
                                 "(1048576) vertices");
  if (src >= n) throw_error(TRC_ERR_INVALID, "source vertex out of range");
  int prev = 0;
  TRC_CUDA(cudaGetDevice(&prev));
  if (prev != device) TRC_CUDA(cudaSetDevice(device));
  try {
    uint32_t *S = na_scratch;  // looked up when the graph was created
    uint32_t *F = S, *Nx = S + NOALLOC_QUEUE, *cnt = S + 2 * NOALLOC_QUEUE;
    TRC_LAUNCH(prof, stream, "na_init", ceil_div(n, 256), 256, 0, k_na_init, levels, parents, n, src,
               F);
    DevView G = view();
    uint32_t nf = 1, d = 0;
    while (nf > 0) {
      TRC_CUDA(cudaMemsetAsync(cnt, 0, 4, stream));  // the shared counter starts at zero
      TRC_LAUNCH(prof, stream, "na_push", ceil_div((uint64_t)nf * 32, 256), 256, 0, k_na_push, G,
                 F, nf, levels, parents, Nx, cnt, d);
      TRC_CUDA(cudaMemcpyAsync(&nf, cnt, 4, cudaMemcpyDeviceToHost, stream));
      sync();
      uint32_t *t = F;
      F = Nx;
      Nx = t;
      d++;
    }
  } catch (...) {
    if (prev != device) cudaSetDevice(prev);
    throw;
  }
  if (prev != device) TRC_CUDA(cudaSetDevice(prev));
}

}  // namespace trc
