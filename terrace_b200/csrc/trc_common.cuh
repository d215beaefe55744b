// trc_common.cuh -- shared definitions of the sm_100a Terrace hot path:
// the device view of the three degree tiers, error handling, device
// allocation under an HBM budget, and per-kernel CUDA-event profiling.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <map>
#include <string>
#include <utility>
#include <vector>

#include "terrace_b200.h"

namespace trc {

// ---------------------------------------------------------------------------
// Tier constants.
//
// Tier 1: the first K_INLINE neighbours of every vertex live in a 64-byte
// row (one 128-bit load per 4 neighbours).  The reference keeps 13 in-place
// neighbours because its 64-byte block also holds the degree and a pointer
// (include/graph.h:34-38, :216-224); here degree and tier pointers live in
// separate arrays, so the row holds 16.
constexpr uint32_t K_INLINE = 16;
constexpr uint32_t HUB_THRESHOLD_MAX = 12288;  // largest configurable hub threshold
// Tier 3: hub neighbours are kept in blocks of HUB_BLOCK slots, found through
// a per-hub directory (see DevView).
constexpr uint32_t HUB_BLOCK = 256;
constexpr uint32_t NONE32 = 0xFFFFFFFFu;

// Device error word bits.
constexpr uint32_t ERR_BAD_VERTEX = 1u;
constexpr uint32_t ERR_BOUNDS = 2u;
constexpr uint32_t ERR_TIMEOUT = 4u;
constexpr uint32_t ERR_BIGSEG = 8u;  // the bucket sort met a source with too many keys

// ---------------------------------------------------------------------------
// Device view of the graph, passed to kernels by value.
//
//   deg[n]        total degree of every vertex
//   inl[n*16]     tier 1: sorted neighbours 0..min(deg,16)-1
//   pbeg[n+1]     tier 2 (packed-memory array over vertex segments): vertex
//                 u's neighbours 16..deg-1 sit in pma[pbeg[u] .. pbeg[u]+c2[u])
//                 with slack up to pbeg[u+1]; pbeg[n] = capacity
//   c2[n]         tier-2 element count (0 for hubs and low-degree vertices)
//   hub_of[n]     hub index or -1
//   tier 3, a two-level B-tree per hub (the reference's per-vertex BTree,
//   include/btree.h:27-826, with one directory level over sorted leaves):
//     hub_vtx[h], hub_nblk[h]   vertex; blocks in use
//     hub_dir0[h]               the hub's directory in hdir/hpre/hkey: entry
//                               i < hub_nblk[h] at hub_dir0[h] + i describes
//                               the i-th block in key order --
//     hdir[e]                   its pool block id,
//     hpre[e]                   the number of hub elements before it (the
//                               hub part starts at list rank 16), and
//     hkey[e]                   its first (smallest) element
//     hslot[b*256 ..], bcnt[b], bmin[b], bown[b]
//                               block pool: slots (the first bcnt[b] used,
//                               sorted), count, first key, owner vertex
//   Rank r >= 16 of a hub is in the block whose hpre is the largest <= r-16;
//   blocks are filled between 1 and 256 elements, so inserting or removing
//   an edge rewrites one block (and the directory), not the whole list.
struct DevView {
  uint32_t n;
  uint32_t hub_T;
  uint32_t *deg;
  uint32_t *inl;
  uint64_t *pbeg;
  uint32_t *c2;
  uint32_t *pma;
  uint64_t N;
  int32_t *hub_of;
  uint32_t *hub_vtx;
  uint64_t *hub_dir0;
  uint32_t *hub_nblk;
  uint32_t *hdir;
  uint32_t *hpre;
  uint32_t *hkey;
  uint32_t *hslot;
  uint32_t *bcnt;
  uint32_t *bmin;
  uint32_t *bown;
  uint32_t *err;  // device error word
};

// Directory entry of hub-part rank r (0 <= r < rest): the largest i < nb
// with pre[i] <= r.  Blocks are mostly filled alike, so a proportional guess
// usually hits; otherwise a binary search on the side it missed.
__device__ __forceinline__ uint32_t hub_entry_of_rank(const uint32_t *pre, uint32_t nb,
                                                      uint32_t rest, uint32_t r) {
  uint32_t i = (uint32_t)(((uint64_t)r * nb) / (rest ? rest : 1));
  if (i >= nb) i = nb - 1;
  uint32_t lo, hi;
  if (pre[i] > r) {
    lo = 0;
    hi = i;
  } else if (i + 1 < nb && pre[i + 1] <= r) {
    lo = i + 1;
    hi = nb;
  } else {
    return i;
  }
  while (hi - lo > 1) {  // invariant: pre[lo] <= r, answer in [lo, hi)
    uint32_t mid = (lo + hi) >> 1;
    if (pre[mid] <= r) lo = mid;
    else hi = mid;
  }
  return lo;
}

// Directory entry whose block holds key x if present: the largest i < nb
// with key[i] <= x, or 0.
__device__ __forceinline__ uint32_t hub_entry_of_key(const uint32_t *key, uint32_t nb, uint32_t x) {
  uint32_t lo = 0, hi = nb;  // count of entries with key <= x
  while (lo < hi) {
    uint32_t mid = (lo + hi) >> 1;
    if (key[mid] <= x) lo = mid + 1;
    else hi = mid;
  }
  return lo ? lo - 1 : 0;
}

// Read-only accessor for one vertex's sorted neighbour list by rank.
struct NbrList {
  const uint32_t *inl;   // row
  const uint32_t *seg;   // tier-2 segment (non-hub) or the block pool's slots (hub)
  const uint32_t *dir;   // hub: block ids in key order
  const uint32_t *pre;   // hub: elements before each block
  const uint32_t *key;   // hub: first element of each block
  uint32_t ni;           // inline count
  uint32_t rest;         // elements after the inline ones
  uint32_t nb;           // hub: blocks; 0 = tier-2 segment (or no hub part)
  uint32_t deg;

  __device__ __forceinline__ uint32_t at(uint32_t r) const {
    if (r < ni) return inl[r];
    r -= ni;
    if (nb == 0) return seg[r];
    const uint32_t i = hub_entry_of_rank(pre, nb, rest, r);
    return seg[(uint64_t)dir[i] * HUB_BLOCK + (r - pre[i])];
  }
};

__device__ __forceinline__ NbrList nbr_list(const DevView &G, uint32_t u) {
  NbrList L;
  uint32_t d = G.deg[u];
  L.deg = d;
  L.inl = G.inl + (uint64_t)u * K_INLINE;
  L.ni = d < K_INLINE ? d : K_INLINE;
  L.rest = d - L.ni;
  int32_t h = G.hub_of[u];
  if (h < 0) {
    L.seg = G.pma + G.pbeg[u];
    L.nb = 0;
    L.dir = L.pre = L.key = nullptr;
  } else {
    const uint64_t e0 = G.hub_dir0[h];
    L.seg = G.hslot;
    L.nb = L.rest ? G.hub_nblk[h] : 0;
    L.dir = G.hdir + e0;
    L.pre = G.hpre + e0;
    L.key = G.hkey + e0;
  }
  return L;
}

// A hub's list in chunks for traversals that need no order: chunk c is the
// 32-element piece c % 8 of unit c / 8, unit 0 being the inline row and unit
// 1 + e the block of directory entry e (a block holds at most 256).  Sets the
// piece's pointer and length (0: an empty piece).  Reads each element from
// its slot, without a directory search per element.
__device__ __forceinline__ uint32_t hub_chunks(const NbrList &L) { return (1 + L.nb) * 8; }

__device__ __forceinline__ void hub_chunk(const NbrList &L, uint32_t c, const uint32_t *&p,
                                          uint32_t &len) {
  const uint32_t unit = c >> 3, off = (c & 7) * 32;
  uint32_t ulen;
  const uint32_t *up;
  if (unit == 0) {
    up = L.inl;
    ulen = L.ni;
  } else {
    const uint32_t e = unit - 1;
    up = L.seg + (uint64_t)L.dir[e] * HUB_BLOCK;
    ulen = (e + 1 < L.nb ? L.pre[e + 1] : L.rest) - L.pre[e];
  }
  p = up + off;
  len = off < ulen ? (ulen - off < 32 ? ulen - off : 32) : 0;
}

// Any list as pieces of at most 32 elements, for traversals that need no
// order: a hub's pieces are its hub_chunk()s; a tier-1/2 vertex has piece 0
// = the inline row, then 32-element pieces of its segment.  Every list has
// at least one piece (possibly empty).
__device__ __forceinline__ uint32_t list_pieces(const NbrList &L) {
  return L.nb ? hub_chunks(L) : 1 + (L.rest + 31) / 32;
}

__device__ __forceinline__ void list_piece(const NbrList &L, uint32_t c, const uint32_t *&p,
                                           uint32_t &len) {
  if (L.nb) {
    hub_chunk(L, c, p, len);
  } else if (c == 0) {
    p = L.inl;
    len = L.ni;
  } else {
    const uint32_t off = (c - 1) * 32;
    p = L.seg + off;
    len = L.rest - off < 32 ? L.rest - off : 32;
  }
}

// Binary search for x in the neighbour list (lists are sorted, unique); a
// hub's blocked part is searched through its directory's first keys.
__device__ __forceinline__ bool list_has(const NbrList &L, uint32_t x) {
  uint32_t lo = 0, hi = L.deg;
  if (L.nb) {
    if (L.ni == 0 || x > L.inl[L.ni - 1]) {
      const uint32_t i = hub_entry_of_key(L.key, L.nb, x);
      const uint32_t *b = L.seg + (uint64_t)L.dir[i] * HUB_BLOCK;
      uint32_t blo = 0, bhi = (i + 1 < L.nb ? L.pre[i + 1] : L.rest) - L.pre[i];
      while (blo < bhi) {
        uint32_t mid = (blo + bhi) >> 1;
        uint32_t v = b[mid];
        if (v < x) blo = mid + 1;
        else if (v > x) bhi = mid;
        else return true;
      }
      return false;
    }
    hi = L.ni;  // x is at most the last inline element
  }
  while (lo < hi) {
    uint32_t mid = (lo + hi) >> 1;
    uint32_t v = L.at(mid);
    if (v < x) lo = mid + 1;
    else if (v > x) hi = mid;
    else return true;
  }
  return false;
}

// Number of list elements < x.
__device__ __forceinline__ uint32_t list_lower_bound(const NbrList &L, uint32_t x) {
  uint32_t lo = 0, hi = L.deg;
  if (L.nb) {
    if (L.ni == 0 || x > L.inl[L.ni - 1]) {
      const uint32_t i = hub_entry_of_key(L.key, L.nb, x);
      const uint32_t *b = L.seg + (uint64_t)L.dir[i] * HUB_BLOCK;
      uint32_t blo = 0, bhi = (i + 1 < L.nb ? L.pre[i + 1] : L.rest) - L.pre[i];
      while (blo < bhi) {
        uint32_t mid = (blo + bhi) >> 1;
        if (b[mid] < x) blo = mid + 1;
        else bhi = mid;
      }
      return L.ni + L.pre[i] + blo;
    }
    hi = L.ni;
  }
  while (lo < hi) {
    uint32_t mid = (lo + hi) >> 1;
    if (L.at(mid) < x) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// ---------------------------------------------------------------------------
// Host-side error handling: internal code throws Error; the C ABI layer
// converts it into a trc_status plus a thread-local message.
struct Error {
  trc_status status;
  std::string msg;
};

[[noreturn]] void throw_error(trc_status s, const std::string &msg);
void cuda_check(cudaError_t e, const char *what, const char *file, int line);
#define TRC_CUDA(call) ::trc::cuda_check((call), #call, __FILE__, __LINE__)

// ---------------------------------------------------------------------------
// Device memory under a per-graph HBM budget.  Allocations are
// stream-ordered (cudaMallocFromPoolAsync / cudaFreeAsync on the graph's
// stream) from a pool owned by the graph that keeps freed memory for reuse,
// so per-call scratch of the analytics costs no device synchronisation.
class Budget {
 public:
  uint64_t limit = 0;  // 0 = device free memory is the only limit
  uint64_t used = 0;
  cudaStream_t stream = nullptr;  // allocation / free order
  cudaMemPool_t pool = nullptr;
  void open_pool(int device);
  void trim();  // returns cached free memory to the device
  ~Budget();
  void *alloc(uint64_t bytes);
  void release(void *p, uint64_t bytes);
};

template <typename T>
class DBuf {
 public:
  DBuf() = default;
  DBuf(const DBuf &) = delete;
  DBuf &operator=(const DBuf &) = delete;
  ~DBuf() { reset(); }
  void bind(Budget *b) { budget_ = b; }
  // Ensures capacity for `count` elements; contents are NOT preserved.
  T *ensure(uint64_t count) {
    if (count > cap_) {
      reset();
      uint64_t c = count < 16 ? 16 : count;
      ptr_ = static_cast<T *>(bud().alloc(c * sizeof(T)));
      cap_ = c;
    }
    return ptr_;
  }
  // Exactly `count` elements, contents NOT preserved.
  T *alloc_exact(uint64_t count) {
    reset();
    uint64_t c = count < 1 ? 1 : count;
    ptr_ = static_cast<T *>(bud().alloc(c * sizeof(T)));
    cap_ = c;
    return ptr_;
  }
  // Grows to at least `count`, preserving the first `keep` elements (at
  // most the old capacity).
  T *grow(uint64_t count, uint64_t keep, cudaStream_t s) {
    if (count <= cap_) return ptr_;
    if (keep > cap_) keep = cap_;
    uint64_t c = count < 16 ? 16 : count;
    T *np = static_cast<T *>(bud().alloc(c * sizeof(T)));
    if (keep) TRC_CUDA(cudaMemcpyAsync(np, ptr_, keep * sizeof(T), cudaMemcpyDeviceToDevice, s));
    TRC_CUDA(cudaStreamSynchronize(s));
    reset();
    ptr_ = np;
    cap_ = c;
    return ptr_;
  }
  void swap(DBuf &o) {
    std::swap(ptr_, o.ptr_);
    std::swap(cap_, o.cap_);
    std::swap(budget_, o.budget_);
  }
  void reset() {
    if (ptr_) budget_->release(ptr_, cap_ * sizeof(T));
    ptr_ = nullptr;
    cap_ = 0;
  }
  T *get() const { return ptr_; }
  uint64_t capacity() const { return cap_; }
  uint64_t bytes() const { return cap_ * sizeof(T); }

 private:
  T *ptr_ = nullptr;
  uint64_t cap_ = 0;
  Budget *budget_ = nullptr;
  Budget &bud() {
    if (!budget_) throw_error(TRC_ERR_STATE, "device buffer used before it was bound to a budget");
    return *budget_;
  }
};

// ---------------------------------------------------------------------------
// Per-kernel profiling with CUDA events on the launching stream.
class Profiler {
 public:
  bool on = false;
  uint64_t launches = 0;  // every kernel launch, profiled or not
  struct Rec {
    cudaEvent_t a, b;
    std::string name;
  };
  std::vector<Rec> pending;
  std::map<std::string, std::pair<double, uint64_t>> totals;

  int begin(const char *name, cudaStream_t s);
  void end(int idx, cudaStream_t s);
  void resolve();
  void reset();
  ~Profiler();

 private:
  std::vector<cudaEvent_t> pool_;
  cudaEvent_t get_event();
};

// Launch wrapper: skips empty grids, records events when profiling, checks
// the launch error.
#define TRC_LAUNCH(prof, stream, name, grid, block, smem, kern, ...)          \
  do {                                                                       \
    uint64_t _g = (uint64_t)(grid);                                          \
    if (_g > 0) {                                                            \
      int _pi = (prof).begin(name, stream);                                  \
      kern<<<(unsigned)_g, (block), (smem), (stream)>>>(__VA_ARGS__);        \
      (prof).end(_pi, stream);                                               \
      TRC_CUDA(cudaGetLastError());                                          \
    }                                                                        \
  } while (0)

inline uint64_t ceil_div(uint64_t a, uint64_t b) { return (a + b - 1) / b; }

// Number of SMs on the current device (cached).
int num_sms();
// CTAs of `threads` threads (and `smem` dynamic shared bytes) of `kernel`
// that fit on the whole GPU at once: the grid of a grid-stride kernel.
template <typename K>
unsigned resident_grid(K kernel, int threads, size_t smem = 0) {
  int per = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, threads, smem) != cudaSuccess ||
      per < 1)
    per = 1;
  return (unsigned)(per * num_sms());
}

}  // namespace trc
