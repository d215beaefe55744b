// hubs.cu -- tier 3: batch updates of the hubs' blocked lists.
//
// Replaces the reference's per-vertex B-tree updates (BTree::insert with
// preemptive split, include/btree.h:283-381, :437-486; delete with borrow
// and merge, :498-826; Graph::add_btree, include/graph.h:375-426).  A hub's
// neighbours past the 16 inline ones live in pool blocks of up to 256 sorted
// slots; a per-hub directory lists the blocks in key order with each block's
// first key and element prefix (the B-tree's root level over its leaves).
//
// A batch touching a hub takes one of two paths:
//
//   block-local (existing hubs): every batch key is located in the directory
//   (largest first key <= key); keys of one block form a group.  Group 0 is
//   the inline row plus the first block, so displacement out of (and refill
//   of) the inline row stays inside one group.  One CTA per touched group
//   merges the block (and, for group 0, the inline row) with its keys in
//   shared memory and writes it back in place; a block that grows past 256
//   elements splits into evenly filled blocks (new ids from the free list or
//   the pool), an emptied block is freed, and a block left with fewer than
//   HB_MIN elements after deletes absorbs its successor when that block is
//   untouched and both fit (the reference's merge on underflow).  Then one
//   CTA per hub rebuilds its directory: untouched entries are copied, touched
//   ones replaced by their output blocks.  Bytes moved scale with the blocks
//   touched, not with the hub's degree.
//
//   rewrite (new hubs, hubs of fewer than HB_LOCAL_MIN neighbours, hubs
//   without blocks, growth past the old size, a group with more keys than
//   one merge stages, an inline row that cannot be refilled from the first
//   two blocks): every old element and every key is placed at its new rank
//   directly in uniformly filled blocks taken from the free list (then the
//   pool); the old blocks are freed.
//
// Which groups of a block-local hub need the rewrite is known only after the
// groups are counted, so the host reads those counts once; the small-vertex
// merge of tiers 1-2 runs on the graph's stream meanwhile.
#include <algorithm>
#include <cstring>

#include "graph.cuh"

namespace trc {

constexpr uint32_t HB_MIN = 64;    // fewer elements after a delete: absorb the successor
constexpr uint32_t HB_OUT = 32;    // most blocks one touched block becomes
constexpr uint32_t HB_GK = 4096;   // most keys one block merge stages in shared memory
constexpr uint32_t HB_STAGE = K_INLINE + 2 * HUB_BLOCK;  // old elements of a group, at most
// Hubs of fewer neighbours than this are rewritten whole: their list is a
// few KB, less than locating the keys and rebuilding the directory costs.
constexpr uint32_t HB_LOCAL_MIN = 8192;

// Counter slots in the batch's device counter array (update.cu uses 0..10,
// the analytics 24..29).
enum { H_NTG = 12, H_ALLOC = 13, H_FREED = 14, H_READ = 15, H_WRITE = 16, H_ABSORB = 17,
       H_ALLOC_REQ = 18 };

// Rows of the block-local plan (per hub li) and the rewrite plan (per hub r).
enum { LP_H = 0, LP_U, LP_IHW, LP_Q0, LP_DN, LP_W };
enum { RP_H = 0, RP_U, RP_IHW, RP_DO, RP_DN, RP_BLK0, RP_PER, RP_NB, RP_Q0, RP_E1, RP_W };

__device__ __forceinline__ uint32_t lb_u64lo(const uint64_t *K, uint32_t k, uint32_t x) {
  uint32_t lo = 0, hi = k;
  while (lo < hi) {
    uint32_t mid = (lo + hi) >> 1;
    if ((uint32_t)K[mid] < x) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ uint32_t lb_u32(const uint32_t *A, uint32_t n, uint32_t x) {
  uint32_t lo = 0, hi = n;
  while (lo < hi) {
    uint32_t mid = (lo + hi) >> 1;
    if (A[mid] < x) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// largest i < n with a[i * stride + off] <= x (a's column ascending, a[off] <= x)
__device__ __forceinline__ uint64_t row_of(const uint64_t *a, uint64_t n, uint32_t stride,
                                           uint32_t off, uint64_t x) {
  uint64_t lo = 0, hi = n;
  while (hi - lo > 1) {
    uint64_t mid = (lo + hi) >> 1;
    if (a[mid * stride + off] <= x) lo = mid;
    else hi = mid;
  }
  return lo;
}

// The batch slice of touched hub i_hw: keys [tpos[t], tpos[t] + k).
__device__ __forceinline__ const uint64_t *hub_keys(const uint32_t *hw_t, const uint64_t *tpos,
                                                    const uint64_t *bkeys, uint64_t i_hw) {
  return bkeys + tpos[hw_t[i_hw]];
}

// ---------------------------------------------------------------- block-local

// One thread per key of a block-local hub: its group (directory entry).
__global__ void k_hub_locate(DevView G, const uint64_t *lp, uint64_t NL, uint64_t QL,
                             const uint32_t *hw_t, const uint64_t *tpos, const uint64_t *bkeys,
                             uint32_t *lli, uint32_t *lg, uint32_t *lx) {
  const uint64_t q = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= QL) return;
  const uint64_t li = row_of(lp, NL, LP_W, LP_Q0, q);
  const uint64_t *row = lp + li * LP_W;
  const uint32_t x = (uint32_t)hub_keys(hw_t, tpos, bkeys, row[LP_IHW])[q - row[LP_Q0]];
  const uint32_t h = (uint32_t)row[LP_H];
  const uint64_t e0 = G.hub_dir0[h];
  lli[q] = (uint32_t)li;
  lg[q] = hub_entry_of_key(G.hkey + e0, G.hub_nblk[h], x);
  lx[q] = x;
}

struct GroupStartPred {
  const uint32_t *lli, *lg;
  __device__ bool operator()(uint64_t q) const {
    return q == 0 || lli[q] != lli[q - 1] || lg[q] != lg[q - 1];
  }
};

struct IndexVal32H {
  __device__ uint32_t operator()(uint64_t i) const { return (uint32_t)i; }
};

// tgo word of a touched group: blocks out (6 bits), absorbs its successor
// (1 bit), hub-part elements after the merge (from bit 8).
__device__ __forceinline__ uint32_t tgo_pack(uint32_t nout, uint32_t absorb, uint32_t hp) {
  return nout | (absorb << 6) | (hp << 8);
}

// Thread per touched group: counts after the merge (every insert key is
// absent and every delete key present, so they follow from the key count),
// the blocks out, absorption of an underfull block's successor, and the
// flag that sends the hub to the rewrite path.
__global__ void k_hub_count(DevView G, const uint64_t *lp, const uint64_t *cnt, uint64_t QL,
                            const uint32_t *tgq, const uint32_t *lli, const uint32_t *lg, int insert,
                            uint32_t gk, uint32_t fill, uint32_t *tgo, uint32_t *hflag, int32_t *hnbd,
                            unsigned long long *alloc_req) {
  const uint64_t ntg = cnt[H_NTG];
  const uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= ntg) return;
  const uint64_t q0 = tgq[j], q1 = j + 1 < ntg ? tgq[j + 1] : QL;
  const uint32_t li = lli[q0], g = lg[q0];
  const uint32_t k = (uint32_t)(q1 - q0);
  const uint32_t h = (uint32_t)lp[(uint64_t)li * LP_W + LP_H];
  const uint64_t e0 = G.hub_dir0[h];
  const uint32_t nb = G.hub_nblk[h];
  const uint32_t c = G.bcnt[G.hdir[e0 + g]];
  const bool next_touched = j + 1 < ntg && lli[tgq[j + 1]] == li && lg[tgq[j + 1]] == g + 1;
  bool flag = k > gk;
  uint32_t absorb = 0;
  int64_t hp;  // hub-part elements of the group's output
  if (g == 0) {
    const int64_t tot = (int64_t)K_INLINE + c + (insert ? (int64_t)k : -(int64_t)k);
    hp = tot - K_INLINE;
    if (tot < (int64_t)K_INLINE && nb > 1) {  // the inline row needs the next block
      const uint32_t c1 = G.bcnt[G.hdir[e0 + 1]];
      if (next_touched || (tot + c1 < (int64_t)K_INLINE && nb > 2)) {
        flag = true;
      } else {
        absorb = 1;
        hp = tot + c1 - K_INLINE;
      }
    }
    if (hp < 0) hp = 0;
  } else {
    hp = (int64_t)c + (insert ? (int64_t)k : -(int64_t)k);
  }
  if (!flag && !insert && g + 1 < nb && hp > 0 && hp < HB_MIN && !next_touched && !absorb) {
    const uint32_t c1 = G.bcnt[G.hdir[e0 + g + 1]];
    if (hp + c1 <= HUB_BLOCK) {
      absorb = 1;
      hp += c1;
    }
  }
  uint32_t nout = 0;
  if (hp > 0) nout = hp <= HUB_BLOCK ? 1u : (uint32_t)((hp + fill - 1) / fill);
  if (nout > HB_OUT) flag = true;
  if (flag) {
    atomicOr(hflag + li, 1u);
    tgo[j] = 0;
    return;
  }
  tgo[j] = tgo_pack(nout, absorb, (uint32_t)hp);
  atomicAdd(hnbd + li, (int32_t)nout - 1 - (int32_t)absorb);
  if (nout > 1) atomicAdd(alloc_req, (unsigned long long)(nout - 1));
}

// Pool id of the a-th block allocated in this batch: the free list first
// (from its top), then fresh blocks.  Indices [0, R) belong to the rewritten
// hubs (ranges planned on the host), R on to the splits (a device counter).
__device__ __forceinline__ uint32_t alloc_id(uint64_t a, const uint32_t *bfree, uint64_t F,
                                            uint64_t fresh0) {
  return a < F ? bfree[F - 1 - a] : (uint32_t)(fresh0 + (a - F));
}

// CTA per touched group of a block-local hub: stage, merge, write in place,
// split, free, absorb.
__global__ void __launch_bounds__(256) k_hub_merge_group(
    DevView G, const uint64_t *lp, const uint64_t *cnt, uint64_t QL, const uint32_t *tgq,
    const uint32_t *lli, const uint32_t *lg, const uint32_t *lx, const uint32_t *tgo,
    const uint32_t *hflag, int insert, const uint32_t *bfree, uint64_t F, uint64_t fresh0,
    uint64_t R, uint32_t *bfreed, uint32_t *tgb, unsigned long long *ctr) {
  __shared__ uint32_t A[HB_STAGE];
  __shared__ uint32_t O[HB_STAGE + HB_GK];
  __shared__ uint32_t ids[HB_OUT];
  const uint64_t ntg = ctr[H_NTG];
  const uint64_t j = blockIdx.x;
  if (j >= ntg) return;
  const uint64_t q0 = tgq[j], q1 = j + 1 < ntg ? tgq[j + 1] : QL;
  const uint32_t li = lli[q0];
  if (hflag[li]) return;
  const uint32_t g = lg[q0];
  const uint32_t k = (uint32_t)(q1 - q0);
  const uint32_t *K = lx + q0;
  const uint64_t *row = lp + (uint64_t)li * LP_W;
  const uint32_t h = (uint32_t)row[LP_H], u = (uint32_t)row[LP_U];
  const uint64_t e0 = G.hub_dir0[h];
  const uint32_t b = G.hdir[e0 + g];
  const uint32_t c = G.bcnt[b];
  const uint32_t o = tgo[j];
  const uint32_t nout = o & 63u, absorb = (o >> 6) & 1u, hp = o >> 8;
  const uint32_t base = g == 0 ? K_INLINE : 0u;
  const uint32_t b2 = absorb ? G.hdir[e0 + g + 1] : NONE32;
  const uint32_t c2 = absorb ? G.bcnt[b2] : 0u;
  uint32_t *row_inl = G.inl + (uint64_t)u * K_INLINE;
  // stage the old elements: [inline row] block [successor]
  const uint32_t na = base + c + c2;
  for (uint32_t i = threadIdx.x; i < na; i += blockDim.x) {
    uint32_t v;
    if (i < base) v = row_inl[i];
    else if (i < base + c) v = G.hslot[(uint64_t)b * HUB_BLOCK + (i - base)];
    else v = G.hslot[(uint64_t)b2 * HUB_BLOCK + (i - base - c)];
    A[i] = v;
  }
  __syncthreads();
  uint32_t total;
  if (insert) {
    for (uint32_t i = threadIdx.x; i < na; i += blockDim.x) O[i + lb_u32(K, k, A[i])] = A[i];
    for (uint32_t i = threadIdx.x; i < k; i += blockDim.x) O[i + lb_u32(A, na, K[i])] = K[i];
    total = na + k;
  } else {
    for (uint32_t i = threadIdx.x; i < na; i += blockDim.x) {
      const uint32_t x = A[i];
      const uint32_t cc = lb_u32(K, k, x);
      if (!(cc < k && K[cc] == x)) O[i - cc] = x;
    }
    total = na - k;
  }
  if (threadIdx.x == 0) {
    const unsigned long long a0 = nout > 1 ? atomicAdd(ctr + H_ALLOC, (unsigned long long)(nout - 1)) : 0ull;
    if (nout > 0) ids[0] = b;
    for (uint32_t t = 1; t < nout; t++) ids[t] = alloc_id(R + a0 + t - 1, bfree, F, fresh0);
    if (nout == 0) bfreed[atomicAdd(ctr + H_FREED, 1ull)] = b;
    if (absorb) {
      bfreed[atomicAdd(ctr + H_FREED, 1ull)] = b2;
      atomicAdd(ctr + H_ABSORB, 1ull);
    }
    atomicAdd(ctr + H_READ, (unsigned long long)na);
    atomicAdd(ctr + H_WRITE, (unsigned long long)total);
  }
  __syncthreads();
  // the inline row (group 0): the first min(total, 16) elements
  if (g == 0) {
    const uint32_t ni = total < K_INLINE ? total : K_INLINE;
    for (uint32_t i = threadIdx.x; i < ni; i += blockDim.x) row_inl[i] = O[i];
  }
  // the hub part, hp = total - base elements (0 when the list ends inline),
  // split evenly over the output blocks
  for (uint32_t t = 0; t < nout; t++) {
    const uint32_t s0 = (uint32_t)((uint64_t)t * hp / nout), s1 = (uint32_t)((uint64_t)(t + 1) * hp / nout);
    const uint32_t id = ids[t];
    uint32_t *dst = G.hslot + (uint64_t)id * HUB_BLOCK;
    for (uint32_t i = s0 + threadIdx.x; i < s1; i += blockDim.x) dst[i - s0] = O[base + i];
    if (threadIdx.x == 0) {
      G.bcnt[id] = s1 - s0;
      G.bmin[id] = O[base + s0];
      G.bown[id] = u;
      tgb[j * HB_OUT + t] = id;
    }
  }
}

// CTA per block-local hub: the new directory (untouched entries copied,
// touched ones replaced by their output blocks, absorbed ones dropped) in the
// hub's other directory half, then its prefixes and first keys; the hub's
// table entry and degree last.
__global__ void __launch_bounds__(256) k_hub_dir(DevView G, const uint64_t *lp, uint64_t NL,
                                                 const uint64_t *cnt, uint64_t QL,
                                                 const uint32_t *tgq, const uint32_t *lg,
                                                 const uint32_t *tgo, const uint32_t *tgb,
                                                 const uint32_t *hflag, const uint64_t *e1s) {
  __shared__ uint32_t ws[256 / 32 + 1];
  __shared__ uint32_t carry;
  const uint32_t li = blockIdx.x;
  if (hflag[li]) return;
  const uint64_t ntg = cnt[H_NTG];
  const uint64_t *row = lp + (uint64_t)li * LP_W;
  const uint32_t h = (uint32_t)row[LP_H], u = (uint32_t)row[LP_U], dn = (uint32_t)row[LP_DN];
  const uint64_t e0 = G.hub_dir0[h], e1 = e1s[li];
  const uint32_t nb = G.hub_nblk[h];
  // this hub's touched groups: tgq entries in [q0(li), q0(li+1))
  const uint64_t qa = row[LP_Q0], qb = li + 1 < NL ? lp[(uint64_t)(li + 1) * LP_W + LP_Q0] : QL;
  uint64_t j0, j1;
  {
    uint64_t lo = 0, hi = ntg;
    while (lo < hi) { uint64_t m = (lo + hi) >> 1; if (tgq[m] < qa) lo = m + 1; else hi = m; }
    j0 = lo;
    hi = ntg;
    while (lo < hi) { uint64_t m = (lo + hi) >> 1; if (tgq[m] < qb) lo = m + 1; else hi = m; }
    j1 = lo;
  }
  auto touched = [&](uint32_t i) -> int64_t {  // touched-group index of entry i, or -1
    uint64_t lo = j0, hi = j1;
    while (lo < hi) { uint64_t m = (lo + hi) >> 1; if (lg[tgq[m]] < i) lo = m + 1; else hi = m; }
    return lo < j1 && lg[tgq[lo]] == i ? (int64_t)lo : -1;
  };
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (uint32_t base = 0; base < nb; base += blockDim.x) {
    const uint32_t i = base + threadIdx.x;
    uint32_t c = 0;
    int64_t tj = -1;
    if (i < nb) {
      tj = touched(i);
      if (tj >= 0) {
        c = tgo[tj] & 63u;
      } else {
        const int64_t pj = i > 0 ? touched(i - 1) : -1;
        c = (pj >= 0 && ((tgo[pj] >> 6) & 1u)) ? 0u : 1u;
      }
    }
    uint32_t tot;
    const uint32_t ex = block_excl_scan<uint32_t, 256>(c, ws, tot);
    const uint32_t pos = carry + ex;
    if (i < nb) {
      if (tj >= 0) {
        for (uint32_t t = 0; t < c; t++) G.hdir[e1 + pos + t] = tgb[tj * HB_OUT + t];
      } else if (c) {
        G.hdir[e1 + pos] = G.hdir[e0 + i];
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) carry += tot;
    __syncthreads();
  }
  const uint32_t nbn = carry;
  __syncthreads();
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (uint32_t base = 0; base < nbn; base += blockDim.x) {
    const uint32_t e = base + threadIdx.x;
    const uint32_t bid = e < nbn ? G.hdir[e1 + e] : 0u;
    const uint32_t c = e < nbn ? G.bcnt[bid] : 0u;
    uint32_t tot;
    const uint32_t ex = block_excl_scan<uint32_t, 256>(c, ws, tot);
    if (e < nbn) {
      G.hpre[e1 + e] = carry + ex;
      G.hkey[e1 + e] = G.bmin[bid];
    }
    __syncthreads();
    if (threadIdx.x == 0) carry += tot;
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    G.hub_dir0[h] = e1;
    G.hub_nblk[h] = nbn;
    G.deg[u] = dn;
  }
}

// ---------------------------------------------------------------- rewrite

// A CTA per rewritten hub whose old list fits in shared memory (at most
// HB_RW_SMEM elements): the old list is staged (inline row, then the blocks
// or the PMA segment), every old element and key is written at its new rank
// (ranks below 16 straight to the inline row, whose old contents are
// staged), then the old blocks go to the freed list, the new blocks get
// their counts, first keys and owner, and the directory and the hub table
// entry are written.
constexpr uint32_t HB_RW_SMEM = 48 * 1024;

__global__ void __launch_bounds__(256) k_hub_rw_cta(DevView G, const uint64_t *rp,
                                                    const uint32_t *hw_t, const uint64_t *tpos,
                                                    const uint64_t *bkeys, int insert,
                                                    const uint32_t *bfree, uint64_t F,
                                                    uint64_t fresh0, uint32_t *bfreed,
                                                    unsigned long long *ctr) {
  extern __shared__ uint32_t A[];
  __shared__ unsigned long long fbase;
  const uint64_t *row = rp + (uint64_t)blockIdx.x * RP_W;
  const uint32_t h = (uint32_t)row[RP_H], u = (uint32_t)row[RP_U];
  const uint32_t dold = (uint32_t)row[RP_DO], dn = (uint32_t)row[RP_DN];
  const uint64_t blk0 = row[RP_BLK0], e1 = row[RP_E1];
  const uint32_t per = (uint32_t)row[RP_PER], nbw = (uint32_t)row[RP_NB];
  const uint32_t k = insert ? dn - dold : dold - dn;
  const uint64_t *K = hub_keys(hw_t, tpos, bkeys, row[RP_IHW]);
  const NbrList L = nbr_list(G, u);  // the old list (tables unchanged until the end)
  const bool was_hub = G.hub_of[u] >= 0;
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarp = blockDim.x >> 5;
  for (uint32_t i = threadIdx.x; i < L.ni; i += blockDim.x) A[i] = L.inl[i];
  if (L.nb) {
    for (uint32_t e = warp; e < L.nb; e += nwarp) {
      const uint32_t *blk = L.seg + (uint64_t)L.dir[e] * HUB_BLOCK;
      const uint32_t c = (e + 1 < L.nb ? L.pre[e + 1] : L.rest) - L.pre[e];
      uint32_t *dst = A + L.ni + L.pre[e];
      for (uint32_t j = lane; j < c; j += 32) dst[j] = blk[j];
    }
  } else {
    for (uint32_t j = threadIdx.x; j < L.rest; j += blockDim.x) A[L.ni + j] = L.seg[j];
  }
  __syncthreads();
  uint32_t *row_inl = G.inl + (uint64_t)u * K_INLINE;
  auto put = [&](uint32_t r, uint32_t x) {
    if (r < K_INLINE) {
      row_inl[r] = x;
    } else {
      const uint32_t rr = r - K_INLINE;
      const uint32_t b = alloc_id(blk0 + rr / per, bfree, F, fresh0);
      G.hslot[(uint64_t)b * HUB_BLOCK + rr % per] = x;
    }
  };
  if (insert) {
    for (uint32_t i = threadIdx.x; i < dold; i += blockDim.x) put(i + lb_u64lo(K, k, A[i]), A[i]);
    for (uint32_t j = threadIdx.x; j < k; j += blockDim.x) {
      const uint32_t x = (uint32_t)K[j];
      put(j + lb_u32(A, dold, x), x);
    }
  } else {
    for (uint32_t i = threadIdx.x; i < dold; i += blockDim.x) {
      const uint32_t x = A[i];
      const uint32_t c = lb_u64lo(K, k, x);
      if (!(c < k && (uint32_t)K[c] == x)) put(i - c, x);
    }
  }
  if (threadIdx.x == 0 && was_hub && L.nb)
    fbase = atomicAdd(ctr + H_FREED, (unsigned long long)L.nb);
  __syncthreads();
  if (was_hub)
    for (uint32_t i = threadIdx.x; i < L.nb; i += blockDim.x) bfreed[fbase + i] = L.dir[i];
  const uint32_t rest = dn > K_INLINE ? dn - K_INLINE : 0;
  for (uint32_t i = threadIdx.x; i < nbw; i += blockDim.x) {
    const uint32_t b = alloc_id(blk0 + i, bfree, F, fresh0);
    const uint32_t c = rest - i * per < per ? rest - i * per : per;
    const uint32_t first = G.hslot[(uint64_t)b * HUB_BLOCK];
    G.bcnt[b] = c;
    G.bmin[b] = first;
    G.bown[b] = u;
    G.hdir[e1 + i] = b;
    G.hpre[e1 + i] = i * per;
    G.hkey[e1 + i] = first;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    G.hub_vtx[h] = u;
    G.hub_dir0[h] = e1;
    G.hub_nblk[h] = nbw;
    G.hub_of[u] = (int32_t)h;
    G.deg[u] = dn;
    atomicAdd(ctr + H_READ, (unsigned long long)dold);
    atomicAdd(ctr + H_WRITE, (unsigned long long)dn);
  }
}

// One thread per item of a rewritten hub (old elements, then insert keys):
// its new rank, then its slot -- the inline staging row for ranks < 16, else
// the hub's fresh blocks, uniformly filled with `per` elements.  The old list
// is read through the unchanged tiers.
__global__ void k_hub_rw_place(DevView G, const uint64_t *rp, uint64_t NR, uint64_t QR,
                               const uint32_t *hw_t, const uint64_t *tpos, const uint64_t *bkeys,
                               int insert, uint32_t *stage, const uint32_t *bfree, uint64_t F,
                               uint64_t fresh0) {
  const uint64_t q = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= QR) return;
  const uint64_t r = row_of(rp, NR, RP_W, RP_Q0, q);
  const uint64_t *row = rp + r * RP_W;
  const uint32_t u = (uint32_t)row[RP_U], dold = (uint32_t)row[RP_DO], dn = (uint32_t)row[RP_DN];
  const uint32_t k = insert ? dn - dold : dold - dn;
  const uint64_t *K = hub_keys(hw_t, tpos, bkeys, row[RP_IHW]);
  const uint32_t z = (uint32_t)(q - row[RP_Q0]);
  const NbrList L = nbr_list(G, u);
  uint32_t x, rank;
  if (z < dold) {
    x = L.at(z);
    const uint32_t c = lb_u64lo(K, k, x);
    if (insert) {
      rank = z + c;
    } else {
      if (c < k && (uint32_t)K[c] == x) return;
      rank = z - c;
    }
  } else {
    const uint32_t jj = z - dold;
    x = (uint32_t)K[jj];
    rank = jj + list_lower_bound(L, x);
  }
  if (rank < K_INLINE) {
    stage[r * K_INLINE + rank] = x;
  } else {
    const uint32_t rr = rank - K_INLINE, per = (uint32_t)row[RP_PER];
    const uint32_t b = alloc_id(row[RP_BLK0] + rr / per, bfree, F, fresh0);
    G.hslot[(uint64_t)b * HUB_BLOCK + rr % per] = x;
  }
}

// CTA per rewritten hub: inline row from the staging row, the old blocks to
// the freed list, the new blocks' counts / first keys / owner, the directory,
// the hub table entry and the degree.
__global__ void k_hub_rw_finish(DevView G, const uint64_t *rp, const uint32_t *stage,
                                uint32_t *bfreed, unsigned long long *ctr, const uint32_t *bfree,
                                uint64_t F, uint64_t fresh0) {
  const uint64_t r = blockIdx.x;
  const uint64_t *row = rp + r * RP_W;
  const uint32_t h = (uint32_t)row[RP_H], u = (uint32_t)row[RP_U], dn = (uint32_t)row[RP_DN];
  const uint32_t dold = (uint32_t)row[RP_DO];
  const uint64_t blk0 = row[RP_BLK0], e1 = row[RP_E1];
  const uint32_t per = (uint32_t)row[RP_PER], nbw = (uint32_t)row[RP_NB];
  const uint32_t ni = dn < K_INLINE ? dn : K_INLINE;
  const uint32_t rest = dn - ni;
  for (uint32_t i = threadIdx.x; i < ni; i += blockDim.x)
    G.inl[(uint64_t)u * K_INLINE + i] = stage[r * K_INLINE + i];
  __shared__ unsigned long long fbase;
  const bool was_hub = G.hub_of[u] >= 0;
  const uint64_t e0 = was_hub ? G.hub_dir0[h] : 0;
  const uint32_t nb = was_hub ? G.hub_nblk[h] : 0;
  if (threadIdx.x == 0 && nb) fbase = atomicAdd(ctr + H_FREED, (unsigned long long)nb);
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < nb; i += blockDim.x) bfreed[fbase + i] = G.hdir[e0 + i];
  for (uint32_t i = threadIdx.x; i < nbw; i += blockDim.x) {
    const uint32_t b = alloc_id(blk0 + i, bfree, F, fresh0);
    const uint32_t c = rest - i * per < per ? rest - i * per : per;
    const uint32_t first = G.hslot[(uint64_t)b * HUB_BLOCK];
    G.bcnt[b] = c;
    G.bmin[b] = first;
    G.bown[b] = u;
    G.hdir[e1 + i] = b;
    G.hpre[e1 + i] = i * per;
    G.hkey[e1 + i] = first;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    G.hub_vtx[h] = u;
    G.hub_dir0[h] = e1;
    G.hub_nblk[h] = nbw;
    G.hub_of[u] = (int32_t)h;
    G.deg[u] = dn;
    atomicAdd(ctr + H_READ, (unsigned long long)dold);
    atomicAdd(ctr + H_WRITE, (unsigned long long)dn);
  }
}

// The free list after the batch: the entries the splits did not take (its
// bottom F - min(F, allocated)), then the blocks freed.
__global__ void k_hub_free_merge(uint32_t *bfree, uint64_t F, uint64_t R, const uint32_t *bfreed,
                                 const unsigned long long *ctr) {
  const uint64_t nf = ctr[H_FREED], na = R + ctr[H_ALLOC];
  const uint64_t keep = F - (na < F ? na : F);
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nf;
       i += (uint64_t)gridDim.x * blockDim.x)
    bfree[keep + i] = bfreed[i];
}

// ---------------------------------------------------------------- host side

void Graph::hub_init() {
  // the staged rewrite may use up to 192 KB of dynamic shared memory; the
  // limit applies per device (a graph is created with its device current)
  TRC_CUDA(cudaFuncSetAttribute(k_hub_rw_cta, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)(HB_RW_SMEM * sizeof(uint32_t))));
  grow_hub_tables(64);
  grow_pool(64);
  grow_dir_pool(256);
}

void Graph::grow_hub_tables(uint32_t need) {
  uint64_t cap = hub_vtx.capacity();
  if (need <= cap && cap) return;
  uint64_t nc = std::max<uint64_t>(need, cap * 2);
  hub_vtx.grow(nc, H, stream);
  hub_nblk.grow(nc, H, stream);
  hub_dir0.grow(nc, H, stream);
}

void Graph::grow_pool(uint64_t need_blocks) {
  if (need_blocks <= NBP) return;
  uint64_t nc = std::max<uint64_t>(need_blocks, NBP * 2);
  hslot.grow(nc * HUB_BLOCK, pool_top * HUB_BLOCK, stream);
  bcnt.grow(nc, pool_top, stream);
  bmin.grow(nc, pool_top, stream);
  bown.grow(nc, pool_top, stream);
  bfree.grow(nc, nfree, stream);
  NBP = nc;
}

void Graph::grow_dir_pool(uint64_t need) {
  if (need <= DP) return;
  uint64_t nc = std::max<uint64_t>(need, DP * 2);
  hdir.grow(nc, dir_top, stream);
  hpre.grow(nc, dir_top, stream);
  hkey.grow(nc, dir_top, stream);
  DP = nc;
}

uint32_t *Graph::hub_pin(uint64_t words) {
  if (words > hub_pin_cap_) {
    if (hub_pin_) {
      TRC_CUDA(cudaStreamSynchronize(side_stream));
      TRC_CUDA(cudaFreeHost(hub_pin_));
      hub_pin_ = nullptr;
    }
    const uint64_t cap = std::max<uint64_t>(words, 2 * hub_pin_cap_);
    TRC_CUDA(cudaMallocHost(&hub_pin_, cap * 4));
    hub_pin_cap_ = cap;
  }
  return hub_pin_;
}

// Directory entries for a hub that will have nb blocks: the half not in use
// of its region, or a new region of two halves when that is too small.
uint64_t Graph::hub_dir_target(uint32_t h, uint32_t nb) {
  if (h_hub_dcap[h] && nb <= h_hub_dcap[h]) {
    h_hub_dside[h] ^= 1;
    return h_hub_dbase[h] + (uint64_t)h_hub_dside[h] * h_hub_dcap[h];
  }
  const uint32_t cap = std::max<uint32_t>(4, 2 * nb);
  h_hub_dbase[h] = dir_top;
  h_hub_dcap[h] = cap;
  h_hub_dside[h] = 0;
  dir_top += 2ull * cap;
  return h_hub_dbase[h];
}

void Graph::apply_hubs(uint64_t nh, const std::vector<uint32_t> &hu,
                       const std::vector<uint32_t> &hdn, const std::vector<int32_t> &hh,
                       const std::vector<uint32_t> &hdo, const uint32_t *hw_t,
                       const uint64_t *bkeys, const uint64_t *tpos, bool insert) {
  HubCtx &c = hub_ctx_;
  c = HubCtx{};
  c.insert = insert;
  c.hw_t = hw_t;
  c.bkeys = bkeys;
  c.tpos = tpos;
  c.hu = &hu;
  c.hdn = &hdn;
  c.hdo = &hdo;
  uint64_t *cnt = s_cnt.get();
  unsigned long long *ctr = reinterpret_cast<unsigned long long *>(cnt);
  const double fillf = cfg.hub_block_fill > 0 && cfg.hub_block_fill <= 1 ? cfg.hub_block_fill : 0.75;
  c.fill = std::max<uint32_t>(1, (uint32_t)(HUB_BLOCK * fillf));
  const uint32_t gk = std::max<uint32_t>(1, std::min<uint32_t>(cfg.hub_stage_limit, HB_GK));
  for (auto &x : hub_last) x = 0;
  hub_last[0] = nh;

  // ---- hub indices for new hubs; block-local or rewrite
  uint64_t freed_bound = 2;
  for (uint64_t i = 0; i < nh; i++) {
    int32_t h = hh[i];
    bool rewrite = false;
    if (h < 0) {
      h = (int32_t)H++;
      h_hub_vtx.push_back(hu[i]);
      h_hub_nblk.push_back(0);
      h_hub_dcap.push_back(0);
      h_hub_dbase.push_back(0);
      h_hub_dside.push_back(0);
      rewrite = true;
    } else {
      const uint32_t nbo = h_hub_nblk[h];
      const uint32_t rest_old = hdo[i] > K_INLINE ? hdo[i] - K_INLINE : 0;
      const uint32_t rest_new = hdn[i] > K_INLINE ? hdn[i] - K_INLINE : 0;
      const uint32_t k = insert ? hdn[i] - hdo[i] : hdo[i] - hdn[i];
      rewrite = nbo == 0 || hdo[i] < HB_LOCAL_MIN || (insert && k > rest_old) ||
                rest_new < 2 * HB_MIN;
      freed_bound += nbo;
    }
    (rewrite ? c.rw : c.loc).push_back({i, (uint32_t)h});
  }
  grow_hub_tables(H);

  // ---- block-local hubs: plan rows, then locate every key and count the
  // touched groups on the side stream
  const uint64_t NL = c.loc.size();
  uint64_t QL = 0;
  c.lp.assign(NL * LP_W, 0);
  for (uint64_t li = 0; li < NL; li++) {
    const uint64_t i = c.loc[li].i;
    uint64_t *row = &c.lp[li * LP_W];
    row[LP_H] = c.loc[li].h;
    row[LP_U] = hu[i];
    row[LP_IHW] = i;
    row[LP_Q0] = QL;
    row[LP_DN] = hdn[i];
    QL += insert ? hdn[i] - hdo[i] : hdo[i] - hdn[i];
  }
  c.NL = NL;
  c.QL = QL;
  // scratch, all taken here, before the fork (allocations are stream-ordered
  // on the graph's stream)
  c.d_lp = s_hplan.ensure(NL * LP_W + 2 * nh * RP_W + 2 * nh + 4);
  c.lli = s_lli.ensure(QL + 1);
  c.lg = s_lg.ensure(QL + 1);
  c.lx = s_lx.ensure(QL + 1);
  c.tgq = s_tgq.ensure(QL + 1);
  c.tgo = s_tgo.ensure(QL + 1);
  c.tgb = s_tgb.ensure((QL + 1) * HB_OUT);
  c.hflag = s_hflag.ensure(NL + 1);
  c.hnbd = s_hnbd.ensure(NL + 1);
  c.stage = s_rwstage.ensure((uint64_t)nh * K_INLINE + 1);
  freed_bound += 2 * QL;
  c.freed = bfreed.ensure(freed_bound);
  uint64_t *st = s_hsel.ensure(select_tmp_elems(std::max<uint64_t>(QL, 1)) + 4);
  TRC_CUDA(cudaMemsetAsync(cnt + H_NTG, 0, (H_ALLOC_REQ - H_NTG + 1) * 8, stream));
  if (NL) {
    TRC_CUDA(cudaMemsetAsync(c.hflag, 0, NL * 4, stream));
    TRC_CUDA(cudaMemsetAsync(c.hnbd, 0, NL * 4, stream));
  }
  TRC_CUDA(cudaEventRecord(ev_fork, stream));
  TRC_CUDA(cudaStreamWaitEvent(side_stream, ev_fork, 0));
  cudaStream_t z = side_stream;
  const DevView G = view();
  c.pin = hub_pin(2 * NL + 16);
  if (NL) {
    TRC_CUDA(cudaMemcpyAsync(c.d_lp, c.lp.data(), c.lp.size() * 8, cudaMemcpyHostToDevice, z));
    TRC_LAUNCH(prof, z, "hub_locate", ceil_div(QL, 256), 256, 0, k_hub_locate, G, c.d_lp, NL, QL,
               hw_t, tpos, bkeys, c.lli, c.lg, c.lx);
    select_if(GroupStartPred{c.lli, c.lg}, IndexVal32H{}, QL, c.tgq, cnt + H_NTG, st, z, prof,
              "hub_groups");
    TRC_LAUNCH(prof, z, "hub_count", ceil_div(QL, 256), 256, 0, k_hub_count, G, c.d_lp, cnt, QL,
               c.tgq, c.lli, c.lg, insert ? 1 : 0, gk, c.fill, c.tgo, c.hflag, c.hnbd,
               ctr + H_ALLOC_REQ);
    TRC_CUDA(cudaMemcpyAsync(c.pin, cnt + H_NTG, 8, cudaMemcpyDeviceToHost, z));
    TRC_CUDA(cudaMemcpyAsync(c.pin + 2, cnt + H_ALLOC_REQ, 8, cudaMemcpyDeviceToHost, z));
    TRC_CUDA(cudaMemcpyAsync(c.pin + 16, c.hflag, NL * 4, cudaMemcpyDeviceToHost, z));
    TRC_CUDA(cudaMemcpyAsync(c.pin + 16 + NL, c.hnbd, NL * 4, cudaMemcpyDeviceToHost, z));
    TRC_CUDA(cudaEventRecord(ev_hub, z));
  }
  c.active = true;
}

void Graph::apply_hubs_finish() {
  HubCtx &c = hub_ctx_;
  if (!c.active) return;
  c.active = false;
  uint64_t *cnt = s_cnt.get();
  unsigned long long *ctr = reinterpret_cast<unsigned long long *>(cnt);
  const std::vector<uint32_t> &hu = *c.hu, &hdn = *c.hdn, &hdo = *c.hdo;
  const bool insert = c.insert;
  const uint64_t NL = c.NL, QL = c.QL;
  uint64_t ntg = 0, alloc_req = 0;
  std::vector<uint8_t> flagged(NL, 0);
  std::vector<int32_t> nbd(NL, 0);
  if (NL) {
    TRC_CUDA(cudaEventSynchronize(ev_hub));
    memcpy(&ntg, c.pin, 8);
    memcpy(&alloc_req, c.pin + 2, 8);
    for (uint64_t li = 0; li < NL; li++) {
      flagged[li] = c.pin[16 + li] != 0;
      nbd[li] = (int32_t)c.pin[16 + NL + li];
    }
  }
  // ---- flagged block-local hubs take the rewrite path too
  std::vector<HubItem> rw = c.rw;
  uint64_t nloc = 0;
  for (uint64_t li = 0; li < NL; li++) {
    if (flagged[li]) rw.push_back(c.loc[li]);
    else nloc++;
  }
  const uint64_t NR = rw.size();
  // ---- blocks, by allocation index (free list top first, then fresh):
  // each rewritten hub a planned range of indices, then the splits from a
  // device counter (alloc_req bounds them: groups of hubs flagged later
  // allocate nothing, so the pool top is set from the device's count)
  const uint64_t F = nfree;
  const uint64_t fresh0 = pool_top;
  uint64_t R = 0;
  // rows: hubs whose old list fits in shared memory (a CTA each, staged)
  // first, then the others (a thread per element)
  std::vector<uint64_t> rp(NR * RP_W, 0);
  std::stable_partition(rw.begin(), rw.end(),
                        [&](const HubItem &x) { return hdo[x.i] <= HB_RW_SMEM; });
  uint64_t NRC = 0;
  uint32_t smem_max = 1;
  while (NRC < NR && hdo[rw[NRC].i] <= HB_RW_SMEM) smem_max = std::max(smem_max, hdo[rw[NRC++].i]);
  uint64_t QR = 0, written_blocks = 0;
  for (uint64_t r = 0; r < NR; r++) {
    const uint64_t i = rw[r].i;
    const uint32_t h = rw[r].h;
    const uint32_t rest = hdn[i] > K_INLINE ? hdn[i] - K_INLINE : 0;
    const uint32_t nb = rest ? (uint32_t)ceil_div(rest, c.fill) : 0;
    const uint32_t per = nb ? (uint32_t)ceil_div(rest, nb) : 1;
    uint64_t *row = &rp[r * RP_W];
    row[RP_H] = h;
    row[RP_U] = hu[i];
    row[RP_IHW] = i;
    row[RP_DO] = hdo[i];
    row[RP_DN] = hdn[i];
    row[RP_BLK0] = R;
    row[RP_PER] = per;
    row[RP_NB] = nb;
    row[RP_Q0] = QR;
    if (r >= NRC) QR += insert ? hdn[i] : hdo[i];  // old elements (+ keys on insert)
    R += nb;
    written_blocks += nb;
    h_hub_nblk[h] = nb;
    row[RP_E1] = hub_dir_target(h, nb);
  }
  const uint64_t top_bound = fresh0 + (R + alloc_req > F ? R + alloc_req - F : 0);
  std::vector<uint64_t> e1s(NL, 0);
  for (uint64_t li = 0; li < NL; li++) {
    if (flagged[li]) continue;
    const uint32_t h = c.loc[li].h;
    const uint32_t nbn = (uint32_t)((int64_t)h_hub_nblk[h] + nbd[li]);
    h_hub_nblk[h] = nbn;
    e1s[li] = hub_dir_target(h, nbn);
  }
  // ---- capacity (a growth synchronises the graph's stream, then the side
  // stream waits for it: allocations are stream-ordered)
  const uint64_t nbp = NBP, dp = DP;
  grow_pool(top_bound);
  grow_dir_pool(dir_top);
  if (NBP != nbp || DP != dp) {
    TRC_CUDA(cudaEventRecord(ev_fork, stream));
    TRC_CUDA(cudaStreamWaitEvent(side_stream, ev_fork, 0));
  }
  cudaStream_t z = side_stream;
  const DevView G = view();
  uint64_t *d_rp = c.d_lp + NL * LP_W;
  uint64_t *d_e1 = d_rp + NR * RP_W;
  if (NR) TRC_CUDA(cudaMemcpyAsync(d_rp, rp.data(), rp.size() * 8, cudaMemcpyHostToDevice, z));
  if (NL) TRC_CUDA(cudaMemcpyAsync(d_e1, e1s.data(), NL * 8, cudaMemcpyHostToDevice, z));
  // ---- block-local merges and directories
  if (NL && ntg) {
    TRC_LAUNCH(prof, z, "hub_merge_group", ntg, 256, 0, k_hub_merge_group, G, c.d_lp, cnt, QL,
               c.tgq, c.lli, c.lg, c.lx, c.tgo, c.hflag, insert ? 1 : 0, bfree.get(), F, fresh0,
               R, c.freed, c.tgb, ctr);
    TRC_LAUNCH(prof, z, "hub_dir", NL, 256, 0, k_hub_dir, G, c.d_lp, NL, cnt, QL, c.tgq, c.lg,
               c.tgo, c.tgb, c.hflag, d_e1);
  }
  // ---- rewrites
  if (NRC)
    TRC_LAUNCH(prof, z, "hub_rw_cta", NRC, 256, (size_t)smem_max * 4, k_hub_rw_cta, G, d_rp,
               c.hw_t, c.tpos, c.bkeys, insert ? 1 : 0, bfree.get(), F, fresh0, c.freed, ctr);
  if (NR > NRC) {
    const uint64_t *d_rpe = d_rp + NRC * RP_W;
    TRC_LAUNCH(prof, z, "hub_rw_place", ceil_div(QR, 256), 256, 0, k_hub_rw_place, G, d_rpe,
               NR - NRC, QR, c.hw_t, c.tpos, c.bkeys, insert ? 1 : 0, c.stage, bfree.get(), F,
               fresh0);
    TRC_LAUNCH(prof, z, "hub_rw_finish", NR - NRC, 256, 0, k_hub_rw_finish, G, d_rpe, c.stage,
               c.freed, ctr, bfree.get(), F, fresh0);
  }
  // ---- the free list: what the splits did not take, then the freed blocks
  // (free ids are distinct pool blocks, so bfree's pool-sized capacity holds
  // them all)
  TRC_LAUNCH(prof, z, "hub_free_merge", (unsigned)num_sms(), 256, 0, k_hub_free_merge, bfree.get(),
             F, R, c.freed, ctr);
  TRC_CUDA(cudaMemcpyAsync(c.pin + 4, cnt + H_ALLOC, 8 * 5, cudaMemcpyDeviceToHost, z));
  TRC_CUDA(cudaEventRecord(ev_join, z));
  TRC_CUDA(cudaStreamWaitEvent(stream, ev_join, 0));
  c.F = F;
  c.fresh0 = fresh0;
  c.R = R;
  c.readback = true;
  pool_top = top_bound;  // corrected to the blocks taken in hubs_finish
  hub_last[1] = nloc;
  hub_last[2] = NR;
  hub_last[3] = written_blocks;
  hub_rewrites += NR;
}

// After the batch's final synchronisation: the free list's size and the
// elements the tier-3 kernels read and wrote.
void Graph::hubs_finish() {
  HubCtx &c = hub_ctx_;
  if (!c.readback) return;
  c.readback = false;
  uint64_t v[5];
  memcpy(v, c.pin + 4, sizeof(v));  // H_ALLOC, H_FREED, H_READ, H_WRITE, H_ABSORB
  const uint64_t allocated = c.R + v[0];
  const uint64_t from_free = std::min<uint64_t>(c.F, allocated);
  nfree = c.F - from_free + v[1];
  pool_top = c.fresh0 + (allocated - from_free);
  hub_splits += v[0];
  hub_last[3] += v[0];
  hub_last[4] = v[2];
  hub_last[5] = v[3];
  hub_absorbs += v[4];
}

}  // namespace trc
