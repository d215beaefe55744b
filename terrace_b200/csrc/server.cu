// server.cu -- continuous-batching request server over one device-resident
// graph (the serving layer; the reference has no serving mode and no
// concurrency between updates and analytics, include/graph.h:73-230).
//
// A persistent worker thread runs rounds.  In BATCHED mode a round takes
// every request pending when it starts:
//   1. queries run against the current snapshot (version v): BFS requests
//      are packed 64 at a time into multi-source BFS launches, degree
//      lookups into one launch, PageRank requests with equal iteration
//      counts share one computation;
//   2. then all updates of the round are applied as ONE net change: their
//      keys (symmetrized when configured) carry the request's arrival rank,
//      one radix sort groups equal edges, the last request touching an edge
//      decides insert or delete, and the graph receives one delete batch and
//      one insert batch -> version v+1.
// Requests pending together have not completed when the others arrived, so
// any order between them is a valid linearisation; "queries of a round,
// then its updates" is the order used, and every request records the
// snapshot version it observed (trc_server_result) so a test can replay it
// alone.  Requests that arrive while a round is on the GPU join the next
// round.  Update admission is bounded by max_round_edges and by the graph's
// HBM budget: an update whose estimated working memory does not fit waits
// for a later round (alone in a round it fails with TRC_ERR_NOMEM).
// FIFO mode runs one request per round in arrival order (the plain path).
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstring>
#include <string>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "graph.cuh"

namespace trc {

namespace {

double now_ms() {
  return std::chrono::duration<double, std::milli>(
             std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

struct Request {
  uint64_t id;
  trc_request_kind kind;
  std::vector<uint32_t> a, b;
  uint32_t param = 0;
  double t_arrive = 0, t_done = 0;
  uint64_t version = 0;  // snapshot observed (queries) / produced (updates)
  std::vector<uint32_t> out_u32;
  std::vector<double> out_f64;
  uint64_t out_count = 0;
  trc_status status = TRC_OK;
  bool done = false;
  bool in_round = false;  // taken by the worker; deleted by it if released meanwhile
  bool released = false;
};

// reached count and deepest level of one level array (summary of a BFS)
__global__ void k_level_summary(const uint32_t *lv, uint32_t n, unsigned long long *reached,
                                uint32_t *depth) {
  uint32_t c = 0, d = 0;
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n;
       v += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t x = lv[v];
    if (x != TRC_UNREACHED) {
      c++;
      d = max(d, x);
    }
  }
  c = __reduce_add_sync(0xFFFFFFFFu, c);
  d = __reduce_max_sync(0xFFFFFFFFu, d);
  if ((threadIdx.x & 31) == 0) {
    if (c) atomicAdd(reached, (unsigned long long)c);
    atomicMax(depth, d);
  }
}

__global__ void k_fill_f64(double *x, uint32_t n, double v) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] = v;
}

// per-block partial sum and max of a rank vector; the host adds the
// partials in block order, so the sum does not depend on scheduling
__global__ void k_rank_summary(const double *x, uint32_t n, double *part) {
  __shared__ double ss[8], sm[8];
  double s = 0, m = 0;
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n;
       v += (uint64_t)gridDim.x * blockDim.x) {
    s += x[v];
    m = fmax(m, x[v]);
  }
  for (int o = 16; o > 0; o >>= 1) {
    s += __shfl_xor_sync(0xFFFFFFFFu, s, o);
    m = fmax(m, __shfl_xor_sync(0xFFFFFFFFu, m, o));
  }
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    ss[w] = s;
    sm[w] = m;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int i = 1; i < (int)(blockDim.x >> 5); i++) {
      s += ss[i];
      m = fmax(m, sm[i]);
    }
    part[2 * blockIdx.x] = s;
    part[2 * blockIdx.x + 1] = m;
  }
}

// tags every pair with its request's arrival rank and operation: one launch
// over the round's concatenated pairs, the request found by binary search
// over its offsets
__global__ void k_tag_round(const uint32_t *src, const uint32_t *dst, uint64_t k,
                            const uint64_t *roff, const uint32_t *rop, uint32_t nreq, uint32_t n,
                            int sym, uint32_t vb, uint32_t tagbits, uint64_t *out, uint32_t *err) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= k) return;
  uint32_t lo = 0, hi = nreq;  // last request with roff[r] <= i
  while (hi - lo > 1) {
    uint32_t mid = (lo + hi) >> 1;
    if (roff[mid] <= i) lo = mid;
    else hi = mid;
  }
  const uint64_t tag = ((uint64_t)lo << 1) | rop[lo];
  uint32_t s = src[i], d = dst[i];
  uint64_t a = ~0ull, b = ~0ull;
  if (s >= n || d >= n) {
    atomicOr(err, 1u);
  } else if (s != d) {
    a = ((((uint64_t)s << vb) | d) << tagbits) | tag;
    b = ((((uint64_t)d << vb) | s) << tagbits) | tag;
  }
  if (sym) {
    out[2 * i] = a;
    out[2 * i + 1] = b;
  } else {
    out[i] = a;
  }
}

// last entry of each edge group decides; op bit 1 = insert
struct LastOpPred {
  const uint64_t *k;
  uint64_t nk;
  uint32_t tagbits;
  int want_insert;
  __device__ bool operator()(uint64_t i) const {
    uint64_t x = k[i];
    if (x == ~0ull) return false;
    if (i + 1 < nk && (k[i + 1] >> tagbits) == (x >> tagbits)) return false;
    return (int)(x & 1u) == want_insert;
  }
};

struct KeySrc {
  const uint64_t *k;
  uint32_t shift, vb;
  __device__ uint32_t operator()(uint64_t i) const { return (uint32_t)(k[i] >> (shift + vb)); }
};
struct KeyDst {
  const uint64_t *k;
  uint32_t shift, vb;
  __device__ uint32_t operator()(uint64_t i) const {
    return (uint32_t)((k[i] >> shift) & ((1ull << vb) - 1));
  }
};

}  // namespace

class Server {
 public:
  Server(Graph &g, const trc_server_config &c) : g_(g), cfg_(c) {
    if (!cfg_.max_round_edges) cfg_.max_round_edges = 1ull << 24;
    if (!cfg_.max_bfs_group || cfg_.max_bfs_group > 64) cfg_.max_bfs_group = 64;
    t0_ = now_ms();
    worker_ = std::thread([this] { loop(); });
  }
  ~Server() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    worker_.join();
    for (auto &kv : all_) delete kv.second;
  }

  uint64_t submit(trc_request_kind kind, const uint32_t *a, const uint32_t *b, uint64_t k,
                  uint32_t param) {
    Request *r = new Request();
    r->kind = kind;
    r->param = param;
    if (a) r->a.assign(a, a + k);
    if (b) r->b.assign(b, b + k);
    r->t_arrive = now_ms();
    std::lock_guard<std::mutex> lk(mu_);
    r->id = next_id_++;
    all_[r->id] = r;
    pending_.push_back(r);
    cv_.notify_all();
    return r->id;
  }

  // While held, the worker starts no new round and requests queue up; on
  // release the next round takes every pending request (subject to the
  // admission limits).  Destroying a held server still drains it.
  void hold(bool on) {
    std::lock_guard<std::mutex> lk(mu_);
    hold_ = on;
    cv_.notify_all();
  }

  trc_status wait(uint64_t id, int64_t timeout_ms) {
    std::unique_lock<std::mutex> lk(mu_);
    auto it = all_.find(id);
    if (it == all_.end()) throw_error(TRC_ERR_INVALID, "unknown request id");
    Request *r = it->second;
    auto pred = [&] { return r->done; };
    if (timeout_ms < 0) {
      done_cv_.wait(lk, pred);
    } else if (!done_cv_.wait_for(lk, std::chrono::milliseconds(timeout_ms), pred)) {
      return TRC_ERR_TIMEOUT;
    }
    return TRC_OK;
  }

  void result(uint64_t id, void *out, uint64_t cap, uint64_t *bytes, double *lat, uint64_t *ver,
              trc_status *st) {
    std::lock_guard<std::mutex> lk(mu_);
    auto it = all_.find(id);
    if (it == all_.end()) throw_error(TRC_ERR_INVALID, "unknown request id");
    Request *r = it->second;
    if (!r->done) throw_error(TRC_ERR_STATE, "request not finished");
    uint64_t nb;
    const void *src;
    if (is_update(r->kind)) {
      nb = 8;
      src = &r->out_count;
    } else if (r->kind == TRC_REQ_PAGERANK) {
      nb = r->out_f64.size() * 8;
      src = r->out_f64.data();
    } else {  // may be empty (an isolated vertex's neighbours)
      nb = r->out_u32.size() * 4;
      src = r->out_u32.data();
    }
    if (bytes) *bytes = nb;
    if (out && cap && nb) memcpy(out, src, nb < cap ? nb : cap);
    if (lat) *lat = r->t_done - r->t_arrive;
    if (ver) *ver = r->version;
    if (st) *st = r->status;
  }

  void release(uint64_t id) {
    std::lock_guard<std::mutex> lk(mu_);
    auto it = all_.find(id);
    if (it == all_.end()) return;
    Request *r = it->second;
    if (!r->done) throw_error(TRC_ERR_STATE, "request not finished");
    all_.erase(it);
    if (r->in_round) r->released = true;  // the worker still holds it
    else delete r;
  }

  void stats(int kind, trc_server_stats *o) {
    std::lock_guard<std::mutex> lk(mu_);
    std::vector<double> lat;
    for (auto &p : lat_)
      if (kind < 0 || p.first == kind) lat.push_back(p.second);
    std::sort(lat.begin(), lat.end());
    memset(o, 0, sizeof(*o));
    o->completed = lat.size();
    o->elapsed_s = ((last_done_ > 0 ? last_done_ : now_ms()) - t0_) / 1e3;
    if (!lat.empty()) {
      o->p50_ms = lat[(size_t)(0.50 * (lat.size() - 1))];
      o->p99_ms = lat[(size_t)(0.99 * (lat.size() - 1))];
      double s = 0;
      for (double x : lat) s += x;
      o->mean_ms = s / lat.size();
      o->max_ms = lat.back();
    }
    o->rounds = rounds_;
    o->device_calls = calls_;
    o->rejected = rejected_;
    o->version = version_;
    o->worst_round_ms = worst_.ms;
    o->worst_update_ms = worst_.upd_ms;
    o->worst_bfs_ms = worst_.bfs_ms;
    o->worst_pagerank_ms = worst_.pr_ms;
    o->worst_round_requests = worst_.requests;
    o->worst_round_rebuilds = worst_.rebuilds;
    o->pma_rebuilds = rebuilds_;
  }

  void reset_stats() {
    std::lock_guard<std::mutex> lk(mu_);
    lat_.clear();
    t0_ = now_ms();
    last_done_ = 0;
    rounds_ = calls_ = rejected_ = 0;
    worst_ = RoundInfo();
    rebuilds_ = 0;
    trace_.clear();
    trace_next_ = 0;
  }

  uint64_t rounds_trace(trc_round_record *out, uint64_t cap) {
    std::lock_guard<std::mutex> lk(mu_);
    const uint64_t held = trace_.size();
    const uint64_t first = held < kTrace ? 0 : trace_next_ % kTrace;
    for (uint64_t i = 0; i < held && i < cap; i++) out[i] = trace_[(first + i) % held];
    return held;
  }

 private:
  Graph &g_;
  trc_server_config cfg_;
  std::thread worker_;
  std::mutex mu_;
  std::condition_variable cv_, done_cv_;
  std::deque<Request *> pending_;
  std::unordered_map<uint64_t, Request *> all_;
  uint64_t next_id_ = 1;
  bool stop_ = false;
  bool hold_ = false;
  std::vector<std::pair<int, double>> lat_;
  double t0_ = 0, last_done_ = 0;
  std::atomic<uint64_t> rounds_{0}, calls_{0}, rejected_{0}, version_{0};
  DBuf<uint64_t> keys_[2], roff_;
  DBuf<uint32_t> ins_s_, ins_d_, del_s_, del_d_, up_s_, up_d_, rop_, lvl_;
  DBuf<int32_t> par_;
  DBuf<double> ranks_, pr0_, pr1_, pr_part_;
  DBuf<uint64_t> red_;
  bool bufs_bound_ = false;
  cudaStream_t s1_ = nullptr;  // the graph's stream while serving (high priority)
  cudaStream_t s2_ = nullptr;  // PageRank overlapping the BFS groups (low priority)
  double *pin_ = nullptr;      // pinned PageRank partial sums
  unsigned pin_cap_ = 0;
  std::vector<std::pair<size_t, size_t>> pr_groups_;
  struct RoundInfo {
    double ms = 0, upd_ms = 0, bfs_ms = 0, pr_ms = 0;
    uint64_t requests = 0, rebuilds = 0;
  } worst_;                    // guarded by mu_
  uint64_t rebuilds_ = 0;      // guarded by mu_
  static constexpr size_t kTrace = 1u << 16;
  std::vector<trc_round_record> trace_;  // ring of the last kTrace rounds, guarded by mu_
  uint64_t trace_next_ = 0;              // guarded by mu_
  uint32_t round_groups_ = 0, round_singles_ = 0;  // BFS launches of the running round
  size_t pending_at_start_ = 0;                    // queue length when it was formed

  void bind_bufs() {
    if (bufs_bound_) return;
    for (auto *b : {&keys_[0], &keys_[1], &roff_, &red_}) b->bind(&g_.budget);
    for (auto *b : {&ins_s_, &ins_d_, &del_s_, &del_d_, &up_s_, &up_d_, &rop_, &lvl_})
      b->bind(&g_.budget);
    par_.bind(&g_.budget);
    for (auto *b : {&ranks_, &pr0_, &pr1_, &pr_part_}) b->bind(&g_.budget);
    bufs_bound_ = true;
  }

  unsigned reduce_grid() const {
    return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(ceil_div(g_.n, 256),
                                                              (uint64_t)num_sms() * 4));
  }

  // single-source BFS summary on the device: {reached, deepest level}
  void bfs_summary(uint32_t src, uint64_t *reached, uint32_t *depth) {
    const uint32_t n = g_.n;
    uint32_t *lv = lvl_.ensure(n);
    int32_t *par = par_.ensure(n);
    g_.bfs(src, par, lv, TRC_DEVICE_PTR);
    uint64_t *red = red_.ensure(2);
    cudaStream_t st = g_.stream;
    TRC_CUDA(cudaMemsetAsync(red, 0, 16, st));
    TRC_LAUNCH(g_.prof, st, "srv_bfs_summary", reduce_grid(), 256, 0, k_level_summary, lv, n,
               (unsigned long long *)red, (uint32_t *)(red + 1));
    uint64_t h[2];
    TRC_CUDA(cudaMemcpyAsync(h, red, 16, cudaMemcpyDeviceToHost, st));
    g_.sync();
    *reached = h[0];
    *depth = (uint32_t)h[1];
  }

  // PageRank summary on the device: {sum, max}
  void pagerank_summary(uint32_t iters, double *sum, double *mx) {
    const uint32_t n = g_.n;
    double *x = ranks_.ensure(n);
    g_.pagerank(iters, 0.0, x, TRC_DEVICE_PTR);
    const unsigned nb = reduce_grid();
    double *part = (double *)red_.ensure(2 * nb);
    cudaStream_t st = g_.stream;
    TRC_LAUNCH(g_.prof, st, "srv_pr_summary", nb, 256, 0, k_rank_summary, x, n, part);
    std::vector<double> h(2 * nb);
    TRC_CUDA(cudaMemcpyAsync(h.data(), part, 16 * nb, cudaMemcpyDeviceToHost, st));
    g_.sync();
    double s = 0, m = 0;
    for (unsigned b = 0; b < nb; b++) {
      s += h[2 * b];
      m = std::max(m, h[2 * b + 1]);
    }
    *sum = s;
    *mx = m;
  }

  static bool is_update(trc_request_kind k) { return k == TRC_REQ_INSERT || k == TRC_REQ_DELETE; }

  // completes requests (each part of a round completes as soon as it is done)
  void finish(std::vector<Request *> &rs) {
    if (rs.empty()) return;
    double t = now_ms();
    std::lock_guard<std::mutex> lk(mu_);
    for (Request *r : rs) {
      if (r->done) continue;
      r->t_done = t;
      r->done = true;
      lat_.push_back({(int)r->kind, r->t_done - r->t_arrive});
    }
    last_done_ = t;
    done_cv_.notify_all();
  }

  // HBM estimate of applying `edges` directed keys: sort buffers + merge
  // staging + a tier-2 rebuild of the grown PMA.
  bool fits(uint64_t edges) {
    if (!g_.budget.limit) return true;
    uint64_t est = edges * 48 + (g_.tier2_total + edges) * 4 * 3;
    return g_.budget.used + est <= g_.budget.limit;
  }

  void loop() {
    cudaSetDevice(g_.device);
    // the round's own work (lookups, updates, BFS) on a high-priority
    // stream, PageRank on a low-priority one: a BFS launched while a
    // PageRank runs gets the SMs as the PageRank's CTAs retire, so the
    // BFS requests complete one by one instead of at the PageRank's end
    int least = 0, greatest = 0;
    cudaDeviceGetStreamPriorityRange(&least, &greatest);
    cudaStream_t user = g_.stream;
    g_.sync();  // work queued on the graph's stream before the server
    if (cudaStreamCreateWithPriority(&s1_, cudaStreamNonBlocking, greatest) == cudaSuccess) {
      g_.stream = s1_;
      g_.budget.stream = s1_;
    } else {
      s1_ = nullptr;
    }
    if (cudaStreamCreateWithPriority(&s2_, cudaStreamNonBlocking, least) != cudaSuccess) s2_ = nullptr;
    while (true) {
      std::vector<Request *> round;
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return stop_ || (!hold_ && !pending_.empty()); });
        if (pending_.empty() && stop_) break;
        pending_at_start_ = pending_.size();
        if (cfg_.mode == TRC_SERVE_FIFO) {
          round.push_back(pending_.front());
          pending_.pop_front();
          round.back()->in_round = true;
        } else {
          // all pending queries, and updates up to the admission limits
          std::deque<Request *> keep;
          uint64_t edges = 0;
          bool blocked = false;
          for (Request *r : pending_) {
            if (!is_update(r->kind)) {
              r->in_round = true;
              round.push_back(r);
              continue;
            }
            uint64_t e = r->a.size() * (cfg_.symmetrize ? 2 : 1);
            bool first = edges == 0;
            if (!blocked && (first || (edges + e <= cfg_.max_round_edges && fits(edges + e)))) {
              r->in_round = true;
              round.push_back(r);
              edges += e;
            } else {
              blocked = true;  // later updates wait too: arrival order among updates
              keep.push_back(r);
            }
          }
          pending_.swap(keep);
        }
      }
      run_round(round);
      rounds_++;
      std::lock_guard<std::mutex> lk(mu_);
      for (Request *r : round) {
        r->in_round = false;
        if (r->released) delete r;
      }
    }
    if (s2_) {
      cudaStreamSynchronize(s2_);
      cudaStreamDestroy(s2_);
    }
    if (s1_) {
      cudaStreamSynchronize(s1_);
      g_.stream = user;
      g_.budget.stream = user;
      cudaStreamDestroy(s1_);
    }
    if (pin_) cudaFreeHost(pin_);
  }

  template <typename F>
  void guarded(std::vector<Request *> &rs, F &&f) {
    try {
      f();
    } catch (const Error &e) {
      if (e.status == TRC_ERR_NOMEM && !rs.empty() && is_update(rs[0]->kind)) rejected_ += rs.size();
      for (Request *r : rs)
        if (!r->done) r->status = e.status;
    } catch (const std::exception &) {
      for (Request *r : rs)
        if (!r->done) r->status = TRC_ERR_STATE;
    }
  }

  // One round, cheapest parts first; every part completes its requests as
  // soon as it is done:
  //   1. degree / neighbour lookups on snapshot v;
  //   2. the updates as one net change -> v+1;
  //   3. PageRank (shared per iteration count) launched on a second stream
  //      and overlapping with
  //   4. the BFS groups (64 sources per multi-source launch) on v+1;
  //   5. PageRank results.
  // Nothing modifies the graph while 3-5 read it.
  void run_round(std::vector<Request *> &round) {
    std::vector<Request *> look, upd, bfs, pr;
    for (Request *r : round) {
      if (is_update(r->kind)) upd.push_back(r);
      else if (r->kind == TRC_REQ_BFS) bfs.push_back(r);
      else if (r->kind == TRC_REQ_PAGERANK) pr.push_back(r);
      else look.push_back(r);
    }
    bind_bufs();
    RoundInfo info;
    info.requests = round.size();
    round_groups_ = round_singles_ = 0;
    trc_round_record rec{};
    rec.lookups = (uint32_t)look.size();
    rec.updates = (uint32_t)upd.size();
    rec.bfs = (uint32_t)bfs.size();
    rec.pageranks = (uint32_t)pr.size();
    for (Request *r : upd) rec.update_pairs += r->a.size();
    rec.pending_after = (uint32_t)(pending_at_start_ - std::min(pending_at_start_, round.size()));
    const uint64_t rb0 = g_.rebuilds;
    const double t0 = now_ms();
    guarded(look, [&] { run_lookups(look); });
    finish(look);
    const double t1 = now_ms();
    if (!upd.empty()) {
      guarded(upd, [&] {
        if (cfg_.mode == TRC_SERVE_FIFO || upd.size() == 1) {
          for (Request *r : upd) apply_one(r);
        } else {
          apply_net(upd);
        }
      });
      finish(upd);
    }
    const double t2 = now_ms();
    for (Request *r : bfs) r->version = version_;
    for (Request *r : pr) r->version = version_;
    bool pr_async = false;
    guarded(pr, [&] { pr_async = start_pagerank(pr); });
    if (!pr_async) finish(pr);  // computed synchronously (or failed)
    const double t3 = now_ms();
    guarded(bfs, [&] { run_bfs(bfs); });
    finish(bfs);  // groups that completed were finished already
    const double t4 = now_ms();
    if (pr_async) {
      guarded(pr, [&] { end_pagerank(pr); });
      finish(pr);
    }
    const double t5 = now_ms();
    info.ms = t5 - t0;
    info.upd_ms = t2 - t1;
    info.bfs_ms = t4 - t3;
    info.pr_ms = (t3 - t2) + (t5 - t4);  // synchronous part + wait after the BFS groups
    info.rebuilds = g_.rebuilds - rb0;
    rec.ms = info.ms;
    rec.lookup_ms = t1 - t0;
    rec.update_ms = info.upd_ms;
    rec.bfs_ms = info.bfs_ms;
    rec.pagerank_ms = info.pr_ms;
    rec.bfs_groups = round_groups_;
    rec.bfs_singles = round_singles_;
    rec.rebuilds = (uint32_t)info.rebuilds;
    std::lock_guard<std::mutex> lk(mu_);
    rec.t_start_ms = t0 - t0_;
    if (trace_.size() < kTrace) trace_.push_back(rec);
    else trace_[trace_next_ % kTrace] = rec;
    trace_next_++;
    rebuilds_ += info.rebuilds;
    if (info.ms > worst_.ms) worst_ = info;
  }

  void run_lookups(std::vector<Request *> &q) {
    const uint32_t n = g_.n;
    std::vector<Request *> deg;
    for (Request *r : q) {
      r->version = version_;
      if (r->kind == TRC_REQ_DEGREE) {
        deg.push_back(r);
        continue;
      }
      if (r->param >= n) {  // neighbours
        r->status = TRC_ERR_INVALID;
        continue;
      }
      uint32_t d = 0;
      g_.degree(&r->param, 1, &d, 0);
      r->out_u32.resize(d ? d : 1);
      g_.neighbors(r->param, r->out_u32.data(), d, 0);
      r->out_u32.resize(d);
      r->out_count = d;
      calls_ += 2;
    }
    if (deg.empty()) return;
    std::vector<uint32_t> all;  // one lookup launch for every degree request
    for (Request *r : deg) all.insert(all.end(), r->a.begin(), r->a.end());
    std::vector<uint32_t> out(all.size());
    bool ok = true;
    for (uint32_t v : all) ok &= v < n;
    if (ok && !all.empty()) {
      g_.degree(all.data(), all.size(), out.data(), 0);
      calls_++;
    }
    size_t o = 0;
    for (Request *r : deg) {
      if (!ok) r->status = TRC_ERR_INVALID;
      else r->out_u32.assign(out.begin() + o, out.begin() + o + r->a.size());
      o += r->a.size();
      r->out_count = r->a.size();
    }
  }

  // smallest BFS group run as one multi-source launch: up to three
  // single-source BFS (direction-optimising, compacted candidates) beat a
  // multi-source launch on RMAT scale 25 (3 sources: 27-30 ms one by one vs
  // 34-42 ms together)
  static constexpr size_t kMinGroup = 4;

  // BFS grouping by measured cost.  A multi-source launch costs about the
  // same whatever its number of sources (its dense levels read every list
  // once for all of them), so the model is: one single-source BFS takes
  // bfs1_ms_, one multi-source launch msb_ms_ (host times, exponentially
  // weighted averages).  k requests run as one launch only when it is
  // estimated at most 3/4 of k single runs, because single runs complete
  // one by one (each request as soon as its own traversal ends) while a
  // group completes all its requests at its end.  Until a launch has been
  // timed its cost is taken as kMsbPrior single runs, so groups are first
  // tried only when the queue of BFS requests is long; until a single run
  // has been timed, groups are not formed.
  static constexpr double kMsbPrior = 24.0;
  double bfs1_ms_ = 0;
  double msb_ms_ = 0;
  static void ewma(double &avg, double x) { avg = avg > 0 ? 0.75 * avg + 0.25 * x : x; }
  bool group_pays(size_t k) const {
    if (k < kMinGroup || bfs1_ms_ <= 0) return false;
    const double launch = msb_ms_ > 0 ? msb_ms_ : kMsbPrior * bfs1_ms_;
    return launch <= 0.75 * (double)k * bfs1_ms_;
  }

  void run_bfs(std::vector<Request *> &bfs) {
    const uint32_t n = g_.n;
    const bool full = cfg_.result_mode == TRC_RESULT_FULL;
    for (size_t i = 0; i < bfs.size();) {
      size_t k = cfg_.mode == TRC_SERVE_FIFO ? 1 : std::min<size_t>(cfg_.max_bfs_group, bfs.size() - i);
      std::vector<Request *> grp(bfs.begin() + i, bfs.begin() + i + k);
      std::vector<uint32_t> src(k);
      bool bad = false;
      for (size_t j = 0; j < k; j++) {
        src[j] = grp[j]->param;
        bad |= src[j] >= n;
      }
      if (bad) {  // the group's valid sources run one by one
        for (Request *r : grp) {
          if (r->param >= n) {
            r->status = TRC_ERR_INVALID;
          } else {
            bfs_one(r, full);
            round_singles_++;
          }
        }
      } else if (cfg_.mode == TRC_SERVE_FIFO || !group_pays(k)) {
        // one by one, each request completing when its traversal ends
        for (Request *r : grp) {
          const double t0 = now_ms();
          bfs_one(r, full);
          round_singles_++;
          ewma(bfs1_ms_, now_ms() - t0);
          std::vector<Request *> one{r};
          finish(one);
        }
      } else {
        const double t0 = now_ms();
        if (full) {
          std::vector<uint32_t> lv((uint64_t)k * n);
          g_.msbfs(src.data(), (uint32_t)k, lv.data(), 0);
          for (size_t j = 0; j < k; j++) {
            const uint32_t *row = lv.data() + (uint64_t)j * n;
            grp[j]->out_u32.assign(row, row + n);
            grp[j]->out_count = n;
          }
        } else {
          std::vector<uint64_t> reached(k);
          std::vector<uint32_t> ecc(k);
          g_.msbfs_summary(src.data(), (uint32_t)k, reached.data(), ecc.data());
          for (size_t j = 0; j < k; j++) {
            grp[j]->out_u32 = {(uint32_t)reached[j], ecc[j]};
            grp[j]->out_count = reached[j];
          }
        }
        calls_++;
        round_groups_++;
        ewma(msb_ms_, now_ms() - t0);
      }
      finish(grp);
      i += k;
    }
  }

  // PageRank groups (one computation per distinct iteration count).  In
  // summary mode they run on the second stream and the call returns true;
  // end_pagerank collects them.  Full results are copied synchronously.
  bool start_pagerank(std::vector<Request *> &pr) {
    pr_groups_.clear();
    if (pr.empty()) return false;
    const uint32_t n = g_.n;
    std::sort(pr.begin(), pr.end(), [](Request *x, Request *y) { return x->param < y->param; });
    for (size_t i = 0; i < pr.size();) {
      size_t j = i;
      while (j < pr.size() && pr[j]->param == pr[i]->param && (cfg_.mode != TRC_SERVE_FIFO || j == i))
        j++;
      pr_groups_.push_back({i, j});
      i = j;
    }
    const bool full = cfg_.result_mode == TRC_RESULT_FULL;
    if (full || !s2_) {
      for (auto &gr : pr_groups_) {
        std::vector<double> ranks(full ? n : 0);
        double sum = 0, mx = 0;
        if (full) g_.pagerank(pr[gr.first]->param, 0.0, ranks.data(), 0);
        else pagerank_summary(pr[gr.first]->param, &sum, &mx);
        calls_++;
        for (size_t t = gr.first; t < gr.second; t++) {
          pr[t]->out_f64 = full ? ranks : std::vector<double>{sum, mx};
          pr[t]->out_count = n;
        }
      }
      return false;
    }
    // async: class lists current, buffers sized, then everything on s2_
    g_.ensure_lists();
    const unsigned nb = reduce_grid();
    double *p0 = pr0_.ensure(n), *p1 = pr1_.ensure(n), *x = ranks_.ensure(n);
    double *part = pr_part_.ensure(2 * (uint64_t)nb * pr_groups_.size());
    if (pin_cap_ < 2 * nb * pr_groups_.size()) {
      if (pin_) cudaFreeHost(pin_);
      pin_cap_ = 2 * nb * (unsigned)pr_groups_.size();
      TRC_CUDA(cudaMallocHost(&pin_, pin_cap_ * sizeof(double)));
    }
    g_.sync();  // allocations and lists complete before s2_ reads them
    for (size_t gi = 0; gi < pr_groups_.size(); gi++) {
      const uint32_t iters = pr[pr_groups_[gi].first]->param;
      double *out = part + 2 * nb * gi;
      if (iters == 0) {
        TRC_LAUNCH(g_.prof, s2_, "srv_pr_uniform", ceil_div(n, 256), 256, 0, k_fill_f64, x, n,
                   1.0 / (double)n);
      } else {
        g_.pagerank_launch(iters, 0.0, p0, p1, x, s2_);
      }
      TRC_LAUNCH(g_.prof, s2_, "srv_pr_summary", nb, 256, 0, k_rank_summary, x, n, out);
      TRC_CUDA(cudaMemcpyAsync(pin_ + 2 * nb * gi, out, 16 * nb, cudaMemcpyDeviceToHost, s2_));
      calls_++;
    }
    return true;
  }

  void end_pagerank(std::vector<Request *> &pr) {
    TRC_CUDA(cudaStreamSynchronize(s2_));
    const unsigned nb = reduce_grid();
    for (size_t gi = 0; gi < pr_groups_.size(); gi++) {
      double s = 0, m = 0;
      const double *h = pin_ + 2 * nb * gi;
      for (unsigned b = 0; b < nb; b++) {
        s += h[2 * b];
        m = std::max(m, h[2 * b + 1]);
      }
      for (size_t t = pr_groups_[gi].first; t < pr_groups_[gi].second; t++) {
        pr[t]->out_f64 = {s, m};
        pr[t]->out_count = g_.n;
      }
    }
  }

  void bfs_one(Request *r, bool full) {
    const uint32_t n = g_.n;
    if (full) {
      r->out_u32.resize(n);
      std::vector<int32_t> par(n);
      g_.bfs(r->param, par.data(), r->out_u32.data(), 0);
      r->out_count = n;
    } else {
      uint64_t reached = 0;
      uint32_t depth = 0;
      bfs_summary(r->param, &reached, &depth);
      r->out_u32 = {(uint32_t)reached, depth};
      r->out_count = reached;
    }
    calls_++;
  }

  void apply_one(Request *r) {
    uint32_t flags = (cfg_.symmetrize ? TRC_SYMMETRIZE : 0) | TRC_DROP_SELF_LOOPS;
    if (!fits(r->a.size() * (cfg_.symmetrize ? 2 : 1)))
      throw_error(TRC_ERR_NOMEM, "update exceeds the HBM budget");
    r->out_count = r->kind == TRC_REQ_INSERT
                       ? g_.apply_batch(r->a.data(), r->b.data(), r->a.size(), flags, true)
                       : g_.apply_batch(r->a.data(), r->b.data(), r->a.size(), flags, false);
    calls_++;
    r->version = ++version_;
  }

  // The round's updates as one net change (last request touching an edge
  // decides), applied as one delete batch then one insert batch.
  void apply_net(std::vector<Request *> &u) {
    const uint32_t vb = g_.vbits();
    // key = (src, dst, arrival rank, op), the tag directly below the edge so
    // that the sorted bits are contiguous: ceil((2 vb + tagbits) / 8) <= 8
    // radix digits.  If the tag does not fit, apply the updates one by one.
    uint32_t tagbits = 1;  // bits of (rank << 1 | op)
    while ((1ull << tagbits) < ((uint64_t)u.size() << 1)) tagbits++;
    if (2 * vb + tagbits > 64) {
      for (Request *r : u) apply_one(r);
      return;
    }
    bind_bufs();
    g_.phase(nullptr);
    const int sym = cfg_.symmetrize ? 1 : 0;
    uint64_t total = 0;
    for (Request *r : u) total += r->a.size() * (sym ? 2 : 1);
    uint64_t *K = keys_[0].ensure(total + 1), *K2 = keys_[1].ensure(total + 1);
    cudaStream_t s = g_.stream;
    // the round's pairs, concatenated, and per request its offset and op
    const uint32_t R = (uint32_t)u.size();
    uint64_t np = 0;
    for (Request *r : u) np += r->a.size();
    std::vector<uint32_t> hs(np), hd(np), hop(R);
    std::vector<uint64_t> hoff(R);
    uint64_t off = 0;
    for (uint32_t i = 0; i < R; i++) {
      Request *r = u[i];
      hoff[i] = off;
      hop[i] = r->kind == TRC_REQ_INSERT ? 1u : 0u;
      std::copy(r->a.begin(), r->a.end(), hs.begin() + off);
      std::copy(r->b.begin(), r->b.end(), hd.begin() + off);
      off += r->a.size();
    }
    g_.phase("srv_concat");
    uint32_t *ps = up_s_.ensure(np), *pd = up_d_.ensure(np), *dop = rop_.ensure(R);
    uint64_t *doff = roff_.ensure(R);
    TRC_CUDA(cudaMemcpyAsync(ps, hs.data(), np * 4, cudaMemcpyHostToDevice, s));
    TRC_CUDA(cudaMemcpyAsync(pd, hd.data(), np * 4, cudaMemcpyHostToDevice, s));
    TRC_CUDA(cudaMemcpyAsync(dop, hop.data(), R * 4, cudaMemcpyHostToDevice, s));
    TRC_CUDA(cudaMemcpyAsync(doff, hoff.data(), R * 8, cudaMemcpyHostToDevice, s));
    uint32_t *err = g_.err.get();
    TRC_CUDA(cudaMemsetAsync(err, 0, 4, s));
    if (np)
      TRC_LAUNCH(g_.prof, s, "srv_tag_round", ceil_div(np, 256), 256, 0, k_tag_round, ps, pd, np,
                 doff, dop, R, g_.n, sym, vb, tagbits, K, err);
    uint32_t herr = 0;
    TRC_CUDA(cudaMemcpyAsync(&herr, err, 4, cudaMemcpyDeviceToHost, s));
    TRC_CUDA(cudaStreamSynchronize(s));
    if (herr) throw_error(TRC_ERR_INVALID, "vertex id out of range in an update");
    g_.phase("srv_tag");
    // sort by (edge, arrival rank): the 2 vb + tagbits low bits
    int shifts[16];
    int ns = 0;
    for (uint32_t sh = 0; sh < 2 * vb + tagbits; sh += 8) shifts[ns++] = (int)sh;
    uint64_t *t = g_.s_tmp.ensure(radix_tmp_elems(total) + 2 * select_tmp_elems(total) + 8);
    uint64_t *sorted = radix_sort_u64_shifts(K, K2, total, shifts, ns, t, s, g_.prof, err);
    uint64_t *cnt = g_.s_cnt.get() + 30;
    uint32_t *ds = del_s_.ensure(total), *dd = del_d_.ensure(total);
    uint32_t *is = ins_s_.ensure(total), *id = ins_d_.ensure(total);
    select_if(LastOpPred{sorted, total, tagbits, 0}, KeySrc{sorted, tagbits, vb}, total, ds, cnt, t,
              s, g_.prof, "srv_net_del");
    select_if(LastOpPred{sorted, total, tagbits, 0}, KeyDst{sorted, tagbits, vb}, total, dd, cnt, t,
              s, g_.prof, "srv_net_del");
    uint64_t nd = g_.read_u64(cnt);
    select_if(LastOpPred{sorted, total, tagbits, 1}, KeySrc{sorted, tagbits, vb}, total, is, cnt, t,
              s, g_.prof, "srv_net_ins");
    select_if(LastOpPred{sorted, total, tagbits, 1}, KeyDst{sorted, tagbits, vb}, total, id, cnt, t,
              s, g_.prof, "srv_net_ins");
    uint64_t ni = g_.read_u64(cnt);
    uint32_t herr2 = 0;
    TRC_CUDA(cudaMemcpyAsync(&herr2, err, 4, cudaMemcpyDeviceToHost, s));
    TRC_CUDA(cudaStreamSynchronize(s));
    if (herr2 & ERR_TIMEOUT) throw_error(TRC_ERR_TIMEOUT, "radix sort look-back wait gave up");
    g_.phase("srv_net");
    uint64_t removed = nd ? g_.apply_batch(ds, dd, nd, TRC_DEVICE_PTR, false) : 0;
    uint64_t added = ni ? g_.apply_batch(is, id, ni, TRC_DEVICE_PTR, true) : 0;
    calls_ += 2;
    ++version_;
    for (Request *r : u) {
      r->version = version_;
      r->out_count = r->kind == TRC_REQ_INSERT ? added : removed;
    }
  }
};

}  // namespace trc

struct trc_server {
  trc::Server *s;
};

extern "C" const char *trc_last_error(void);
extern "C" trc_status trc_internal_set_error(trc_status st, const char *msg);

namespace {
template <typename F>
trc_status sguard(F &&f) {
  try {
    f();
    return TRC_OK;
  } catch (const trc::Error &e) {
    return trc_internal_set_error(e.status, e.msg.c_str());
  } catch (const std::exception &e) {
    return trc_internal_set_error(TRC_ERR_STATE, e.what());
  }
}
trc::Server &S(trc_server *s) {
  if (!s || !s->s) trc::throw_error(TRC_ERR_INVALID, "null server handle");
  return *s->s;
}
}  // namespace

trc::Graph &trc_internal_graph(trc_graph *g);

extern "C" {

void trc_server_config_default(trc_server_config *c) {
  if (!c) return;
  c->mode = TRC_SERVE_BATCHED;
  c->result_mode = TRC_RESULT_FULL;
  c->symmetrize = 1;
  c->max_bfs_group = 64;
  c->max_round_edges = 1ull << 24;
}

trc_status trc_server_create(trc_graph *g, const trc_server_config *cfg, trc_server **out) {
  return sguard([&] {
    if (!out) trc::throw_error(TRC_ERR_INVALID, "null output");
    trc_server_config c;
    trc_server_config_default(&c);
    if (cfg) c = *cfg;
    trc::Graph &gr = trc_internal_graph(g);
    *out = new trc_server{new trc::Server(gr, c)};
  });
}

trc_status trc_server_destroy(trc_server *s) {
  return sguard([&] {
    if (!s) return;
    delete s->s;
    delete s;
  });
}

trc_status trc_server_submit(trc_server *s, trc_request_kind kind, const uint32_t *a,
                             const uint32_t *b, uint64_t k, uint32_t param, uint64_t *id) {
  return sguard([&] {
    if ((int)kind < 0 || kind > TRC_REQ_PAGERANK) trc::throw_error(TRC_ERR_INVALID, "bad kind");
    if ((kind == TRC_REQ_INSERT || kind == TRC_REQ_DELETE) && k && (!a || !b))
      trc::throw_error(TRC_ERR_INVALID, "null edge array");
    if (kind == TRC_REQ_DEGREE && k && !a) trc::throw_error(TRC_ERR_INVALID, "null vertex array");
    uint64_t r = S(s).submit(kind, a, (kind == TRC_REQ_DEGREE) ? nullptr : b, k, param);
    if (id) *id = r;
  });
}

trc_status trc_server_wait(trc_server *s, uint64_t id, int64_t timeout_ms) {
  trc_status st = TRC_OK;
  trc_status g = sguard([&] { st = S(s).wait(id, timeout_ms); });
  if (g != TRC_OK) return g;
  if (st != TRC_OK) return trc_internal_set_error(st, "request not finished within the timeout");
  return TRC_OK;
}

trc_status trc_server_result(trc_server *s, uint64_t id, void *out, uint64_t cap,
                             uint64_t *bytes, double *latency_ms, uint64_t *version,
                             trc_status *status) {
  return sguard([&] { S(s).result(id, out, cap, bytes, latency_ms, version, status); });
}

trc_status trc_server_release(trc_server *s, uint64_t id) {
  return sguard([&] { S(s).release(id); });
}

trc_status trc_server_get_stats(trc_server *s, int kind, trc_server_stats *out) {
  return sguard([&] {
    if (!out) trc::throw_error(TRC_ERR_INVALID, "null output");
    S(s).stats(kind, out);
  });
}

trc_status trc_server_reset_stats(trc_server *s) {
  return sguard([&] { S(s).reset_stats(); });
}

trc_status trc_server_hold(trc_server *s, int hold) {
  return sguard([&] { S(s).hold(hold != 0); });
}

trc_status trc_server_rounds(trc_server *s, trc_round_record *out, uint64_t cap, uint64_t *count) {
  return sguard([&] {
    if (!out && cap) trc::throw_error(TRC_ERR_INVALID, "null output");
    const uint64_t c = S(s).rounds_trace(out, cap);
    if (count) *count = c;
  });
}

}  // extern "C"
