// io.cu -- graph files.  The reference's input format is the AdjacencyGraph
// text file (include/io_util.h:112-145): the word "AdjacencyGraph", n, m,
// n offsets, m targets, separated by white space; vertex i's edges are
// targets [offsets[i], offsets[i+1]) (offsets[n] taken as m).  Here the file
// is parsed on the GPU: word starts are found by a compaction over the bytes,
// each word is converted by its own thread, the edge sources are recovered
// by a binary search of the offsets per edge, and the edges go through the
// batch insert pipeline.  The writer formats on the GPU too (digit counts,
// exclusive scan, one thread per number).  A binary CSR file
// (magic "TRCCSR01", n, m as u64, offsets[n+1] u64, targets[m] u32) is the
// compact exchange format.
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "graph.cuh"

struct trc_graph;
trc::Graph &trc_internal_graph(trc_graph *g);
extern "C" trc_status trc_internal_set_error(trc_status st, const char *msg);

namespace trc {
namespace {

constexpr uint32_t IO_T = 256;
constexpr char CSR_MAGIC[8] = {'T', 'R', 'C', 'C', 'S', 'R', '0', '1'};
constexpr uint32_t ERR_IO_CHAR = 1u, ERR_IO_RANGE = 2u, ERR_IO_OFFSETS = 4u;

// white space as the reference's reader splits words (include/io_util.h:
// 27-36: space, tab, newline, carriage return, NUL)
__device__ __forceinline__ bool adj_space(uint8_t c) {
  return c == ' ' || c == '\n' || c == '\r' || c == '\t' || c == 0;
}

struct WordStartPred {
  const uint8_t *b;
  __device__ bool operator()(uint64_t i) const {
    return !adj_space(b[i]) && (i == 0 || adj_space(b[i - 1]));
  }
};

struct IndexU64 {
  __device__ uint64_t operator()(uint64_t i) const { return i; }
};

// vals[w - 1] = unsigned decimal value of word w (w >= 1; word 0 is the
// header word)
__global__ void k_adj_parse(const uint8_t *b, uint64_t len, const uint64_t *pos, uint64_t nw,
                            uint64_t *vals, uint32_t *err) {
  const uint64_t w = (uint64_t)blockIdx.x * IO_T + threadIdx.x + 1;
  if (w >= nw) return;
  uint64_t p = pos[w], v = 0;
  uint32_t e = 0;
  for (; p < len; p++) {
    const uint8_t c = b[p];
    if (adj_space(c)) break;
    if (c < '0' || c > '9') {
      e |= ERR_IO_CHAR;
      break;
    }
    const uint64_t dg = c - '0';
    if (v > (~0ull - dg) / 10) {
      e |= ERR_IO_RANGE;
      break;
    }
    v = v * 10 + dg;
  }
  vals[w - 1] = v;
  if (e) atomicOr(err, e);
}

// offsets: off[0] == 0, non-decreasing, at most m (the last vertex's list
// ends at m)
__global__ void k_check_offsets(const uint64_t *off, uint64_t n, uint64_t m, uint32_t *err) {
  const uint64_t i = (uint64_t)blockIdx.x * IO_T + threadIdx.x;
  if (i >= n) return;
  const uint64_t o = off[i];
  bool bad = o > m || (i == 0 && o != 0) || (i + 1 < n && off[i + 1] < o);
  if (bad) atomicOr(err, ERR_IO_OFFSETS);
}

// edge j: source = the vertex i with off[i] <= j < off[i + 1], target
// tgt[j] (64-bit words from the text parser, 32-bit from a CSR file)
template <typename TT>
__global__ void k_expand_edges(const uint64_t *off, uint64_t n, const TT *tgt, uint64_t m,
                               uint32_t *src, uint32_t *dst, uint32_t *err) {
  const uint64_t j = (uint64_t)blockIdx.x * IO_T + threadIdx.x;
  if (j >= m) return;
  uint64_t lo = 0, hi = n;  // last i with off[i] <= j
  while (hi - lo > 1) {
    const uint64_t mid = (lo + hi) >> 1;
    if (off[mid] <= j) lo = mid;
    else hi = mid;
  }
  const uint64_t t = (uint64_t)tgt[j];
  if (t > 0xFFFFFFFFull) atomicOr(err, ERR_IO_RANGE);
  src[j] = (uint32_t)lo;
  dst[j] = (uint32_t)t;
}

__device__ __forceinline__ uint32_t dec_digits(uint64_t v) {
  uint32_t d = 1;
  while (v >= 10) {
    v /= 10;
    d++;
  }
  return d;
}

// the numbers of an AdjacencyGraph file after its header word: n, m,
// offsets[0..n), targets[0..m)
struct AdjValue {
  uint64_t n, m;
  const uint64_t *off;
  const uint32_t *tgt;
  __device__ uint64_t operator()(uint64_t k) const {
    if (k == 0) return n;
    if (k == 1) return m;
    if (k < 2 + n) return off[k - 2];
    return tgt[k - 2 - n];
  }
};

struct AdjLen {
  AdjValue v;
  __device__ uint64_t operator()(uint64_t k) const { return dec_digits(v(k)) + 1; }
};

__global__ void k_adj_format(AdjValue v, uint64_t count, const uint64_t *at, uint8_t *out) {
  const uint64_t k = (uint64_t)blockIdx.x * IO_T + threadIdx.x;
  if (k >= count) return;
  uint64_t x = v(k);
  const uint32_t d = dec_digits(x);
  uint8_t *p = out + at[k];
  p[d] = '\n';
  for (int i = (int)d - 1; i >= 0; i--) {
    p[i] = (uint8_t)('0' + x % 10);
    x /= 10;
  }
}

struct FileCloser {
  FILE *f;
  ~FileCloser() {
    if (f) fclose(f);
  }
};

std::vector<uint8_t> read_file(const char *path) {
  if (!path) throw_error(TRC_ERR_INVALID, "null path");
  FileCloser fc{fopen(path, "rb")};
  if (!fc.f) throw_error(TRC_ERR_IO, std::string("cannot open ") + path);
  if (fseek(fc.f, 0, SEEK_END) != 0) throw_error(TRC_ERR_IO, "cannot seek");
  const long len = ftell(fc.f);
  if (len < 0) throw_error(TRC_ERR_IO, "cannot size file");
  rewind(fc.f);
  std::vector<uint8_t> buf((size_t)len);
  if (len && fread(buf.data(), 1, (size_t)len, fc.f) != (size_t)len)
    throw_error(TRC_ERR_IO, "short read");
  return buf;
}

void write_file(const char *path, const std::vector<std::pair<const void *, uint64_t>> &parts) {
  if (!path) throw_error(TRC_ERR_INVALID, "null path");
  FileCloser fc{fopen(path, "wb")};
  if (!fc.f) throw_error(TRC_ERR_IO, std::string("cannot create ") + path);
  for (auto &p : parts)
    if (p.second && fwrite(p.first, 1, p.second, fc.f) != p.second)
      throw_error(TRC_ERR_IO, "short write");
  if (fclose(fc.f) != 0) {
    fc.f = nullptr;
    throw_error(TRC_ERR_IO, "close failed");
  }
  fc.f = nullptr;
}

// The first three words on the host: the header word, n and m.
void adj_header(const std::vector<uint8_t> &b, uint64_t &n, uint64_t &m) {
  auto sp = [](uint8_t c) { return c == ' ' || c == '\n' || c == '\r' || c == '\t' || c == 0; };
  size_t p = 0;
  std::string w[3];
  for (int i = 0; i < 3; i++) {
    while (p < b.size() && sp(b[p])) p++;
    while (p < b.size() && !sp(b[p]) && w[i].size() < 32) w[i].push_back((char)b[p++]);
  }
  if (w[0] != "AdjacencyGraph")
    throw_error(TRC_ERR_INVALID, "bad input file: missing header AdjacencyGraph");
  for (int i = 1; i < 3; i++) {
    if (w[i].empty() || w[i].size() > 20 || w[i].find_first_not_of("0123456789") != std::string::npos)
      throw_error(TRC_ERR_INVALID, "bad input file: n and m must be decimal integers");
  }
  n = std::stoull(w[1]);
  m = std::stoull(w[2]);
  // range checks before any sum of the two: vertex ids are 32-bit, and a
  // file of b bytes holds fewer than b/2 + 1 numbers
  if (n > 0xFFFFFFFFull) throw_error(TRC_ERR_INVALID, "bad input file: n exceeds 2^32 - 1");
  if (m > b.size() / 2 + 1)
    throw_error(TRC_ERR_INVALID, "bad input file: m exceeds the numbers the file can hold");
}

}  // namespace

// Parses the AdjacencyGraph bytes on the device and inserts the edges.
void Graph::load_adj(const uint8_t *bytes, uint64_t len, uint64_t m_file, uint32_t flags) {
  DBuf<uint8_t> db;
  DBuf<uint64_t> pos, vals, tmpb, cntb;
  DBuf<uint32_t> srcb, dstb;
  db.bind(&budget);
  for (auto *b : {&pos, &vals, &tmpb, &cntb}) b->bind(&budget);
  srcb.bind(&budget);
  dstb.bind(&budget);
  uint8_t *d = db.alloc_exact(len);
  TRC_CUDA(cudaMemcpyAsync(d, bytes, len, cudaMemcpyHostToDevice, stream));
  uint64_t *cnt = cntb.alloc_exact(2);
  // word starts: count per tile, scan, then the exact-size compaction
  const uint64_t tiles = ceil_div(len, PTILE);
  uint64_t *t = tmpb.alloc_exact(select_tmp_elems(len) + 4);
  uint64_t *sums = t, *offs = t + tiles;
  TRC_LAUNCH(prof, stream, "adj_words.count", tiles, PT, 0, k_tile_sum<PredCount<WordStartPred>>,
             PredCount<WordStartPred>{WordStartPred{d}}, len, sums);
  exclusive_scan(LoadU64{sums}, tiles, offs, offs + tiles + 1, stream, prof, "scan_tiles");
  const uint64_t nw = read_u64(offs + tiles);
  const uint64_t n64 = n;
  if (nw != n64 + m_file + 3)
    throw_error(TRC_ERR_INVALID, "bad input file: " + std::to_string(nw - 1) +
                                     " numbers after the header, n + m + 2 = " +
                                     std::to_string(n64 + m_file + 2));
  uint64_t *ps = pos.alloc_exact(nw);
  auto kscatter = k_select_scatter<WordStartPred, IndexU64, uint64_t>;
  TRC_LAUNCH(prof, stream, "adj_words.scatter", tiles, PT, 0, kscatter, WordStartPred{d}, IndexU64{},
             len, offs, ps, cnt);
  uint64_t *v = vals.alloc_exact(nw);
  TRC_CUDA(cudaMemsetAsync(err.get(), 0, 4, stream));
  TRC_LAUNCH(prof, stream, "adj_parse", ceil_div(nw, IO_T), IO_T, 0, k_adj_parse, d, len, ps, nw,
             v, err.get());
  db.reset();
  pos.reset();
  tmpb.reset();
  const uint64_t *off = v + 2, *tg = v + 2 + n64;
  TRC_LAUNCH(prof, stream, "adj_offsets", ceil_div(n64, IO_T), IO_T, 0, k_check_offsets, off, n64,
             m_file, err.get());
  uint32_t *s = srcb.alloc_exact(m_file), *dd = dstb.alloc_exact(m_file);
  TRC_LAUNCH(prof, stream, "adj_expand", ceil_div(m_file, IO_T), IO_T, 0, k_expand_edges<uint64_t>,
             off, n64, tg, m_file, s, dd, err.get());
  uint32_t herr = 0;
  TRC_CUDA(cudaMemcpyAsync(&herr, err.get(), 4, cudaMemcpyDeviceToHost, stream));
  sync();
  if (herr & ERR_IO_CHAR) throw_error(TRC_ERR_INVALID, "bad input file: a word is not a number");
  if (herr & ERR_IO_RANGE) throw_error(TRC_ERR_INVALID, "bad input file: number out of range");
  if (herr & ERR_IO_OFFSETS) throw_error(TRC_ERR_INVALID, "bad input file: offsets not monotone from 0");
  vals.reset();
  if (m_file) apply_batch(s, dd, m_file, flags | TRC_DEVICE_PTR, true);
}

// Inserts the edges of a CSR given in host memory.
void Graph::load_csr(const uint64_t *offsets, const uint32_t *targets, uint64_t m_file,
                     uint32_t flags) {
  DBuf<uint64_t> offb;
  DBuf<uint32_t> tgb, srcb, dstb;
  offb.bind(&budget);
  for (auto *b : {&tgb, &srcb, &dstb}) b->bind(&budget);
  const uint64_t n64 = n;
  if (offsets[n64] != m_file) throw_error(TRC_ERR_INVALID, "bad CSR file: offsets[n] != m");
  uint64_t *off = offb.alloc_exact(n64 + 1);
  uint32_t *tg = tgb.alloc_exact(m_file);
  TRC_CUDA(cudaMemcpyAsync(off, offsets, (n64 + 1) * 8, cudaMemcpyHostToDevice, stream));
  if (m_file) TRC_CUDA(cudaMemcpyAsync(tg, targets, m_file * 4, cudaMemcpyHostToDevice, stream));
  TRC_CUDA(cudaMemsetAsync(err.get(), 0, 4, stream));
  TRC_LAUNCH(prof, stream, "csr_offsets", ceil_div(n64, IO_T), IO_T, 0, k_check_offsets, off, n64,
             m_file, err.get());
  uint32_t *s = srcb.alloc_exact(m_file), *dd = dstb.alloc_exact(m_file);
  TRC_LAUNCH(prof, stream, "csr_expand", ceil_div(m_file, IO_T), IO_T, 0, k_expand_edges<uint32_t>,
             off, n64, tg, m_file, s, dd, err.get());
  uint32_t herr = 0;
  TRC_CUDA(cudaMemcpyAsync(&herr, err.get(), 4, cudaMemcpyDeviceToHost, stream));
  sync();
  if (herr) throw_error(TRC_ERR_INVALID, "bad CSR file: offsets not monotone from 0");
  if (m_file) apply_batch(s, dd, m_file, flags | TRC_DEVICE_PTR, true);
}

// The graph as AdjacencyGraph text, formatted on the device.
std::vector<uint8_t> Graph::format_adj() {
  const uint64_t n64 = n, mm = m;
  DBuf<uint64_t> offb, at, tmpb;
  DBuf<uint32_t> tgb;
  DBuf<uint8_t> outb;
  for (auto *b : {&offb, &at, &tmpb}) b->bind(&budget);
  tgb.bind(&budget);
  outb.bind(&budget);
  uint64_t *off = offb.alloc_exact(n64 + 1);
  uint32_t *tg = tgb.alloc_exact(mm ? mm : 1);
  dump_csr(off, tg, TRC_DEVICE_PTR);
  const uint64_t count = 2 + n64 + mm;
  AdjValue val{n64, mm, off, tg};
  uint64_t *a = at.alloc_exact(count + 1);
  uint64_t *t = tmpb.alloc_exact(scan_tmp_elems(count) + 4);
  exclusive_scan(AdjLen{val}, count, a, t, stream, prof, "adj_len");
  const uint64_t body = read_u64(a + count);
  static const char head[] = "AdjacencyGraph\n";
  const uint64_t hl = sizeof(head) - 1;
  uint8_t *o = outb.alloc_exact(hl + body);
  TRC_CUDA(cudaMemcpyAsync(o, head, hl, cudaMemcpyHostToDevice, stream));
  TRC_LAUNCH(prof, stream, "adj_format", ceil_div(count, IO_T), IO_T, 0, k_adj_format, val, count,
             a, o + hl);
  std::vector<uint8_t> text(hl + body);
  TRC_CUDA(cudaMemcpyAsync(text.data(), o, hl + body, cudaMemcpyDeviceToHost, stream));
  sync();
  return text;
}

}  // namespace trc

namespace {
template <typename F>
trc_status io_guard(F &&f) {
  try {
    f();
    return trc_internal_set_error(TRC_OK, "");
  } catch (const trc::Error &e) {
    return trc_internal_set_error(e.status, e.msg.c_str());
  } catch (const std::bad_alloc &) {
    return trc_internal_set_error(TRC_ERR_NOMEM, "host allocation failed");
  } catch (const std::exception &e) {
    return trc_internal_set_error(TRC_ERR_STATE, e.what());
  }
}

// Creates the graph of n vertices; on a later failure it is destroyed.
struct NewGraph {
  trc_graph *h = nullptr;
  NewGraph(uint64_t n, uint64_t budget, const trc_config *cfg) {
    if (n == 0 || n > 0xFFFFFFFFull)
      trc::throw_error(TRC_ERR_INVALID, "vertex count must be in [1, 2^32)");
    trc_status st = trc_graph_create((uint32_t)n, budget, cfg, &h);
    if (st != TRC_OK) trc::throw_error(st, trc_last_error());
  }
  ~NewGraph() {
    if (h) trc_graph_destroy(h);
  }
  trc_graph *release() {
    trc_graph *x = h;
    h = nullptr;
    return x;
  }
};
}  // namespace

extern "C" {

trc_status trc_graph_load_adj(const char *path, uint64_t hbm_budget_bytes, const trc_config *cfg,
                              uint32_t flags, trc_graph **out) {
  return io_guard([&] {
    if (!out) trc::throw_error(TRC_ERR_INVALID, "null output handle");
    if (flags & TRC_DEVICE_PTR) trc::throw_error(TRC_ERR_INVALID, "TRC_DEVICE_PTR has no meaning here");
    *out = nullptr;
    std::vector<uint8_t> b = trc::read_file(path);
    uint64_t n = 0, m = 0;
    trc::adj_header(b, n, m);
    NewGraph g(n, hbm_budget_bytes, cfg);
    trc_internal_graph(g.h).load_adj(b.data(), b.size(), m, flags);
    *out = g.release();
  });
}

trc_status trc_graph_save_adj(trc_graph *g, const char *path) {
  return io_guard([&] {
    trc::Graph &G = trc_internal_graph(g);
    if (!path) trc::throw_error(TRC_ERR_INVALID, "null path");
    std::vector<uint8_t> text = G.format_adj();
    trc::write_file(path, {{text.data(), text.size()}});
  });
}

trc_status trc_graph_load_csr(const char *path, uint64_t hbm_budget_bytes, const trc_config *cfg,
                              uint32_t flags, trc_graph **out) {
  return io_guard([&] {
    if (!out) trc::throw_error(TRC_ERR_INVALID, "null output handle");
    if (flags & TRC_DEVICE_PTR) trc::throw_error(TRC_ERR_INVALID, "TRC_DEVICE_PTR has no meaning here");
    *out = nullptr;
    std::vector<uint8_t> b = trc::read_file(path);
    if (b.size() < 24 || memcmp(b.data(), trc::CSR_MAGIC, 8) != 0)
      trc::throw_error(TRC_ERR_INVALID, "bad CSR file: missing magic TRCCSR01");
    uint64_t n = 0, m = 0;
    memcpy(&n, b.data() + 8, 8);
    memcpy(&m, b.data() + 16, 8);
    if (n == 0 || n > 0xFFFFFFFFull || m > (b.size() / 4))
      trc::throw_error(TRC_ERR_INVALID, "bad CSR file: sizes");
    const uint64_t need = 24 + (n + 1) * 8 + m * 4;
    if (b.size() != need) trc::throw_error(TRC_ERR_INVALID, "bad CSR file: length does not match n, m");
    std::vector<uint64_t> off(n + 1);
    std::vector<uint32_t> tg(m);
    memcpy(off.data(), b.data() + 24, (n + 1) * 8);
    if (m) memcpy(tg.data(), b.data() + 24 + (n + 1) * 8, m * 4);
    b.clear();
    b.shrink_to_fit();
    NewGraph g(n, hbm_budget_bytes, cfg);
    trc_internal_graph(g.h).load_csr(off.data(), tg.data(), m, flags);
    *out = g.release();
  });
}

trc_status trc_graph_save_csr(trc_graph *g, const char *path) {
  return io_guard([&] {
    trc::Graph &G = trc_internal_graph(g);
    if (!path) trc::throw_error(TRC_ERR_INVALID, "null path");
    const uint64_t n = G.n, m = G.m;
    std::vector<uint64_t> off(n + 1);
    std::vector<uint32_t> tg(m ? m : 1);
    G.dump_csr(off.data(), tg.data(), 0);
    uint64_t hdr[3];
    memcpy(&hdr[0], trc::CSR_MAGIC, 8);
    hdr[1] = n;
    hdr[2] = m;
    trc::write_file(path, {{hdr, 24}, {off.data(), (n + 1) * 8}, {tg.data(), m * 4}});
  });
}

}  // extern "C"
