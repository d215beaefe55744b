// common.cu -- error plumbing, budgeted device allocation and the CUDA-event
// profiler shared by every entry point.
#include <atomic>
#include <cstdio>
#include <string>

#include "trc_common.cuh"

namespace trc {

void throw_error(trc_status s, const std::string &msg) { throw Error{s, msg}; }

void cuda_check(cudaError_t e, const char *what, const char *file, int line) {
  if (e == cudaSuccess) return;
  char buf[512];
  snprintf(buf, sizeof(buf), "%s failed: %s (%s:%d)", what, cudaGetErrorString(e), file, line);
  if (e == cudaErrorMemoryAllocation) throw Error{TRC_ERR_NOMEM, buf};
  throw Error{TRC_ERR_CUDA, buf};
}

void Budget::open_pool(int device) {
  cudaMemPoolProps props = {};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = device;
  TRC_CUDA(cudaMemPoolCreate(&pool, &props));
  uint64_t keep = ~0ull;  // never release at synchronisation points
  TRC_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
}

void Budget::trim() {
  if (pool) cudaMemPoolTrimTo(pool, 0);
}

// Outstanding frees complete before the pool's memory is returned (the
// runtime defers the destruction until then).
Budget::~Budget() {
  if (pool) cudaMemPoolDestroy(pool);
}

void *Budget::alloc(uint64_t bytes) {
  if (bytes == 0) bytes = 16;
  if (limit && used + bytes > limit) {
    char buf[256];
    snprintf(buf, sizeof(buf), "HBM budget exhausted: %llu bytes held, %llu requested, limit %llu",
             (unsigned long long)used, (unsigned long long)bytes, (unsigned long long)limit);
    throw Error{TRC_ERR_NOMEM, buf};
  }
  void *p = nullptr;
  cudaError_t e = pool ? cudaMallocFromPoolAsync(&p, bytes, pool, stream) : cudaMalloc(&p, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    char buf[256];
    snprintf(buf, sizeof(buf), "cudaMalloc(%llu) failed: %s", (unsigned long long)bytes,
             cudaGetErrorString(e));
    throw Error{TRC_ERR_NOMEM, buf};
  }
  used += bytes;
  return p;
}

void Budget::release(void *p, uint64_t bytes) {
  if (!p) return;
  if (pool) cudaFreeAsync(p, stream);
  else cudaFree(p);
  if (bytes == 0) bytes = 16;
  used -= bytes;
}

cudaEvent_t Profiler::get_event() {
  if (!pool_.empty()) {
    cudaEvent_t e = pool_.back();
    pool_.pop_back();
    return e;
  }
  cudaEvent_t e;
  TRC_CUDA(cudaEventCreate(&e));
  return e;
}

int Profiler::begin(const char *name, cudaStream_t s) {
  launches++;
  if (!on) return -1;
  Rec r;
  r.a = get_event();
  r.b = get_event();
  r.name = name;
  TRC_CUDA(cudaEventRecord(r.a, s));
  pending.push_back(r);
  return (int)pending.size() - 1;
}

void Profiler::end(int idx, cudaStream_t s) {
  if (idx < 0) return;
  TRC_CUDA(cudaEventRecord(pending[idx].b, s));
  if (pending.size() > 4096) resolve();
}

void Profiler::resolve() {
  for (auto &r : pending) {
    TRC_CUDA(cudaEventSynchronize(r.b));
    float ms = 0;
    TRC_CUDA(cudaEventElapsedTime(&ms, r.a, r.b));
    auto &t = totals[r.name];
    t.first += ms;
    t.second += 1;
    pool_.push_back(r.a);
    pool_.push_back(r.b);
  }
  pending.clear();
}

void Profiler::reset() {
  resolve();
  totals.clear();
}

Profiler::~Profiler() {
  for (auto &r : pending) {
    cudaEventDestroy(r.a);
    cudaEventDestroy(r.b);
  }
  for (auto e : pool_) cudaEventDestroy(e);
}

int num_sms() {
  // per device (the current one), cached; a race between threads only
  // stores the same value twice
  static std::atomic<int> cache[64];
  int dev = 0;
  cudaGetDevice(&dev);
  std::atomic<int> *slot = dev >= 0 && dev < 64 ? &cache[dev] : nullptr;
  int sms = slot ? slot->load(std::memory_order_relaxed) : 0;
  if (!sms) {
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (sms <= 0) sms = 148;
    if (slot) slot->store(sms, std::memory_order_relaxed);
  }
  return sms;
}

}  // namespace trc
