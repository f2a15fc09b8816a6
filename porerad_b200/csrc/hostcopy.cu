// Device -> host copies into pageable memory at the speed of the bus.
//
// A plain cudaMemcpy into pageable memory goes through the driver's own small pinned
// buffers and one host thread: on this machine class a few GB/s, while a pinned
// destination takes the PCIe link's full rate.  The count tables handed back by
// first_hit_counts are gigabytes of (origin, receiver, count) per call, so copies larger
// than kDirectMax bytes into pageable memory run as a pipeline instead:
//
//   * two pinned staging buffers of kChunk bytes per device (allocated once, kept);
//   * the DMA of chunk k + 1 into one buffer overlaps host threads copying chunk k out of the
//     other into the destination (the threads also take the destination's first-touch page
//     faults in parallel);
//   * a pool of host threads (one per hardware thread, at most 16), started on first use.
//
// Device memory, pinned or managed destinations and small copies take cudaMemcpyAsync.
#include <condition_variable>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

#include "pr_internal.cuh"

namespace pr {
namespace {

constexpr size_t kChunk = (size_t)32 << 20;      // bytes per staging buffer
constexpr size_t kDirectMax = (size_t)16 << 20;  // copies up to this size go straight through

// A fixed pool of worker threads running batches of range copies.
class CopyPool {
 public:
  CopyPool() {
    unsigned n = std::thread::hardware_concurrency();
    n_ = n == 0 ? 4 : (n > 16 ? 16 : n);
    for (unsigned t = 1; t < n_; ++t) workers_.emplace_back([this, t] { run(t); });
  }
  ~CopyPool() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      quit_ = true;
    }
    cv_.notify_all();
    for (auto& w : workers_) w.join();
  }
  // memcpy(dst, src, bytes) split over all threads, the caller's thread included; returns when done.
  // Calls from several host threads take turns.
  void copy(char* dst, const char* src, size_t bytes) {
    std::lock_guard<std::mutex> turn(call_mu_);
    std::unique_lock<std::mutex> lk(mu_);
    dst_ = dst;
    src_ = src;
    bytes_ = bytes;
    pending_ = n_ - 1;
    ++generation_;
    lk.unlock();
    cv_.notify_all();
    part(0);
    lk.lock();
    done_cv_.wait(lk, [this] { return pending_ == 0; });
  }

 private:
  void part(unsigned t) {
    // slices aligned to 4 KiB pages so that threads fault in disjoint pages
    const size_t page = 4096;
    const size_t per = ((bytes_ + n_ - 1) / n_ + page - 1) / page * page;
    const size_t b = (size_t)t * per;
    if (b < bytes_) memcpy(dst_ + b, src_ + b, (bytes_ - b) < per ? (bytes_ - b) : per);
  }
  void run(unsigned t) {
    unsigned long long seen = 0;
    for (;;) {
      std::unique_lock<std::mutex> lk(mu_);
      cv_.wait(lk, [&] { return quit_ || generation_ != seen; });
      if (quit_) return;
      seen = generation_;
      lk.unlock();
      part(t);
      lk.lock();
      if (--pending_ == 0) done_cv_.notify_one();
    }
  }

  unsigned n_ = 1;
  std::vector<std::thread> workers_;
  std::mutex call_mu_, mu_;
  std::condition_variable cv_, done_cv_;
  char* dst_ = nullptr;
  const char* src_ = nullptr;
  size_t bytes_ = 0;
  unsigned pending_ = 0;
  unsigned long long generation_ = 0;
  bool quit_ = false;
};

struct Staging {
  char* buf[2] = {nullptr, nullptr};
  cudaEvent_t ready[2] = {nullptr, nullptr};
  std::mutex mu;  // one pipeline at a time per device
};

std::mutex g_mu;
Staging* g_staging[64] = {nullptr};
CopyPool* g_pool = nullptr;

int staging_for(int dev, Staging** out) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (dev < 0 || dev >= 64) {
    set_error("device %d outside the supported range", dev);
    return PR_ERR_LIMIT;
  }
  if (!g_pool) g_pool = new CopyPool();
  if (!g_staging[dev]) {
    Staging* st = new Staging();
    for (int b = 0; b < 2; ++b) {
      if (cudaHostAlloc((void**)&st->buf[b], kChunk, cudaHostAllocDefault) != cudaSuccess ||
          cudaEventCreateWithFlags(&st->ready[b], cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        set_error("pinned staging buffers for host copies could not be allocated");
        return PR_ERR_OOM;
      }
    }
    g_staging[dev] = st;
  }
  *out = g_staging[dev];
  return PR_OK;
}

bool pageable(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return true;
  }
  return a.type == cudaMemoryTypeUnregistered;
}

}  // namespace

int copy_to_host(void* dst, const void* src, size_t bytes, cudaStream_t s) {
  if (bytes == 0) return PR_OK;
  if (bytes <= kDirectMax || !pageable(dst)) {
    PR_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, s));
    return PR_OK;
  }
  int dev = 0;
  PR_CUDA(cudaGetDevice(&dev));
  Staging* st = nullptr;
  PR_TRY(staging_for(dev, &st));
  std::lock_guard<std::mutex> lk(st->mu);
  const char* s8 = static_cast<const char*>(src);
  char* d8 = static_cast<char*>(dst);
  const size_t n = (bytes + kChunk - 1) / kChunk;
  auto issue = [&](size_t k) -> int {
    const size_t off = k * kChunk, len = (bytes - off) < kChunk ? (bytes - off) : kChunk;
    PR_CUDA(cudaMemcpyAsync(st->buf[k & 1], s8 + off, len, cudaMemcpyDeviceToHost, s));
    PR_CUDA(cudaEventRecord(st->ready[k & 1], s));
    return PR_OK;
  };
  PR_TRY(issue(0));
  for (size_t k = 0; k < n; ++k) {
    // the buffer of chunk k + 1 was emptied by the host copy of chunk k - 1 (finished below)
    if (k + 1 < n) PR_TRY(issue(k + 1));
    PR_CUDA(cudaEventSynchronize(st->ready[k & 1]));
    const size_t off = k * kChunk, len = (bytes - off) < kChunk ? (bytes - off) : kChunk;
    g_pool->copy(d8 + off, st->buf[k & 1], len);
  }
  return PR_OK;
}

}  // namespace pr
