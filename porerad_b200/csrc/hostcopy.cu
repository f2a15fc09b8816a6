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
  // job(begin, end) over [0, total) split into one slice per thread (slices aligned to `align`
  // items), the caller's thread included; returns when every slice is done.  Calls from several
  // host threads take turns.
  void run(size_t total, size_t align, const std::function<void(size_t, size_t)>& job) {
    std::lock_guard<std::mutex> turn(call_mu_);
    std::unique_lock<std::mutex> lk(mu_);
    job_ = &job;
    total_ = total;
    align_ = align == 0 ? 1 : align;
    pending_ = n_ - 1;
    ++generation_;
    lk.unlock();
    cv_.notify_all();
    part(0);
    lk.lock();
    done_cv_.wait(lk, [this] { return pending_ == 0; });
  }
  // memcpy split over the threads (4 KiB slices, so that threads fault in disjoint pages)
  void copy(char* dst, const char* src, size_t bytes) {
    run(bytes, 4096, [&](size_t b, size_t e) { memcpy(dst + b, src + b, e - b); });
  }

 private:
  void part(unsigned t) {
    const size_t per = ((total_ + n_ - 1) / n_ + align_ - 1) / align_ * align_;
    const size_t b = (size_t)t * per;
    if (b < total_) (*job_)(b, (total_ - b) < per ? total_ : b + per);
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
  const std::function<void(size_t, size_t)>* job_ = nullptr;
  size_t total_ = 0, align_ = 1;
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

// The pipeline: chunks of src (device) go through the staging buffers; for each chunk, on the
// host, sink(staging, first byte of the chunk, its bytes) runs over the host threads.
static int staged(const void* src, size_t bytes, cudaStream_t s,
                  const std::function<void(const char*, size_t, size_t)>& sink) {
  int dev = 0;
  PR_CUDA(cudaGetDevice(&dev));
  Staging* st = nullptr;
  PR_TRY(staging_for(dev, &st));
  std::lock_guard<std::mutex> lk(st->mu);
  const char* s8 = static_cast<const char*>(src);
  const size_t n = (bytes + kChunk - 1) / kChunk;
  auto issue = [&](size_t k) -> int {
    const size_t off = k * kChunk, len = (bytes - off) < kChunk ? (bytes - off) : kChunk;
    PR_CUDA(cudaMemcpyAsync(st->buf[k & 1], s8 + off, len, cudaMemcpyDeviceToHost, s));
    PR_CUDA(cudaEventRecord(st->ready[k & 1], s));
    return PR_OK;
  };
  PR_TRY(issue(0));
  for (size_t k = 0; k < n; ++k) {
    // the buffer of chunk k + 1 was emptied by the host work of chunk k - 1 (finished below)
    if (k + 1 < n) PR_TRY(issue(k + 1));
    PR_CUDA(cudaEventSynchronize(st->ready[k & 1]));
    const size_t off = k * kChunk, len = (bytes - off) < kChunk ? (bytes - off) : kChunk;
    sink(st->buf[k & 1], off, len);
  }
  return PR_OK;
}

int copy_to_host(void* dst, const void* src, size_t bytes, cudaStream_t s) {
  if (bytes == 0) return PR_OK;
  if (bytes <= kDirectMax || !pageable(dst)) {
    PR_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, s));
    return PR_OK;
  }
  char* d8 = static_cast<char*>(dst);
  return staged(src, bytes, s, [&](const char* buf, size_t off, size_t len) { g_pool->copy(d8 + off, buf, len); });
}

int copy_to_host_i64(int64_t* dst, const int32_t* src, int64_t n, cudaStream_t s) {
  if (n <= 0) return PR_OK;
  if ((size_t)n * 4 <= kDirectMax || !pageable(dst)) {
    std::vector<int32_t> h((size_t)n);
    PR_CUDA(cudaMemcpyAsync(h.data(), src, (size_t)n * 4, cudaMemcpyDeviceToHost, s));
    PR_CUDA(cudaStreamSynchronize(s));
    if (pageable(dst)) {
      for (int64_t i = 0; i < n; ++i) dst[i] = h[i];
    } else {
      std::vector<int64_t> w(h.begin(), h.end());
      PR_CUDA(cudaMemcpyAsync(dst, w.data(), (size_t)n * 8, cudaMemcpyDefault, s));
      PR_CUDA(cudaStreamSynchronize(s));
    }
    return PR_OK;
  }
  return staged(src, (size_t)n * 4, s, [&](const char* buf, size_t off, size_t len) {
    const int32_t* in = reinterpret_cast<const int32_t*>(buf);
    int64_t* out = dst + off / 4;
    g_pool->run(len / 4, 512, [&](size_t b, size_t e) {
      for (size_t i = b; i < e; ++i) out[i] = in[i];
    });
  });
}

void fill_rows_host(int32_t* origin, const int64_t* row_ptr, int64_t n_rows, int64_t first_id) {
  if (n_rows <= 0) return;
  CopyPool* pool = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_pool) g_pool = new CopyPool();
    pool = g_pool;
  }
  pool->run((size_t)n_rows, 64, [&](size_t b, size_t e) {
    for (size_t i = b; i < e; ++i)
      for (int64_t q = row_ptr[i]; q < row_ptr[i + 1]; ++q) origin[q] = (int32_t)(first_id + (int64_t)i);
  });
}

bool is_pageable_host(const void* p) { return pageable(p); }

}  // namespace pr
