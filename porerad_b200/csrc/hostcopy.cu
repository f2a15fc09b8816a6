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
//
// Results that leave the library as host arrays can instead live in pinned host blocks of the
// library (pr_host_block): the device writes them straight into the caller's memory at the
// link's rate, and a block the caller has released is kept for the next result of about its
// size (pinning and first-touch faults are paid once, not per call).
#include <cstdlib>
#include <condition_variable>
#include <functional>
#include <map>
#include <mutex>
#include <thread>
#include <unordered_map>
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

int copy_from_host(void* dst, const void* src, size_t bytes, cudaStream_t s) {
  if (bytes == 0) return PR_OK;
  if (bytes <= kDirectMax || !pageable(src)) {
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
  // host threads fill buffer k & 1 with chunk k while the DMA of chunk k - 1 runs from the other
  for (size_t k = 0; k < n; ++k) {
    const size_t off = k * kChunk, len = (bytes - off) < kChunk ? (bytes - off) : kChunk;
    if (k >= 2) PR_CUDA(cudaEventSynchronize(st->ready[k & 1]));  // chunk k - 2 has left this buffer
    g_pool->copy(st->buf[k & 1], s8 + off, len);
    PR_CUDA(cudaMemcpyAsync(d8 + off, st->buf[k & 1], len, cudaMemcpyHostToDevice, s));
    PR_CUDA(cudaEventRecord(st->ready[k & 1], s));
  }
  // the staging buffers are free again once their last DMAs are done
  for (size_t k = n > 2 ? n - 2 : 0; k < n; ++k) PR_CUDA(cudaEventSynchronize(st->ready[k & 1]));
  return PR_OK;
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

// ---- pinned host blocks handed to callers (sizes rounded up to 2 MiB)
namespace {

constexpr size_t kHostGrain = (size_t)2 << 20;

struct HostBlocks {
  std::mutex mu;
  std::multimap<size_t, char*> free;      // capacity -> cached block
  std::unordered_map<char*, size_t> cap;  // every block of the pool -> capacity
  size_t cached = 0, live = 0;
  long long allocs = 0, hits = 0;
  size_t keep = 0;  // bound on cached bytes
};

HostBlocks& host_blocks() {
  static HostBlocks* h = [] {
    HostBlocks* b = new HostBlocks();
    const char* env = std::getenv("PORERAD_HOST_CACHE_BYTES");
    b->keep = env ? (size_t)std::strtoull(env, nullptr, 10) : ((size_t)32 << 30);
    return b;
  }();
  return *h;
}

// Pinned memory of `bytes` from the driver, or nullptr.  (Registering host memory whose pages
// the copy threads had faulted in together pinned faster, but the c2 count step then showed
// 40 ms more host time per step and the serving rate fell by a quarter: not kept.)
char* pin_new(size_t bytes) {
  char* p = nullptr;
  if (cudaHostAlloc((void**)&p, bytes, cudaHostAllocPortable) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return p;
}

void unpin(char* p) { cudaFreeHost(p); }

// Free cached blocks, largest first, until at most `keep` bytes stay cached (lock held by the
// caller; the blocks to free are returned so that they are unpinned outside the lock).
std::vector<char*> host_trim_locked(HostBlocks& H, size_t keep) {
  std::vector<char*> out;
  while (H.cached > keep && !H.free.empty()) {
    auto it = std::prev(H.free.end());
    H.cached -= it->first;
    H.cap.erase(it->second);
    out.push_back(it->second);
    H.free.erase(it);
  }
  return out;
}

}  // namespace

int host_block_take(size_t bytes, void** out, bool allocate) {
  HostBlocks& H = host_blocks();
  const size_t want = (bytes + kHostGrain - 1) / kHostGrain * kHostGrain;
  *out = nullptr;
  {
    std::lock_guard<std::mutex> lk(H.mu);
    // the smallest cached block that holds the request, if it is at most twice its size
    auto it = H.free.lower_bound(want);
    if (it != H.free.end() && it->first <= 2 * want) {
      *out = it->second;
      H.cached -= it->first;
      H.live += it->first;
      ++H.hits;
      H.free.erase(it);
      return PR_OK;
    }
  }
  if (!allocate) return PR_OK;  // no cached block fits: *out stays NULL
  char* p = pin_new(want);
  if (!p) {
    // cached blocks of other sizes may be what holds the memory: free them and try once more
    std::vector<char*> drop;
    {
      std::lock_guard<std::mutex> lk(H.mu);
      drop = host_trim_locked(H, 0);
    }
    for (char* d : drop) unpin(d);
    p = pin_new(want);
    if (!p) {
      set_error("a pinned host block of %zu bytes could not be allocated", want);
      return PR_ERR_OOM;
    }
  }
  std::lock_guard<std::mutex> lk(H.mu);
  H.cap[p] = want;
  H.live += want;
  ++H.allocs;
  *out = p;
  return PR_OK;
}

int host_block_give(void* ptr) {
  HostBlocks& H = host_blocks();
  char* p = static_cast<char*>(ptr);
  std::vector<char*> drop;
  {
    std::lock_guard<std::mutex> lk(H.mu);
    auto c = H.cap.find(p);
    if (c == H.cap.end()) {
      set_error("not a host block of this library");
      return PR_ERR_ARG;
    }
    for (auto it = H.free.equal_range(c->second).first; it != H.free.end() && it->first == c->second; ++it)
      if (it->second == p) {
        set_error("host block released twice");
        return PR_ERR_ARG;
      }
    H.live -= c->second;
    H.free.emplace(c->second, p);
    H.cached += c->second;
    drop = host_trim_locked(H, H.keep);
  }
  for (char* d : drop) unpin(d);
  return PR_OK;
}

int host_blocks_trim(size_t keep) {
  HostBlocks& H = host_blocks();
  std::vector<char*> drop;
  {
    std::lock_guard<std::mutex> lk(H.mu);
    drop = host_trim_locked(H, keep);
  }
  for (char* d : drop) unpin(d);
  return PR_OK;
}

void host_blocks_stats(long long* live, long long* cached, long long* allocs, long long* hits) {
  HostBlocks& H = host_blocks();
  std::lock_guard<std::mutex> lk(H.mu);
  if (live) *live = (long long)H.live;
  if (cached) *cached = (long long)H.cached;
  if (allocs) *allocs = H.allocs;
  if (hits) *hits = H.hits;
}

}  // namespace pr
