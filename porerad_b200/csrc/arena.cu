// Device-memory cache of libporerad: every DevBuf allocation goes through here.
//
// A served step allocates and frees the same few hundred buffers (ray chunks, stage
// buffers, CSR arrays, sort scratch, solver vectors) in the same sizes every time.  Each
// cudaMallocAsync call is a driver call that has been seen to block the host for tens to
// hundreds of milliseconds on a busy machine, even with the pool's memory already mapped,
// and the GPU idles meanwhile.  Freed blocks are therefore kept per device in free lists
// keyed by a rounded size; a block carries an event recorded on the stream of its last
// use, and the next allocation of that size takes it after an in-stream wait on the event
// (no host synchronisation, no driver allocation).  Cached bytes are bounded
// (PORERAD_CACHE_BYTES, default a quarter of the device memory); the oldest blocks are
// returned to the stream-ordered pool beyond that, and an allocation that fails releases
// the whole cache and retries once.
#include <cstdlib>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "pr_internal.cuh"

namespace pr {
namespace {

struct Block {
  void* ptr;
  size_t size;
  cudaEvent_t ev;
  unsigned long long tick;
};

struct DeviceArena {
  std::mutex mu;
  std::unordered_map<size_t, std::vector<Block>> free;
  std::vector<cudaEvent_t> spare;
  size_t cached = 0, live = 0, limit = 0;
  long long mallocs = 0, hits = 0;
  unsigned long long tick = 0;
  bool init = false;
};

constexpr int kMaxDevices = 64;

// Never destroyed: the process may end after the CUDA context is gone.
DeviceArena* arenas() {
  static DeviceArena* a = new DeviceArena[kMaxDevices];
  return a;
}

// Size classes: powers of two up to 1 MiB; above, multiples of max(2 MiB, 2^floor(log2 b) / 8),
// so a block serves requests within 12.5 % of its size.
size_t bucket(size_t b) {
  if (b <= 512) return 512;
  if (b <= ((size_t)1 << 20)) {
    size_t p = 512;
    while (p < b) p <<= 1;
    return p;
  }
  size_t hi = (size_t)1 << 20;
  while ((hi << 1) <= b) hi <<= 1;
  size_t g = hi / 8;
  if (g < ((size_t)2 << 20)) g = (size_t)2 << 20;
  return (b + g - 1) / g * g;
}

cudaEvent_t take_event(DeviceArena& A) {
  if (!A.spare.empty()) {
    cudaEvent_t e = A.spare.back();
    A.spare.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return e;
}

void setup(DeviceArena& A) {
  if (A.init) return;
  size_t free_b = 0, total_b = 0;
  A.limit = cudaMemGetInfo(&free_b, &total_b) == cudaSuccess ? total_b / 4 : ((size_t)16 << 30);
  if (const char* env = std::getenv("PORERAD_CACHE_BYTES")) A.limit = (size_t)std::strtoull(env, nullptr, 10);
  A.init = true;
}

// Return the oldest cached blocks to the pool until at most `keep` bytes stay cached; the
// frees are ordered after each block's last use by a wait on its event.  Caller holds A.mu.
void trim(DeviceArena& A, size_t keep, cudaStream_t s) {
  while (A.cached > keep) {
    std::vector<Block>* from = nullptr;
    size_t at = 0;
    unsigned long long oldest = ~0ull;
    for (auto& kv : A.free)
      for (size_t k = 0; k < kv.second.size(); ++k)
        if (kv.second[k].tick < oldest) {
          oldest = kv.second[k].tick;
          from = &kv.second;
          at = k;
        }
    if (!from) break;
    Block b = (*from)[at];
    from->erase(from->begin() + (ptrdiff_t)at);
    if (b.ev) cudaStreamWaitEvent(s, b.ev, 0);
    cudaFreeAsync(b.ptr, s);
    if (b.ev) A.spare.push_back(b.ev);
    A.cached -= b.size;
  }
}

}  // namespace

int arena_alloc(size_t bytes, cudaStream_t s, void** out, int* dev_out) {
  int dev = 0;
  PR_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("device %d outside the supported range", dev);
    return PR_ERR_LIMIT;
  }
  *dev_out = dev;
  DeviceArena& A = arenas()[dev];
  const size_t b = bucket(bytes);
  {
    std::lock_guard<std::mutex> lk(A.mu);
    setup(A);
    auto it = A.free.find(b);
    if (it != A.free.end() && !it->second.empty()) {
      Block blk = it->second.back();
      it->second.pop_back();
      if (blk.ev) {
        cudaStreamWaitEvent(s, blk.ev, 0);  // after the block's last use
        A.spare.push_back(blk.ev);
      }
      A.cached -= b;
      A.live += b;
      A.hits++;
      *out = blk.ptr;
      return PR_OK;
    }
  }
  retain_pool_memory();
  cudaError_t e = cudaMallocAsync(out, b, s);
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();
    {
      std::lock_guard<std::mutex> lk(A.mu);
      trim(A, 0, s);
    }
    cudaDeviceSynchronize();  // only on this rare path: let the pool take the released blocks back
    e = cudaMallocAsync(out, b, s);
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    *out = nullptr;
    set_error("device allocation of %zu bytes failed: %s", b, cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? PR_ERR_OOM : PR_ERR_CUDA;
  }
  std::lock_guard<std::mutex> lk(A.mu);
  A.live += b;
  A.mallocs++;
  return PR_OK;
}

void arena_free(void* p, size_t bytes, cudaStream_t s, int dev) {
  if (!p || dev < 0 || dev >= kMaxDevices) return;
  int cur = -1;
  cudaGetDevice(&cur);
  if (cur != dev) cudaSetDevice(dev);
  DeviceArena& A = arenas()[dev];
  const size_t b = bucket(bytes);
  {
    std::lock_guard<std::mutex> lk(A.mu);
    setup(A);
    cudaEvent_t ev = take_event(A);
    if (ev && cudaEventRecord(ev, s) != cudaSuccess) {
      cudaGetLastError();
      A.spare.push_back(ev);
      ev = nullptr;
    }
    if (!ev) {  // no event: give the block back to the pool in stream order instead
      cudaFreeAsync(p, s);
      A.live -= b;
    } else {
      A.free[b].push_back(Block{p, b, ev, ++A.tick});
      A.cached += b;
      A.live -= b;
      if (A.cached > A.limit) trim(A, A.limit, s);
    }
  }
  if (cur != dev && cur >= 0) cudaSetDevice(cur);
}

}  // namespace pr

extern "C" {

// Device-memory cache counters of one device: bytes cached (freed, kept for reuse), bytes
// live in library objects, driver allocations made, and allocations served from the cache.
PR_API int pr_memory_stats(int device, long long* cached_bytes, long long* live_bytes, long long* device_mallocs,
                           long long* cache_hits) {
  if (device < 0 || device >= pr::kMaxDevices) {
    pr::set_error("device %d outside the supported range", device);
    return PR_ERR_ARG;
  }
  pr::DeviceArena& A = pr::arenas()[device];
  std::lock_guard<std::mutex> lk(A.mu);
  if (cached_bytes) *cached_bytes = (long long)A.cached;
  if (live_bytes) *live_bytes = (long long)A.live;
  if (device_mallocs) *device_mallocs = A.mallocs;
  if (cache_hits) *cache_hits = A.hits;
  return PR_OK;
}

// Return every cached block of the device to the driver (waits for their last uses).
PR_API int pr_memory_release_cached(int device) {
  if (device < 0 || device >= pr::kMaxDevices) {
    pr::set_error("device %d outside the supported range", device);
    return PR_ERR_ARG;
  }
  int cur = -1;
  PR_CUDA(cudaGetDevice(&cur));
  PR_CUDA(cudaSetDevice(device));
  pr::DeviceArena& A = pr::arenas()[device];
  {
    std::lock_guard<std::mutex> lk(A.mu);
    for (auto& kv : A.free)
      for (pr::Block& b : kv.second) {
        if (b.ev) {
          cudaEventSynchronize(b.ev);
          A.spare.push_back(b.ev);
        }
        cudaFree(b.ptr);
        A.cached -= b.size;
      }
    A.free.clear();
  }
  PR_CUDA(cudaDeviceSynchronize());
  if (cur >= 0 && cur != device) PR_CUDA(cudaSetDevice(cur));
  return PR_OK;
}
}
