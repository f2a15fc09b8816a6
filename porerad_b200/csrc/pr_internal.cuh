// Internal plumbing of libporerad: status codes, the thread-local error message,
// CUDA error checks and stream-ordered device buffers.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>
#include <atomic>
#include <stdarg.h>
#include <string>
#include <utility>

#include "../../include/porerad.h"

namespace pr {

void set_error(const char* fmt, ...);

// Count of the library's own kernel launches (CUB primitives not included).
extern std::atomic<long long> g_launches;
inline void launch_mark() { g_launches.fetch_add(1, std::memory_order_relaxed); }

// Optional CUDA-event timers around the hot kernels (see timers.cu).
enum TimerId { kTimerTrace = 0, kTimerRle = 1, kTimerBalance = 2, kTimerSeries = 3, kTimerCheb = 4,
               kTimerRefine = 5, kTimerMorph = 6, kTimerLabel = 7, kTimerRender = 8, kTimerCount = 9 };
bool timers_on();
void timer_begin(int id, cudaStream_t s);
void timer_end(int id, cudaStream_t s);

#define PR_CUDA(expr)                                                                      \
  do {                                                                                     \
    cudaError_t _e = (expr);                                                               \
    if (_e != cudaSuccess) {                                                               \
      ::pr::set_error("CUDA error %s (%s) at %s:%d: %s", cudaGetErrorName(_e),             \
                      cudaGetErrorString(_e), __FILE__, __LINE__, #expr);                  \
      return PR_ERR_CUDA;                                                                  \
    }                                                                                      \
  } while (0)

#define PR_TRY(expr)            \
  do {                          \
    int _s = (expr);            \
    if (_s != PR_OK) return _s; \
  } while (0)

#define PR_ARG(cond, ...)                 \
  do {                                    \
    if (!(cond)) {                        \
      ::pr::set_error(__VA_ARGS__);       \
      return PR_ERR_ARG;                  \
    }                                     \
  } while (0)

// Keep freed stream-ordered allocations of the current device's default pool mapped (up to
// PORERAD_POOL_RETAIN_BYTES, default a quarter of the device memory) instead of returning
// them to the driver at every synchronisation; called before each allocation, acts once per device.
void retain_pool_memory();

// The library's device-memory cache (arena.cu): allocate `bytes` for use on stream s (the
// owning device is returned in *dev), and give a block back after its uses on stream s.
int arena_alloc(size_t bytes, cudaStream_t s, void** out, int* dev);
void arena_free(void* p, size_t bytes, cudaStream_t s, int dev);

// Copy bytes from the device to host memory after the work queued on stream s, and return
// once they are there.  Large copies into pageable memory run through pinned staging buffers
// and host threads (hostcopy.cu); everything else is one cudaMemcpyAsync (the caller then
// synchronises the stream as before).
int copy_to_host(void* dst, const void* src, size_t bytes, cudaStream_t s);
// Host (pageable or pinned) -> device copy; pageable sources above 16 MB go through the pinned
// staging buffers, host threads filling one while the other's DMA runs.  Returns once the
// source may be reused.
int copy_from_host(void* dst, const void* src, size_t bytes, cudaStream_t s);
// int32 device values into an int64 host array (widened on the host; same pipeline).
int copy_to_host_i64(int64_t* dst, const int32_t* src, int64_t n, cudaStream_t s);
// origin[q] = first_id + i for every q in [row_ptr[i], row_ptr[i + 1]) (host arrays), over the
// host threads.
void fill_rows_host(int32_t* origin, const int64_t* row_ptr, int64_t n_rows, int64_t first_id);
// Host memory the GPU cannot reach directly (neither pinned nor managed).
bool is_pageable_host(const void* p);
// Pinned host blocks handed to callers, reused after release (PORERAD_HOST_CACHE_BYTES bounds
// the cached bytes, default 32 GiB).
// A block of at least `bytes`: a cached one when one fits (at most twice the size), else a new
// one if `allocate`, else *out = NULL.
int host_block_take(size_t bytes, void** out, bool allocate);
int host_block_give(void* p);
int host_blocks_trim(size_t keep);
void host_blocks_stats(long long* live, long long* cached, long long* allocs, long long* hits);

// A device allocation owned by the library, released in stream order (to the cache).
template <typename T>
struct DevBuf {
  T* ptr = nullptr;
  size_t n = 0;
  cudaStream_t stream = nullptr;
  int dev = -1;

  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept { *this = std::move(o); }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) {
      release();
      ptr = o.ptr;
      n = o.n;
      stream = o.stream;
      dev = o.dev;
      o.ptr = nullptr;
      o.n = 0;
    }
    return *this;
  }
  ~DevBuf() { release(); }

  int alloc(size_t count, cudaStream_t s) {
    release();
    stream = s;
    n = count;
    if (count == 0) return PR_OK;
    const int st = arena_alloc(count * sizeof(T), s, (void**)&ptr, &dev);
    if (st != PR_OK) {
      ptr = nullptr;
      n = 0;
    }
    return st;
  }
  void release() {
    if (ptr) arena_free(ptr, n * sizeof(T), stream, dev);
    ptr = nullptr;
    n = 0;
  }
  size_t bytes() const { return n * sizeof(T); }
};

// True for device (or managed) memory; host and unregistered pointers give false.
inline bool is_device_pointer(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// Device memory (or managed memory) that belongs to the given device.
inline bool is_device_pointer_of(const void* p, int device) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) && a.device == device;
}

inline int grid_for(int64_t n, int block, int cap = 148 * 32) {
  int64_t g = (n + block - 1) / block;
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return (int)g;
}

inline int sm_count() {
  static int n = 0;
  if (n == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}

}  // namespace pr
