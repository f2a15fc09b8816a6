// Launch counter, optional per-kernel CUDA-event timers (benchmark instrumentation) and the
// retention setting of the stream-ordered memory pool.
//
// Timers record one event pair on the launching stream around each launch of the
// instrumented kernels while enabled; pr_timers_read() waits for the pending events
// and accumulates the elapsed times per kernel class.
#include <atomic>
#include <cstdlib>
#include <mutex>
#include <vector>

#include "pr_internal.cuh"

namespace pr {

std::atomic<long long> g_launches{0};

namespace {
struct Pending {
  int id;
  cudaEvent_t a, b;
};
std::mutex g_mu;
bool g_on = false;
std::vector<Pending> g_pending;
std::vector<cudaEvent_t> g_free;
long long g_count[kTimerCount] = {0};
double g_ms[kTimerCount] = {0};

cudaEvent_t take_event() {
  if (!g_free.empty()) {
    cudaEvent_t e = g_free.back();
    g_free.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}
thread_local cudaEvent_t t_start[kTimerCount] = {nullptr};
}  // namespace

bool timers_on() { return g_on; }

void retain_pool_memory() {
  static std::atomic<bool> done[64];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64 || done[dev].load(std::memory_order_acquire)) return;
  static std::mutex mu;
  std::lock_guard<std::mutex> lk(mu);
  if (done[dev].load(std::memory_order_relaxed)) return;
  cudaMemPool_t pool;
  size_t free_b = 0, total_b = 0;
  if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess && cudaMemGetInfo(&free_b, &total_b) == cudaSuccess) {
    unsigned long long keep = total_b / 4;
    if (const char* env = std::getenv("PORERAD_POOL_RETAIN_BYTES")) keep = std::strtoull(env, nullptr, 10);
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  done[dev].store(true, std::memory_order_release);
}

void timer_begin(int id, cudaStream_t s) {
  if (!g_on) return;
  std::lock_guard<std::mutex> lk(g_mu);
  cudaEvent_t e = take_event();
  cudaEventRecord(e, s);
  t_start[id] = e;
}

void timer_end(int id, cudaStream_t s) {
  if (!g_on || !t_start[id]) return;
  std::lock_guard<std::mutex> lk(g_mu);
  cudaEvent_t e = take_event();
  cudaEventRecord(e, s);
  g_pending.push_back({id, t_start[id], e});
  t_start[id] = nullptr;
}

static void collect() {
  for (auto& p : g_pending) {
    float ms = 0.f;
    if (cudaEventSynchronize(p.b) == cudaSuccess && cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) {
      g_count[p.id] += 1;
      g_ms[p.id] += ms;
    }
    g_free.push_back(p.a);
    g_free.push_back(p.b);
  }
  g_pending.clear();
}

}  // namespace pr

extern "C" {

PR_API void pr_timers_enable(int on) {
  std::lock_guard<std::mutex> lk(pr::g_mu);
  pr::g_on = on != 0;
}

PR_API void pr_timers_reset(void) {
  std::lock_guard<std::mutex> lk(pr::g_mu);
  pr::collect();
  for (int i = 0; i < pr::kTimerCount; ++i) {
    pr::g_count[i] = 0;
    pr::g_ms[i] = 0.0;
  }
}

PR_API int pr_timers_read(int id, long long* launches, double* total_ms) {
  if (id < 0 || id >= pr::kTimerCount) {
    pr::set_error("unknown timer %d", id);
    return PR_ERR_ARG;
  }
  std::lock_guard<std::mutex> lk(pr::g_mu);
  pr::collect();
  if (launches) *launches = pr::g_count[id];
  if (total_ms) *total_ms = pr::g_ms[id];
  return PR_OK;
}

PR_API long long pr_kernel_launches(void) { return pr::g_launches.load(); }

}  // extern "C"
