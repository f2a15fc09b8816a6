// extern "C" entry points of libporerad (declared in include/porerad.h).
#include <new>

#include "pr_objects.cuh"

namespace pr {

static thread_local std::string g_error;

void set_error(const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_error = buf;
}

int case_build(pr_case* c, const uint8_t* phases, cudaStream_t s);
int generate_rays(const pr_case* c, int64_t p0, int64_t p1, int64_t R, const pr_pcg64* seed, double* origins,
                  double* dirs, cudaStream_t s);
int trace_given(const pr_case* c, const double* origins, const double* dirs, int64_t n, int32_t* receiver,
                int64_t* n_failed, cudaStream_t s);
int first_hit_counts(const pr_case* c, int64_t R, const pr_pcg64* seeds, int S, cudaStream_t s, pr_counts** out);
struct HostSink;
int counts_batch(const pr_case* const* cases, int nc, int64_t R, const pr_pcg64* seeds, int S, cudaStream_t s,
                 pr_counts** out, HostSink* sink);
int first_hit_counts_host(const pr_case* c, int64_t R, const pr_pcg64* seeds, int S, cudaStream_t s,
                          int32_t* origin, int32_t* receiver, int64_t* count, int64_t capacity, int64_t* n_pairs);
int counts_from_edges(const int32_t* origin, const int32_t* receiver, const int64_t* count, int64_t m, int64_t n,
                      cudaStream_t s, pr_counts** out);
int counts_from_tables(const int32_t* const* origin, const int32_t* const* receiver, const int64_t* const* count,
                       const int64_t* n_edges, int n_tables, int64_t n, cudaStream_t s, pr_counts** out);
int counts_merge(const pr_counts* A, const pr_counts* B, cudaStream_t s, pr_counts** out);
int operator_create(const pr_counts* k, const int64_t* rays, const double* area, double delta, double tol,
                    cudaStream_t s, pr_operator** out);
int operators_create_batch(const pr_counts* const* counts, const int64_t* const* rays, const double* const* area,
                           int n_ops, double delta, double tol, cudaStream_t s, pr_operator** out);
int apply(const pr_operator* op, int which, const double* x, double* y, cudaStream_t s);
int reciprocity_error(const pr_operator* op, double* out, cudaStream_t s);
int operator_edges(const pr_operator* op, int32_t* origin, int32_t* receiver, double* weight, cudaStream_t s);
int reflection_series(const pr_operator* op, const double* emitted, const double* eps, double rtol, int64_t max_it,
                      double* absorbed, double* residual, int64_t* iterations, cudaStream_t s);
int net_patch_power(const pr_operator* op, const double* T, const double* eps, const double* area, double rtol,
                    int has_ref, double ref, int64_t max_it, double* emitted, double* absorbed, double* net,
                    double* residual, int64_t* iterations, cudaStream_t s);
int net_patch_power_jvp(const pr_operator* op, const double* T, const double* dTin, const double* eps,
                        const double* area, double rtol, double* out, cudaStream_t s);
int prescribed_channels(const pr_case* c, const pr_operator* op, double T_m, double dT, double epsv, int precision,
                        double rtol, double* q, double* coarse, double* stats, cudaStream_t s);
int cell_field_channels(const pr_case* c, const pr_operator* op, const double* T_cells, double Th, double Tc,
                        double epsv, int has_ref, double ref, int precision, double rtol, double* q, double* coarse,
                        double* stats, cudaStream_t s);

}  // namespace pr

using namespace pr;

#define PR_ENTRY_GUARD(obj) DeviceGuard _guard((obj)->device)

#define PR_CHECK_NULL(p, name)                                  \
  do {                                                          \
    if (!(p)) {                                                 \
      set_error("%s must not be NULL", name);                   \
      return PR_ERR_ARG;                                        \
    }                                                           \
  } while (0)

extern "C" {

const char* pr_last_error(void) { return g_error.c_str(); }

int pr_version(void) { return 1; }

int pr_case_create(const uint8_t* phases_x, int64_t nx, int64_t ny, int64_t nz, double H_m, void* stream,
                   pr_case** out) {
  PR_CHECK_NULL(out, "out");
  *out = nullptr;
  PR_CHECK_NULL(phases_x, "phases_x");
  PR_ARG(nx > 0 && ny > 0 && nz > 0, "grid dimensions must be positive");
  PR_ARG(nx < (1 << 30) && ny < (1 << 30) && nz < (1 << 30) && nx * ny * nz < ((int64_t)1 << 36),
         "grid too large");
  cudaStream_t s = (cudaStream_t)stream;
  pr_case* c = new (std::nothrow) pr_case();
  if (!c) {
    set_error("host allocation failed");
    return PR_ERR_OOM;
  }
  cudaGetDevice(&c->device);
  c->nx = nx;
  c->ny = ny;
  c->nz = nz;
  c->n_cells = nx * ny * nz;
  c->H = H_m;
  const double h = H_m / (double)nx;
  c->area = h * h;
  c->last_stream = s;
  int st = case_build(c, phases_x, s);
  if (st == PR_OK) {
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
      set_error("CUDA error %s building the surface patches", cudaGetErrorString(e));
      st = PR_ERR_CUDA;
    }
  }
  if (st != PR_OK) {
    delete c;
    return st;
  }
  *out = c;
  return PR_OK;
}

int pr_case_info(const pr_case* c, int64_t* n_patches, int64_t* n_wall, size_t* device_bytes) {
  PR_CHECK_NULL(c, "case");
  if (n_patches) *n_patches = c->n_patches;
  if (n_wall) *n_wall = c->n_wall;
  if (device_bytes) *device_bytes = c->device_bytes();
  return PR_OK;
}

__global__ void k_normals(const int8_t* __restrict__ code, int64_t n, double* __restrict__ out) {
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
    const int c = code[p];
    out[3 * p] = 0.0;
    out[3 * p + 1] = 0.0;
    out[3 * p + 2] = 0.0;
    out[3 * p + (c >> 1)] = (c & 1) ? -1.0 : 1.0;
  }
}

__global__ void k_fill_f64(double* __restrict__ out, int64_t n, double v) {
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) out[p] = v;
}

int pr_case_patches(const pr_case* c, uint8_t* solid, int8_t* patch_class, int32_t* patch_cell, int8_t* patch_face,
                    double* patch_origin, double* patch_normal, double* patch_area_m2, int32_t* cell_face_patch,
                    int32_t* hot_wall_patch, int32_t* cold_wall_patch, void* stream) {
  PR_CHECK_NULL(c, "case");
  PR_ENTRY_GUARD(c);
  cudaStream_t s = (cudaStream_t)stream;
  const int64_t P = c->n_patches, lat = c->ny * c->nz;
  if (solid) PR_CUDA(cudaMemcpyAsync(solid, c->solid.ptr, c->n_cells, cudaMemcpyDefault, s));
  if (patch_class && P) PR_CUDA(cudaMemcpyAsync(patch_class, c->cls.ptr, P, cudaMemcpyDefault, s));
  if (patch_cell && P) PR_CUDA(cudaMemcpyAsync(patch_cell, c->cell.ptr, P * 4, cudaMemcpyDefault, s));
  if (patch_face && P) PR_CUDA(cudaMemcpyAsync(patch_face, c->face.ptr, P, cudaMemcpyDefault, s));
  if (patch_origin && P) PR_CUDA(cudaMemcpyAsync(patch_origin, c->origin.ptr, P * 24, cudaMemcpyDefault, s));
  DevBuf<double> tmp;
  if ((patch_normal || patch_area_m2) && P) {
    PR_TRY(tmp.alloc(3 * P, s));
    if (patch_normal) {
      ::pr::launch_mark(), k_normals<<<grid_for(P, 256), 256, 0, s>>>(c->code.ptr, P, tmp.ptr);
      PR_CUDA(cudaGetLastError());
      PR_CUDA(cudaMemcpyAsync(patch_normal, tmp.ptr, P * 24, cudaMemcpyDefault, s));
    }
  }
  if (patch_area_m2 && P) {
    DevBuf<double> a;
    PR_TRY(a.alloc(P, s));
    ::pr::launch_mark(), k_fill_f64<<<grid_for(P, 256), 256, 0, s>>>(a.ptr, P, c->area);
    PR_CUDA(cudaGetLastError());
    PR_CUDA(cudaMemcpyAsync(patch_area_m2, a.ptr, P * 8, cudaMemcpyDefault, s));
    PR_CUDA(cudaStreamSynchronize(s));
  }
  if (cell_face_patch) PR_CUDA(cudaMemcpyAsync(cell_face_patch, c->cfp(), c->n_cells * 24, cudaMemcpyDefault, s));
  if (hot_wall_patch) PR_CUDA(cudaMemcpyAsync(hot_wall_patch, c->hot(), lat * 4, cudaMemcpyDefault, s));
  if (cold_wall_patch) PR_CUDA(cudaMemcpyAsync(cold_wall_patch, c->cold(), lat * 4, cudaMemcpyDefault, s));
  PR_CUDA(cudaStreamSynchronize(s));
  return PR_OK;
}

void pr_case_destroy(pr_case* c) {
  if (!c) return;
  DeviceGuard g(c->device);
  c->rebind(c->last_stream);
  delete c;
}

static bool seeds_ok(const pr_pcg64* seeds) { return seeds != nullptr; }

int pr_generate_rays(const pr_case* c, int64_t patch_start, int64_t patch_end, int64_t rays_per_patch,
                     const pr_pcg64* seed, double* origins, double* directions, void* stream) {
  PR_CHECK_NULL(c, "case");
  PR_ARG(seeds_ok(seed), "seed must not be NULL");
  PR_ENTRY_GUARD(c);
  return generate_rays(c, patch_start, patch_end, rays_per_patch, seed, origins, directions, (cudaStream_t)stream);
}

int pr_trace_first_hit(const pr_case* c, const double* origins, const double* directions, int64_t n_rays,
                       int32_t* receiver, int64_t* n_failed, void* stream) {
  PR_CHECK_NULL(c, "case");
  PR_ARG(n_rays >= 0, "negative ray count");
  PR_ENTRY_GUARD(c);
  return trace_given(c, origins, directions, n_rays, receiver, n_failed, (cudaStream_t)stream);
}

int pr_first_hit_counts(const pr_case* c, int64_t rays_per_patch, const pr_pcg64* seeds, int n_seeds, void* stream,
                        pr_counts** out) {
  PR_CHECK_NULL(c, "case");
  PR_CHECK_NULL(out, "out");
  *out = nullptr;
  PR_ARG(seeds_ok(seeds), "seeds must not be NULL");
  PR_ENTRY_GUARD(c);
  return first_hit_counts(c, rays_per_patch, seeds, n_seeds, (cudaStream_t)stream, out);
}

int pr_first_hit_counts_host(const pr_case* c, int64_t rays_per_patch, const pr_pcg64* seeds, int n_seeds,
                             void* stream, int32_t* origin, int32_t* receiver, int64_t* count, int64_t capacity,
                             int64_t* n_pairs) {
  PR_CHECK_NULL(c, "case");
  PR_CHECK_NULL(n_pairs, "n_pairs");
  *n_pairs = 0;
  PR_ARG(seeds_ok(seeds), "seeds must not be NULL");
  PR_ARG(origin && receiver && count, "origin, receiver and count must not be NULL");
  PR_ARG(capacity >= 0, "negative capacity");
  PR_ENTRY_GUARD(c);
  return first_hit_counts_host(c, rays_per_patch, seeds, n_seeds, (cudaStream_t)stream, origin, receiver, count,
                               capacity, n_pairs);
}

int pr_first_hit_counts_batch(const pr_case* const* cases, int n_cases, int64_t rays_per_patch,
                              const pr_pcg64* seeds, int n_seeds, void* stream, pr_counts** out) {
  PR_CHECK_NULL(cases, "cases");
  PR_CHECK_NULL(out, "out");
  PR_ARG(n_cases > 0, "n_cases must be positive");
  PR_ARG(seeds_ok(seeds), "seeds must not be NULL");
  for (int c = 0; c < n_cases; ++c) out[c] = nullptr;
  PR_CHECK_NULL(cases[0], "cases[0]");
  PR_ENTRY_GUARD(cases[0]);
  return counts_batch(cases, n_cases, rays_per_patch, seeds, n_seeds, (cudaStream_t)stream, out, nullptr);
}

int pr_counts_info(const pr_counts* k, int64_t* nnz, int64_t* n_patches, int64_t* rays, int64_t* dda_steps) {
  PR_CHECK_NULL(k, "counts");
  if (nnz) *nnz = k->csr->nnz;
  if (n_patches) *n_patches = k->csr->n_rows;
  if (rays) *rays = k->rays_traced;
  if (dda_steps) *dda_steps = k->dda_steps;
  return PR_OK;
}

// Rows [r0, r1) of a count table as the reference's edge arrays: origin id and 64-bit count per
// pair, written from position 0 (pair rp[r0] goes to index 0).  One warp per row.
__global__ void k_expand_rows(const int64_t* __restrict__ rp, const int32_t* __restrict__ cnt, int64_t r0,
                              int64_t r1, int32_t* __restrict__ origin, int64_t* __restrict__ count) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  const int64_t base = rp[r0];
  for (int64_t i = r0 + blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); i < r1; i += warps)
    for (int64_t q = rp[i] + lane; q < rp[i + 1]; q += 32) {
      if (origin) origin[q - base] = (int32_t)i;
      if (count) count[q - base] = cnt[q];
    }
}

// Rows [r0, r1) of a count table into pageable host arrays without expanding them on the device:
// the row offsets come over (8 B per row), origins are filled on the host from them, and
// the counts cross as the table's int32 values, widened to int64 on the host; 8 B per pair cross
// the bus instead of 16.
static int rows_to_pageable(const CountCsr& c, int64_t r0, int64_t r1, int64_t base, int64_t m, int32_t* origin,
                            int32_t* receiver, int64_t* count, cudaStream_t s) {
  if (origin) {
    std::vector<int64_t> rp((size_t)(r1 - r0 + 1));
    PR_CUDA(cudaMemcpyAsync(rp.data(), c.row_ptr.ptr + r0, rp.size() * 8, cudaMemcpyDeviceToHost, s));
    PR_CUDA(cudaStreamSynchronize(s));
    for (auto& v : rp) v -= base;
    fill_rows_host(origin, rp.data(), r1 - r0, r0);
  }
  if (count) PR_TRY(copy_to_host_i64(count, c.cnt.ptr + base, m, s));
  if (receiver) PR_TRY(copy_to_host(receiver, c.col.ptr + base, (size_t)m * 4, s));
  return PR_OK;
}

static bool large_pageable(int64_t m, const void* a, const void* b) {
  return m * 4 > ((int64_t)16 << 20) && (a || b) && (!a || is_pageable_host(a)) && (!b || is_pageable_host(b));
}

int pr_counts_copy(const pr_counts* k, int32_t* origin, int32_t* receiver, int64_t* count, int64_t* rays_per_origin,
                   void* stream) {
  PR_CHECK_NULL(k, "counts");
  PR_ENTRY_GUARD(k);
  cudaStream_t s = (cudaStream_t)stream;
  const CountCsr& c = *k->csr;
  const int64_t m = c.nnz, n = c.n_rows;
  if (large_pageable(m, origin, count)) {
    PR_TRY(rows_to_pageable(c, 0, n, 0, m, origin, receiver, count, s));
    if (rays_per_origin && n > 0) PR_TRY(copy_to_host(rays_per_origin, k->rays.ptr, n * 8, s));
    PR_CUDA(cudaStreamSynchronize(s));
    return PR_OK;
  }
  DevBuf<int32_t> o;
  DevBuf<int64_t> cn;
  if (m > 0 && (origin || count)) {
    if (origin) PR_TRY(o.alloc(m, s));
    if (count) PR_TRY(cn.alloc(m, s));
    ::pr::launch_mark(), k_expand_rows<<<grid_for(n * 32, 256), 256, 0, s>>>(c.row_ptr.ptr, c.cnt.ptr, 0, n,
                                                                             origin ? o.ptr : nullptr,
                                                                             count ? cn.ptr : nullptr);
    PR_CUDA(cudaGetLastError());
    if (origin) PR_TRY(copy_to_host(origin, o.ptr, m * 4, s));
    if (count) PR_TRY(copy_to_host(count, cn.ptr, m * 8, s));
  }
  if (receiver && m > 0) PR_TRY(copy_to_host(receiver, c.col.ptr, m * 4, s));
  if (rays_per_origin && n > 0) PR_TRY(copy_to_host(rays_per_origin, k->rays.ptr, n * 8, s));
  PR_CUDA(cudaStreamSynchronize(s));
  return PR_OK;
}

int pr_host_block(long long bytes, void** out) {
  PR_CHECK_NULL(out, "out");
  PR_ARG(bytes > 0, "a host block needs a positive size");
  return host_block_take((size_t)bytes, out, true);
}

int pr_host_block_release(void* block) {
  PR_CHECK_NULL(block, "block");
  return host_block_give(block);
}

int pr_host_blocks_trim(long long keep_bytes) {
  PR_ARG(keep_bytes >= 0, "keep_bytes must not be negative");
  return host_blocks_trim((size_t)keep_bytes);
}

int pr_host_blocks_stats(long long* live_bytes, long long* cached_bytes, long long* allocations, long long* reuses) {
  host_blocks_stats(live_bytes, cached_bytes, allocations, reuses);
  return PR_OK;
}

int pr_counts_rows(const pr_counts* k, int64_t row_begin, int64_t row_end, int64_t* n_pairs, int32_t* origin,
                   int32_t* receiver, int64_t* count, void* stream) {
  PR_CHECK_NULL(k, "counts");
  PR_CHECK_NULL(n_pairs, "n_pairs");
  PR_ENTRY_GUARD(k);
  cudaStream_t s = (cudaStream_t)stream;
  const CountCsr& c = *k->csr;
  PR_ARG(0 <= row_begin && row_begin <= row_end && row_end <= c.n_rows, "row range outside the count table");
  int64_t bounds[2] = {0, 0};
  if (row_end > row_begin) {
    PR_CUDA(cudaMemcpyAsync(&bounds[0], c.row_ptr.ptr + row_begin, 8, cudaMemcpyDeviceToHost, s));
    PR_CUDA(cudaMemcpyAsync(&bounds[1], c.row_ptr.ptr + row_end, 8, cudaMemcpyDeviceToHost, s));
    PR_CUDA(cudaStreamSynchronize(s));
  }
  const int64_t m = bounds[1] - bounds[0];
  *n_pairs = m;
  if (m == 0 || (!origin && !receiver && !count)) return PR_OK;
  if (large_pageable(m, origin, count)) {
    PR_TRY(rows_to_pageable(c, row_begin, row_end, bounds[0], m, origin, receiver, count, s));
    PR_CUDA(cudaStreamSynchronize(s));
    return PR_OK;
  }
  DevBuf<int32_t> o;
  DevBuf<int64_t> cn;
  if (origin) PR_TRY(o.alloc(m, s));
  if (count) PR_TRY(cn.alloc(m, s));
  if (origin || count) {
    const int64_t rows = row_end - row_begin;
    ::pr::launch_mark(), k_expand_rows<<<grid_for(rows * 32, 256), 256, 0, s>>>(c.row_ptr.ptr, c.cnt.ptr, row_begin,
                                                                                row_end, origin ? o.ptr : nullptr,
                                                                                count ? cn.ptr : nullptr);
    PR_CUDA(cudaGetLastError());
  }
  if (origin) PR_TRY(copy_to_host(origin, o.ptr, m * 4, s));
  if (count) PR_TRY(copy_to_host(count, cn.ptr, m * 8, s));
  if (receiver) PR_TRY(copy_to_host(receiver, c.col.ptr + bounds[0], m * 4, s));
  PR_CUDA(cudaStreamSynchronize(s));
  return PR_OK;
}

int pr_counts_from_edges(const int32_t* origin, const int32_t* receiver, const int64_t* count, int64_t n_edges,
                         int64_t n_patches, void* stream, pr_counts** out) {
  PR_CHECK_NULL(out, "out");
  *out = nullptr;
  PR_ARG(n_edges == 0 || (origin && receiver && count), "edge arrays must not be NULL");
  return counts_from_edges(origin, receiver, count, n_edges, n_patches, (cudaStream_t)stream, out);
}

int pr_counts_from_tables(const int32_t* const* origin, const int32_t* const* receiver, const int64_t* const* count,
                          const int64_t* n_edges, int n_tables, int64_t n_patches, void* stream, pr_counts** out) {
  PR_CHECK_NULL(out, "out");
  PR_ARG(n_tables == 0 || (origin && receiver && count && n_edges), "table arrays must not be NULL");
  return counts_from_tables(origin, receiver, count, n_edges, n_tables, n_patches, (cudaStream_t)stream, out);
}

int pr_counts_merge(const pr_counts* a, const pr_counts* b, void* stream, pr_counts** out) {
  PR_CHECK_NULL(a, "a");
  PR_CHECK_NULL(b, "b");
  PR_CHECK_NULL(out, "out");
  *out = nullptr;
  PR_ARG(a->device == b->device, "count tables live on different devices");
  PR_ENTRY_GUARD(a);
  return counts_merge(a, b, (cudaStream_t)stream, out);
}

void pr_counts_destroy(pr_counts* k) {
  if (!k) return;
  DeviceGuard g(k->device);
  delete k;
}

int pr_operator_create(const pr_counts* counts, const int64_t* rays_per_origin, const double* patch_area_m2,
                       double support_diagonal_fraction, double balance_tolerance, void* stream, pr_operator** out) {
  PR_CHECK_NULL(counts, "counts");
  PR_CHECK_NULL(out, "out");
  *out = nullptr;
  PR_CHECK_NULL(rays_per_origin, "rays_per_origin");
  PR_CHECK_NULL(patch_area_m2, "patch_area_m2");
  PR_ENTRY_GUARD(counts);
  return operator_create(counts, rays_per_origin, patch_area_m2, support_diagonal_fraction, balance_tolerance,
                         (cudaStream_t)stream, out);
}

int pr_operator_create_batch(const pr_counts* const* counts, const int64_t* const* rays_per_origin,
                             const double* const* patch_area_m2, int n_ops, double support_diagonal_fraction,
                             double balance_tolerance, void* stream, pr_operator** out) {
  PR_CHECK_NULL(out, "out");
  PR_ARG(n_ops >= 0, "n_ops must not be negative");
  if (n_ops == 0) return PR_OK;
  PR_CHECK_NULL(counts, "counts");
  PR_CHECK_NULL(rays_per_origin, "rays_per_origin");
  PR_CHECK_NULL(patch_area_m2, "patch_area_m2");
  for (int k = 0; k < n_ops; ++k) {
    out[k] = nullptr;
    PR_ARG(counts[k] && rays_per_origin[k] && patch_area_m2[k], "operator %d: counts, rays and areas must not be NULL",
           k);
    PR_ARG(counts[k]->device == counts[0]->device, "count tables live on different devices");
  }
  PR_ENTRY_GUARD(counts[0]);
  return operators_create_batch(counts, rays_per_origin, patch_area_m2, n_ops, support_diagonal_fraction,
                                balance_tolerance, (cudaStream_t)stream, out);
}

int pr_operator_info(const pr_operator* op, double* scale, int* balance_method, int* balance_iterations,
                     double* row_sum_error, int64_t* nnz_counts, int64_t* nnz_symmetric, int64_t* spmv_calls) {
  PR_CHECK_NULL(op, "operator");
  PR_ENTRY_GUARD(op);
  if (scale && op->n) {
    PR_CUDA(cudaMemcpyAsync(scale, op->scale.ptr, op->n * 8, cudaMemcpyDefault, op->last_stream));
    PR_CUDA(cudaStreamSynchronize(op->last_stream));
  }
  if (balance_method) *balance_method = op->method;
  if (balance_iterations) *balance_iterations = op->iterations;
  if (row_sum_error) *row_sum_error = op->row_sum_error;
  if (nnz_counts) *nnz_counts = op->F->nnz;
  if (nnz_symmetric) *nnz_symmetric = op->S.nnz;
  if (spmv_calls) *spmv_calls = op->spmv_calls;
  return PR_OK;
}

int pr_operator_apply(const pr_operator* op, int which, const double* x, double* y, void* stream) {
  PR_CHECK_NULL(op, "operator");
  PR_ARG(which >= PR_APPLY_RAW && which <= PR_APPLY_RMATVEC, "unknown product %d", which);
  PR_ENTRY_GUARD(op);
  cudaStream_t s = (cudaStream_t)stream;
  const int64_t n = op->n;
  if (n == 0) return PR_OK;
  DevBuf<double> dx, dy;
  PR_TRY(dx.alloc(n, s));
  PR_TRY(dy.alloc(n, s));
  PR_CUDA(cudaMemcpyAsync(dx.ptr, x, n * 8, cudaMemcpyDefault, s));
  PR_TRY(apply(op, which, dx.ptr, dy.ptr, s));
  PR_CUDA(cudaMemcpyAsync(y, dy.ptr, n * 8, cudaMemcpyDefault, s));
  PR_CUDA(cudaStreamSynchronize(s));
  return PR_OK;
}

int pr_operator_reciprocity_error(const pr_operator* op, double* out, void* stream) {
  PR_CHECK_NULL(op, "operator");
  PR_CHECK_NULL(out, "out");
  PR_ENTRY_GUARD(op);
  return reciprocity_error(op, out, (cudaStream_t)stream);
}

int pr_operator_edges(const pr_operator* op, int32_t* origin, int32_t* receiver, double* weight, void* stream) {
  PR_CHECK_NULL(op, "operator");
  PR_ENTRY_GUARD(op);
  return operator_edges(op, origin, receiver, weight, (cudaStream_t)stream);
}

void pr_operator_destroy(pr_operator* op) {
  if (!op) return;
  DeviceGuard g(op->device);
  delete op;
}

int pr_reflection_series(const pr_operator* op, const double* emitted, const double* emissivity,
                         double relative_tolerance, int64_t max_reflections, double* absorbed,
                         double* residual_power, int64_t* iterations, void* stream) {
  PR_CHECK_NULL(op, "operator");
  PR_CHECK_NULL(emitted, "emitted");
  PR_CHECK_NULL(emissivity, "emissivity");
  PR_CHECK_NULL(absorbed, "absorbed");
  PR_ARG(max_reflections >= 1, "max_reflections must be at least 1");
  PR_ENTRY_GUARD(op);
  double res = 0.0;
  int64_t it = 0;
  int st = reflection_series(op, emitted, emissivity, relative_tolerance, max_reflections, absorbed, &res, &it,
                             (cudaStream_t)stream);
  if (residual_power) *residual_power = res;
  if (iterations) *iterations = it;
  return st;
}

int pr_net_patch_power(const pr_operator* op, const double* temperature_K, const double* emissivity,
                       const double* area_m2, double relative_tolerance, int has_reference,
                       double reference_temperature_K, int64_t max_reflections, double* emitted, double* absorbed,
                       double* net, double* residual_power, int64_t* iterations, void* stream) {
  PR_CHECK_NULL(op, "operator");
  PR_CHECK_NULL(temperature_K, "temperature_K");
  PR_CHECK_NULL(emissivity, "emissivity");
  PR_CHECK_NULL(area_m2, "area_m2");
  PR_ARG(max_reflections >= 1, "max_reflections must be at least 1");
  PR_ENTRY_GUARD(op);
  return net_patch_power(op, temperature_K, emissivity, area_m2, relative_tolerance, has_reference,
                         reference_temperature_K, max_reflections, emitted, absorbed, net, residual_power, iterations,
                         (cudaStream_t)stream);
}

int pr_net_patch_power_jvp(const pr_operator* op, const double* temperature_K, const double* delta_temperature_K,
                           const double* emissivity, const double* area_m2, double relative_tolerance, double* out,
                           void* stream) {
  PR_CHECK_NULL(op, "operator");
  PR_CHECK_NULL(temperature_K, "temperature_K");
  PR_CHECK_NULL(delta_temperature_K, "delta_temperature_K");
  PR_CHECK_NULL(emissivity, "emissivity");
  PR_CHECK_NULL(area_m2, "area_m2");
  PR_CHECK_NULL(out, "out");
  PR_ENTRY_GUARD(op);
  return net_patch_power_jvp(op, temperature_K, delta_temperature_K, emissivity, area_m2, relative_tolerance, out,
                             (cudaStream_t)stream);
}

int pr_prescribed_field_channels(const pr_case* c, const pr_operator* op, double T_mean_K, double delta_T_K,
                                 double epsilon, int precision, double relative_tolerance, double* q, double* coarse,
                                 double* stats, void* stream) {
  PR_CHECK_NULL(c, "case");
  PR_CHECK_NULL(op, "operator");
  PR_CHECK_NULL(q, "q");
  PR_ARG(precision == PR_PRECISION_FP64 || precision == PR_PRECISION_MIXED, "unknown precision %d", precision);
  PR_ARG(c->device == op->device, "case and operator live on different devices");
  PR_ENTRY_GUARD(c);
  return prescribed_channels(c, op, T_mean_K, delta_T_K, epsilon, precision, relative_tolerance, q, coarse, stats,
                             (cudaStream_t)stream);
}

int pr_cell_field_channels(const pr_case* c, const pr_operator* op, const double* T_cells, double T_hot_K,
                           double T_cold_K, double epsilon, int has_reference, double reference_temperature_K,
                           int precision, double relative_tolerance, double* q, double* coarse, double* stats,
                           void* stream) {
  PR_CHECK_NULL(c, "case");
  PR_CHECK_NULL(op, "operator");
  PR_CHECK_NULL(T_cells, "T_cells");
  PR_CHECK_NULL(q, "q");
  PR_ARG(precision == PR_PRECISION_FP64 || precision == PR_PRECISION_MIXED, "unknown precision %d", precision);
  PR_ARG(c->device == op->device, "case and operator live on different devices");
  PR_ENTRY_GUARD(c);
  return cell_field_channels(c, op, T_cells, T_hot_K, T_cold_K, epsilon, has_reference, reference_temperature_K,
                             precision, relative_tolerance, q, coarse, stats, (cudaStream_t)stream);
}

}  // extern "C"
