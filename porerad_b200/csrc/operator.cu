// Exchange operator on the device: pooling of arbitrary edge lists, the ray
// accounting check, the symmetric exchange matrix, diagonal balancing, the
// projected products and the reciprocity diagnostic.
//
// Follows porerad/exchange.py:37-197:
//   weight w_ij = n_ij / R_i                                       (exchange.py:72)
//   S = 0.5 (A F + F^T A) + delta A                                (exchange.py:108-112)
//   d > 0 with d * (S d) = A, found as y = log d from the residual
//   f(y) = y + log(S e^y) - log A; convergence when max|f| <= tol, acceptance when
//   the closure max|d (S d) / A - 1| <= min(max(10 tol, 10 eps), 1e-10); otherwise
//   the damped multiplicative iteration y += 0.5 (log A - log(d * S d)) until the
//   closure is <= min(tol, 1e-10) (exchange.py:153-197)
//   row_sum_error = max|F_p 1 - 1| <= 1e-10                       (exchange.py:78-80)
// The reference accelerates the log-residual with scipy.optimize.anderson; here it
// is type-II Anderson acceleration (Walker & Ni 2011) of the damped fixed-point map
// y <- y - beta f(y), history m = 10, beta = 1/2, least squares by the normal
// equations with a pseudo-inverse cut at 10 eps of the largest eigenvalue.  The
// solution d is defined by the equation, so the iterate path may differ from
// SciPy's; d itself agrees to the balancing tolerance.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_reduce.cuh>
#include <cub/device/device_scan.cuh>

#include <cmath>
#include <vector>

#include "pr_spmv.cuh"

namespace pr {

__global__ void k_sum_partials(const double* __restrict__ partial, int blocks, int K, double* __restrict__ out) {
  const int k = blockIdx.x;
  const double s = warp_sum_partials(partial, blocks, K, k, threadIdx.x & 31);
  if (threadIdx.x == 0) out[k] = s;
}

int sum_partials(const double* partial, int blocks, int K, double* out, cudaStream_t s) {
  ::pr::launch_mark(), k_sum_partials<<<K, 32, 0, s>>>(partial, blocks, K, out);
  PR_CUDA(cudaGetLastError());
  return PR_OK;
}

static int red_grid() { return sm_count() * 4; }

// ------------------------------------------------------------------ pooling

__global__ void k_edge_keys(const int32_t* __restrict__ o, const int32_t* __restrict__ r, int64_t m, int64_t n,
                            unsigned long long* __restrict__ key, unsigned int* __restrict__ bad) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < m; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t a = o[t], b = r[t];
    if (a < 0 || a >= n || b < 0 || b >= n) {
      atomicOr(bad, 1u);
      key[t] = 0;
    } else {
      key[t] = (unsigned long long)a * (unsigned long long)n + (unsigned long long)b;
    }
  }
}

__global__ void k_keys_to_csr(const unsigned long long* __restrict__ key, const int64_t* __restrict__ sum, int64_t m,
                              int64_t n, int32_t* __restrict__ col, int32_t* __restrict__ cnt,
                              int32_t* __restrict__ row_len, unsigned int* __restrict__ bad) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < m; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t row = (int64_t)(key[t] / (unsigned long long)n);
    col[t] = (int32_t)(key[t] % (unsigned long long)n);
    const int64_t c = sum[t];
    if (c < 0 || c > INT32_MAX) atomicOr(bad, 2u);
    cnt[t] = (int32_t)c;
    atomicAdd(row_len + row, 1);
  }
}

__global__ void k_zero_i32(int32_t* p, int64_t n) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) p[t] = 0;
}

__global__ void k_widen_scan_input(const int32_t* __restrict__ in, int64_t* __restrict__ out, int64_t n) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
    out[t] = in[t];
}

// row_ptr[0] = 0, row_ptr[1..n] = inclusive sum of len (int64)
static int lengths_to_row_ptr(const int64_t* len, int64_t n, int64_t* row_ptr, cudaStream_t s) {
  PR_CUDA(cudaMemsetAsync(row_ptr, 0, sizeof(int64_t), s));
  if (n == 0) return PR_OK;
  size_t b = 0;
  PR_CUDA(cub::DeviceScan::InclusiveSum(nullptr, b, len, row_ptr + 1, n, s));
  DevBuf<uint8_t> tmp;
  PR_TRY(tmp.alloc(b + 16, s));
  PR_CUDA(cub::DeviceScan::InclusiveSum(tmp.ptr, b, len, row_ptr + 1, n, s));
  return PR_OK;
}

__global__ void k_row_sums(const int64_t* __restrict__ rp, const int32_t* __restrict__ cn, int64_t n,
                           int64_t* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t i = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); i < n; i += warps) {
    int64_t s = 0;
    for (int64_t q = rp[i] + lane; q < rp[i + 1]; q += 32) s += cn[q];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) out[i] = s;
  }
}

int counts_from_tables(const int32_t* const* origin, const int32_t* const* receiver, const int64_t* const* count,
                       const int64_t* n_edges, int n_tables, int64_t n, cudaStream_t s, pr_counts** out) {
  PR_ARG(n >= 0 && n < INT32_MAX, "n_patches %lld outside the int32 patch ids", (long long)n);
  PR_ARG(n_tables >= 0, "negative number of tables");
  int64_t m = 0;
  for (int t = 0; t < n_tables; ++t) {
    PR_ARG(n_edges[t] >= 0, "negative edge count");
    PR_ARG(n_edges[t] == 0 || (origin[t] && receiver[t] && count[t]), "table %d has a NULL array", t);
    m += n_edges[t];
  }
  std::unique_ptr<pr_counts> k(new pr_counts());
  cudaGetDevice(&k->device);
  k->csr = std::make_shared<CountCsr>();
  CountCsr& csr = *k->csr;
  csr.n_rows = n;
  PR_TRY(csr.row_ptr.alloc(n + 1, s));
  DevBuf<int32_t> o, r, row_len;
  DevBuf<int64_t> c, c_sorted, sums, len64;
  DevBuf<unsigned long long> key, key_sorted, ukey;
  DevBuf<unsigned int> bad;
  DevBuf<int64_t> nruns;
  PR_TRY(bad.alloc(1, s));
  PR_CUDA(cudaMemsetAsync(bad.ptr, 0, 4, s));
  PR_TRY(row_len.alloc(n > 0 ? n : 1, s));
  ::pr::launch_mark(), k_zero_i32<<<grid_for(n, 256), 256, 0, s>>>(row_len.ptr, n);
  int64_t u = 0;
  if (m > 0) {
    PR_TRY(o.alloc(m, s));
    PR_TRY(r.alloc(m, s));
    PR_TRY(c.alloc(m, s));
    // the tables one after the other into one device edge list (ids are checked on the device)
    int64_t at = 0;
    for (int t = 0; t < n_tables; ++t) {
      const int64_t mt = n_edges[t];
      PR_TRY(copy_from_host(o.ptr + at, origin[t], (size_t)mt * 4, s));
      PR_TRY(copy_from_host(r.ptr + at, receiver[t], (size_t)mt * 4, s));
      PR_TRY(copy_from_host(c.ptr + at, count[t], (size_t)mt * 8, s));
      at += mt;
    }
    PR_TRY(key.alloc(m, s));
    PR_TRY(key_sorted.alloc(m, s));
    PR_TRY(c_sorted.alloc(m, s));
    ::pr::launch_mark(), k_edge_keys<<<grid_for(m, 256), 256, 0, s>>>(o.ptr, r.ptr, m, n, key.ptr, bad.ptr);
    PR_CUDA(cudaGetLastError());
    int end_bit = 1;
    while (end_bit < 64 && (((unsigned long long)1 << end_bit) < (unsigned long long)n * (unsigned long long)n)) ++end_bit;
    size_t b = 0;
    PR_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, b, key.ptr, key_sorted.ptr, c.ptr, c_sorted.ptr, m, 0, end_bit, s));
    DevBuf<uint8_t> tmp;
    PR_TRY(tmp.alloc(b + 16, s));
    PR_CUDA(cub::DeviceRadixSort::SortPairs(tmp.ptr, b, key.ptr, key_sorted.ptr, c.ptr, c_sorted.ptr, m, 0, end_bit, s));
    PR_TRY(ukey.alloc(m, s));
    PR_TRY(sums.alloc(m, s));
    PR_TRY(nruns.alloc(1, s));
    size_t b2 = 0;
    PR_CUDA(cub::DeviceReduce::ReduceByKey(nullptr, b2, key_sorted.ptr, ukey.ptr, c_sorted.ptr, sums.ptr, nruns.ptr,
                                           cub::Sum(), m, s));
    DevBuf<uint8_t> tmp2;
    PR_TRY(tmp2.alloc(b2 + 16, s));
    PR_CUDA(cub::DeviceReduce::ReduceByKey(tmp2.ptr, b2, key_sorted.ptr, ukey.ptr, c_sorted.ptr, sums.ptr, nruns.ptr,
                                           cub::Sum(), m, s));
    PR_CUDA(cudaMemcpyAsync(&u, nruns.ptr, 8, cudaMemcpyDeviceToHost, s));
    PR_CUDA(cudaStreamSynchronize(s));
  }
  unsigned int hbad = 0;
  PR_CUDA(cudaMemcpyAsync(&hbad, bad.ptr, 4, cudaMemcpyDeviceToHost, s));
  PR_CUDA(cudaStreamSynchronize(s));
  PR_ARG(!(hbad & 1u), "edge list holds patch ids outside [0, %lld)", (long long)n);
  csr.nnz = u;
  PR_TRY(csr.col.alloc(u, s));
  PR_TRY(csr.cnt.alloc(u, s));
  if (u > 0) {
    ::pr::launch_mark(), k_keys_to_csr<<<grid_for(u, 256), 256, 0, s>>>(ukey.ptr, sums.ptr, u, n, csr.col.ptr, csr.cnt.ptr, row_len.ptr,
                                                  bad.ptr);
    PR_CUDA(cudaGetLastError());
  }
  PR_TRY(len64.alloc(n > 0 ? n : 1, s));
  ::pr::launch_mark(), k_widen_scan_input<<<grid_for(n, 256), 256, 0, s>>>(row_len.ptr, len64.ptr, n);
  PR_TRY(lengths_to_row_ptr(len64.ptr, n, csr.row_ptr.ptr, s));
  PR_CUDA(cudaMemcpyAsync(&hbad, bad.ptr, 4, cudaMemcpyDeviceToHost, s));
  PR_CUDA(cudaStreamSynchronize(s));
  PR_ARG(!(hbad & 2u), "pooled counts must be non-negative and below 2^31");
  // rays per origin = row sums of the pooled counts (callers usually pass their own)
  PR_TRY(k->rays.alloc(n > 0 ? n : 1, s));
  ::pr::launch_mark(), k_row_sums<<<grid_for(n * 32, 256), 256, 0, s>>>(csr.row_ptr.ptr, csr.cnt.ptr, n, k->rays.ptr);
  PR_CUDA(cudaGetLastError());
  PR_CUDA(cudaStreamSynchronize(s));
  k->last_stream = s;
  *out = k.release();
  return PR_OK;
}

int counts_from_edges(const int32_t* origin, const int32_t* receiver, const int64_t* count, int64_t m, int64_t n,
                      cudaStream_t s, pr_counts** out) {
  return counts_from_tables(&origin, &receiver, &count, &m, 1, n, s, out);
}

__global__ void k_merge_len(const int64_t* __restrict__ ap, const int32_t* __restrict__ ac,
                            const int64_t* __restrict__ bp, const int32_t* __restrict__ bc, int64_t n,
                            int64_t* __restrict__ len);
__global__ void k_merge_rank(const int64_t* __restrict__ ap, const int32_t* __restrict__ ac,
                             const int32_t* __restrict__ an, const int64_t* __restrict__ bp,
                             const int32_t* __restrict__ bc, const int32_t* __restrict__ bn, int64_t n,
                             const int64_t* __restrict__ op, int32_t* __restrict__ oc, int32_t* __restrict__ on,
                             unsigned int* __restrict__ bad);
__global__ void k_add_i64(const int64_t* __restrict__ a, const int64_t* __restrict__ b, int64_t n,
                          int64_t* __restrict__ out);

// pool_counts of two device tables (view_factors.py:290-300): rows merged, counts and rays summed.
int counts_merge(const pr_counts* A, const pr_counts* B, cudaStream_t s, pr_counts** out) {
  const CountCsr& a = *A->csr;
  const CountCsr& b = *B->csr;
  PR_ARG(a.n_rows == b.n_rows, "count tables of %lld and %lld patches", (long long)a.n_rows, (long long)b.n_rows);
  const int64_t n = a.n_rows;
  std::unique_ptr<pr_counts> k(new pr_counts());
  cudaGetDevice(&k->device);
  k->csr = std::make_shared<CountCsr>();
  CountCsr& c = *k->csr;
  c.n_rows = n;
  PR_TRY(c.row_ptr.alloc(n + 1, s));
  DevBuf<int64_t> len;
  DevBuf<unsigned int> bad;
  PR_TRY(len.alloc(n > 0 ? n : 1, s));
  PR_TRY(bad.alloc(1, s));
  PR_CUDA(cudaMemsetAsync(bad.ptr, 0, 4, s));
  if (n > 0) {
    ::pr::launch_mark(), k_merge_len<<<grid_for(n * 32, 256), 256, 0, s>>>(a.row_ptr.ptr, a.col.ptr, b.row_ptr.ptr, b.col.ptr, n,
                                                                    len.ptr);
    PR_CUDA(cudaGetLastError());
  }
  PR_TRY(lengths_to_row_ptr(len.ptr, n, c.row_ptr.ptr, s));
  int64_t nnz = 0;
  PR_CUDA(cudaMemcpyAsync(&nnz, c.row_ptr.ptr + n, 8, cudaMemcpyDeviceToHost, s));
  PR_CUDA(cudaStreamSynchronize(s));
  c.nnz = nnz;
  PR_TRY(c.col.alloc(nnz, s));
  PR_TRY(c.cnt.alloc(nnz, s));
  PR_TRY(k->rays.alloc(n > 0 ? n : 1, s));
  if (n > 0) {
    ::pr::launch_mark(), k_merge_rank<<<grid_for(n * 32, 256), 256, 0, s>>>(a.row_ptr.ptr, a.col.ptr, a.cnt.ptr, b.row_ptr.ptr, b.col.ptr,
                                                  b.cnt.ptr, n, c.row_ptr.ptr, c.col.ptr, c.cnt.ptr, bad.ptr);
    PR_CUDA(cudaGetLastError());
    ::pr::launch_mark(), k_add_i64<<<grid_for(n, 256), 256, 0, s>>>(A->rays.ptr, B->rays.ptr, n, k->rays.ptr);
    PR_CUDA(cudaGetLastError());
  }
  unsigned int hb = 0;
  PR_CUDA(cudaMemcpyAsync(&hb, bad.ptr, 4, cudaMemcpyDeviceToHost, s));
  PR_CUDA(cudaStreamSynchronize(s));
  PR_ARG(!hb, "pooled counts exceed 2^31");
  k->rays_traced = A->rays_traced + B->rays_traced;
  k->dda_steps = A->dda_steps + B->dda_steps;
  k->last_stream = s;
  *out = k.release();
  return PR_OK;
}

// ------------------------------------------------------------------ transpose / symmetric pattern

// (row << 32 | count) of every entry of F, in row order
__global__ void k_row_count_values(const int64_t* __restrict__ row_ptr, const int32_t* __restrict__ cnt, int64_t n,
                                   unsigned long long* __restrict__ val) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t i = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); i < n; i += warps)
    for (int64_t q = row_ptr[i] + lane; q < row_ptr[i + 1]; q += 32)
      val[q] = ((unsigned long long)(uint32_t)i << 32) | (unsigned long long)(uint32_t)cnt[q];
}

__global__ void k_split_values(const unsigned long long* __restrict__ val, int64_t m, int32_t* __restrict__ col,
                               int32_t* __restrict__ cnt) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < m; t += (int64_t)gridDim.x * blockDim.x) {
    col[t] = (int32_t)(val[t] >> 32);
    cnt[t] = (int32_t)(val[t] & 0xffffffffull);
  }
}

// row_ptr[c] = first position of key c in the sorted keys (lower bound), c = 0..n
__global__ void k_row_ptr_from_sorted(const uint32_t* __restrict__ keys, int64_t m, int64_t n,
                                      int64_t* __restrict__ row_ptr) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c <= n; c += (int64_t)gridDim.x * blockDim.x) {
    int64_t lo = 0, hi = m;
    while (lo < hi) {
      const int64_t mid = (lo + hi) >> 1;
      if ((int64_t)keys[mid] < c) lo = mid + 1;
      else hi = mid;
    }
    row_ptr[c] = lo;
  }
}

// F^T by one stable radix sort of F's entries (already in row order) keyed on the column
// alone: equal columns keep their row order, so every row of F^T comes out sorted.
int build_transpose(const CountCsr& F, CountCsr& T, cudaStream_t s) {
  const int64_t n = F.n_rows, m = F.nnz;
  T.n_rows = n;
  T.nnz = m;
  PR_TRY(T.row_ptr.alloc(n + 1, s));
  PR_TRY(T.col.alloc(m > 0 ? m : 1, s));
  PR_TRY(T.cnt.alloc(m > 0 ? m : 1, s));
  if (m == 0) {
    PR_CUDA(cudaMemsetAsync(T.row_ptr.ptr, 0, (n + 1) * sizeof(int64_t), s));
    return PR_OK;
  }
  DevBuf<uint32_t> keys_out;
  DevBuf<unsigned long long> val, val_out;
  PR_TRY(keys_out.alloc(m, s));
  PR_TRY(val.alloc(m, s));
  PR_TRY(val_out.alloc(m, s));
  ::pr::launch_mark(), k_row_count_values<<<grid_for(n * 32, 256), 256, 0, s>>>(F.row_ptr.ptr, F.cnt.ptr, n, val.ptr);
  PR_CUDA(cudaGetLastError());
  int bits = 1;
  while (bits < 32 && ((int64_t)1 << bits) < n) ++bits;
  const uint32_t* keys_in = (const uint32_t*)F.col.ptr;
  size_t b = 0;
  PR_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, b, keys_in, keys_out.ptr, val.ptr, val_out.ptr, m, 0, bits, s));
  DevBuf<uint8_t> tmp;
  PR_TRY(tmp.alloc(b + 16, s));
  PR_CUDA(cub::DeviceRadixSort::SortPairs(tmp.ptr, b, keys_in, keys_out.ptr, val.ptr, val_out.ptr, m, 0, bits, s));
  ::pr::launch_mark(), k_split_values<<<grid_for(m, 256), 256, 0, s>>>(val_out.ptr, m, T.col.ptr, T.cnt.ptr);
  PR_CUDA(cudaGetLastError());
  ::pr::launch_mark(), k_row_ptr_from_sorted<<<grid_for(n + 1, 256), 256, 0, s>>>(keys_out.ptr, m, n, T.row_ptr.ptr);
  PR_CUDA(cudaGetLastError());
  return PR_OK;
}

// Row offsets of S: len_S(i) = len_F(i) + len_T(i).
__global__ void k_sym_row_ptr(const int64_t* __restrict__ fp, const int64_t* __restrict__ tp, int64_t n,
                              int64_t* __restrict__ sp) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i <= n; i += (int64_t)gridDim.x * blockDim.x)
    sp[i] = fp[i] + tp[i];
}

// Row i of S: the entries of row i of F (value 0.5 A_i n_ij / R_i) then those of row i of
// F^T (value 0.5 A_j n_ji / R_j); one warp per row, coalesced copies.
__global__ void k_sym_fill(const int64_t* __restrict__ fp, const int32_t* __restrict__ fc,
                           const int32_t* __restrict__ fn, const int64_t* __restrict__ tp,
                           const int32_t* __restrict__ tc, const int32_t* __restrict__ tn,
                           const int64_t* __restrict__ rays, const double* __restrict__ area, int64_t n,
                           const int64_t* __restrict__ sp, int mode, int bits, uint32_t* __restrict__ words,
                           int32_t* __restrict__ cnt, double* __restrict__ val) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t i = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); i < n; i += warps) {
    const int64_t o = sp[i], fb = fp[i], lf = fp[i + 1] - fb, tb = tp[i], lt = tp[i + 1] - tb;
    for (int64_t e = lane; e < lf + lt; e += 32) {
      const bool f = e < lf;
      const int64_t src = f ? fb + e : tb + (e - lf);
      const uint32_t col = (uint32_t)(f ? fc[src] : tc[src]);
      const int32_t c = f ? fn[src] : tn[src];
      if (mode == kPacked) {
        words[o + e] = (col << bits) | (uint32_t)c;
      } else {
        words[o + e] = col;
        if (mode == kCounts) {
          cnt[o + e] = c;
        } else {
          const int64_t owner = f ? i : (int64_t)col;
          val[o + e] = 0.5 * area[owner] * ((double)c / (double)rays[owner]);
        }
      }
    }
  }
}

__device__ __forceinline__ int64_t lower_bound_i32(const int32_t* __restrict__ a, int64_t lo, int64_t hi, int32_t x) {
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (a[mid] < x) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// |row i of A  union  row i of B| = |a| + |b| - |a intersect b|, one warp per row.
__global__ void k_merge_len(const int64_t* __restrict__ ap, const int32_t* __restrict__ ac,
                            const int64_t* __restrict__ bp, const int32_t* __restrict__ bc, int64_t n,
                            int64_t* __restrict__ len) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t i = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); i < n; i += warps) {
    const int64_t a0 = ap[i], a1 = ap[i + 1], b0 = bp[i], b1 = bp[i + 1];
    int dup = 0;
    for (int64_t k = a0 + lane; k < a1; k += 32) {
      const int64_t pb = lower_bound_i32(bc, b0, b1, ac[k]);
      dup += pb < b1 && bc[pb] == ac[k];
    }
    for (int o = 16; o > 0; o >>= 1) dup += __shfl_xor_sync(0xffffffffu, dup, o);
    if (lane == 0) len[i] = (a1 - a0) + (b1 - b0) - dup;
  }
}

// Pooled row i of A and B by ranking: an entry of A lands at k + #(b < a_k) - #(common < a_k),
// an entry of B absent from A at m + #(a < b_m) - #(common < b_m); a common column carries
// both counts.  The common-prefix counts come from warp ballots over tiles of 32.
__global__ void k_merge_rank(const int64_t* __restrict__ ap, const int32_t* __restrict__ ac,
                             const int32_t* __restrict__ an, const int64_t* __restrict__ bp,
                             const int32_t* __restrict__ bc, const int32_t* __restrict__ bn, int64_t n,
                             const int64_t* __restrict__ op, int32_t* __restrict__ oc, int32_t* __restrict__ on,
                             unsigned int* __restrict__ bad) {
  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t i = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); i < n; i += warps) {
    const int64_t a0 = ap[i], a1 = ap[i + 1], b0 = bp[i], b1 = bp[i + 1], o = op[i];
    int64_t carry = 0;
    for (int64_t base = 0; base < a1 - a0; base += 32) {
      const int64_t k = base + lane;
      const bool valid = k < a1 - a0;
      int32_t x = 0;
      int64_t pb = b0;
      bool match = false;
      if (valid) {
        x = ac[a0 + k];
        pb = lower_bound_i32(bc, b0, b1, x);
        match = pb < b1 && bc[pb] == x;
      }
      const unsigned m = __ballot_sync(0xffffffffu, valid && match);
      if (valid) {
        const int64_t pos = k + (pb - b0) - (carry + __popc(m & lt));
        const int64_t c = (int64_t)an[a0 + k] + (match ? (int64_t)bn[pb] : 0);
        if (c > INT32_MAX) atomicOr(bad, 1u);
        oc[o + pos] = x;
        on[o + pos] = (int32_t)c;
      }
      carry += __popc(m);
    }
    carry = 0;
    for (int64_t base = 0; base < b1 - b0; base += 32) {
      const int64_t k = base + lane;
      const bool valid = k < b1 - b0;
      int32_t y = 0;
      int64_t pa = a0;
      bool match = false;
      if (valid) {
        y = bc[b0 + k];
        pa = lower_bound_i32(ac, a0, a1, y);
        match = pa < a1 && ac[pa] == y;
      }
      const unsigned m = __ballot_sync(0xffffffffu, valid && match);
      if (valid && !match) {
        const int64_t pos = k + (pa - a0) - (carry + __popc(m & lt));
        oc[o + pos] = y;
        on[o + pos] = bn[b0 + k];
      }
      carry += __popc(m);
    }
  }
}

__global__ void k_add_i64(const int64_t* __restrict__ a, const int64_t* __restrict__ b, int64_t n,
                          int64_t* __restrict__ out) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
    out[t] = a[t] + b[t];
}

// Row sums of the counts must equal the rays of each origin (exchange.py:68-71).
__global__ void k_accounting(const int64_t* __restrict__ fp, const int32_t* __restrict__ fn,
                             const int64_t* __restrict__ rays, int64_t n, unsigned int* __restrict__ bad) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t i = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); i < n; i += warps) {
    int64_t s = 0;
    for (int64_t q = fp[i] + lane; q < fp[i + 1]; q += 32) s += fn[q];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(PR_FULL, s, o);
    if (lane == 0 && s != rays[i]) atomicOr(bad, 1u);
  }
}

// ------------------------------------------------------------------ balancing kernels

struct BalanceScalars {
  double max_f;      // max |f|
  double closure;    // max |d (S d) / A - 1|
  double bad;        // > 0 when S d is not finite and positive, or y left the log range
  double pad;
};

#define PR_LOG_MAX 709.782712893384  // log(DBL_MAX)
#define PR_LOG_MIN -744.4400719213812  // log(smallest subnormal)

__global__ void k_exp_scale(const double* __restrict__ y, int64_t n, double* __restrict__ d, double* __restrict__ sc) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double v = y[i];
    if (!(v < PR_LOG_MAX && v > PR_LOG_MIN)) sc[2] = 1.0;  // benign race: any writer sets the flag
    d[i] = exp(v);
  }
}

// One balancing evaluation at y (d = e^y given, the vector of the product):  s = S d;
// f_new = y + log s - log A;  dF = f_new - f_old (when dF != nullptr);  closure
// |d s / A - 1|;  max |f_new|.  In multiplicative mode (mult = 1), also
// y_next = y + 0.5 (log A - log(d s)).
struct BalanceEpi {
  double delta;
  const double* area;
  const double* y;
  const double* d;
  double* f;
  double* dF;
  double* sc;
  int mult;
  double* y_next;
  struct Red {
    double mf = 0.0, mc = 0.0;
    bool bad = false;
  };
  __device__ bool skip() const { return false; }
  __device__ void row(int64_t i, double sp, Red& r) const {
    const double Ai = area[i];
    const double s = sp + delta * Ai * d[i];
    if (!(s > 0.0 && isfinite(s))) r.bad = true;
    const double fn = y[i] + log(s) - log(Ai);
    if (dF) dF[i] = fn - f[i];
    f[i] = fn;
    const double rowv = d[i] * s;
    r.mf = fmax(r.mf, fabs(fn));
    r.mc = fmax(r.mc, fabs(rowv / Ai - 1.0));
    if (mult) y_next[i] = y[i] + 0.5 * (log(Ai) - log(rowv));
  }
  __device__ void finish(Red& r) const {
    for (int o = 16; o > 0; o >>= 1) {
      r.mf = fmax(r.mf, __shfl_xor_sync(PR_FULL, r.mf, o));
      r.mc = fmax(r.mc, __shfl_xor_sync(PR_FULL, r.mc, o));
    }
    const bool bad = __any_sync(PR_FULL, r.bad);
    if ((threadIdx.x & 31) == 0) {
      atomic_max_nonneg(sc + 0, r.mf);
      atomic_max_nonneg(sc + 1, r.mc);
      if (bad) sc[2] = 1.0;
    }
  }
};

// y_next = y - beta f - sum_c gamma_c (dY_c - beta dF_c);  dY_slot = y_next - y.
struct AAStep {
  double gamma[10];
  int cols;
  int slot;  // ring slot receiving the new differences
  double beta;
};

__global__ void k_aa_update(AAStep st, const double* __restrict__ y, const double* __restrict__ f,
                            const double* __restrict__ dY, const double* __restrict__ dF, int64_t n,
                            double* __restrict__ y_next, double* __restrict__ dY_out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double v = y[i] - st.beta * f[i];
    for (int c = 0; c < st.cols; ++c) v -= st.gamma[c] * (dY[(int64_t)c * n + i] - st.beta * dF[(int64_t)c * n + i]);
    dY_out[(int64_t)st.slot * n + i] = v - y[i];
    y_next[i] = v;
  }
}

// Dots of the history: row r of the Gram matrix (dF_r . dF_c, c < cols) and the
// right-hand side (dF_c . f, c < cols) -> partial[block][2 * 10].
__global__ void __launch_bounds__(256) k_aa_dots(const double* __restrict__ dF, const double* __restrict__ f,
                                                 int64_t n, int cols, int r, double* __restrict__ partial) {
  double acc[20];
#pragma unroll
  for (int k = 0; k < 20; ++k) acc[k] = 0.0;
  const double* vr = dF + (int64_t)r * n;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double a = vr[i], fi = f[i];
#pragma unroll
    for (int c = 0; c < 10; ++c) {
      if (c < cols) {
        const double v = dF[(int64_t)c * n + i];
        acc[c] = fma(a, v, acc[c]);
        acc[10 + c] = fma(v, fi, acc[10 + c]);
      }
    }
  }
  block_sum_store<20>(acc, partial);
}

// ------------------------------------------------------------------ products

// y = S v (mode 0), (d / A) S v with v = d x (mode 1), d S v with v = d (x / A) (mode 2).
struct ApplyEpi {
  double delta;
  const double* area;
  const double* d;
  const double* v;
  int mode;
  double* y;
  struct Red {};
  __device__ bool skip() const { return false; }
  __device__ void row(int64_t i, double sp, Red&) const {
    const double s = sp + delta * area[i] * v[i];
    y[i] = mode == 0 ? s : (mode == 1 ? (d[i] / area[i]) * s : d[i] * s);
  }
  __device__ void finish(Red&) const {}
};

__global__ void k_prep_u(const double* __restrict__ d, const double* __restrict__ area, const double* __restrict__ x,
                         int64_t n, int mode, double* __restrict__ u) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    u[i] = mode == 1 ? d[i] * x[i] : d[i] * (x[i] / area[i]);
}

// F x (transposed = 0) or F^T x (transposed = 1, given the transposed CSR) with w = n / R of the origin.
__global__ void __launch_bounds__(256) k_raw_apply(const int64_t* __restrict__ rp, const int32_t* __restrict__ cl,
                                                   const int32_t* __restrict__ cn, const int64_t* __restrict__ rays,
                                                   int64_t n, int transposed, const double* __restrict__ x,
                                                   double* __restrict__ y) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t i = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); i < n; i += warps) {
    double acc = 0.0;
    for (int64_t q = rp[i] + lane; q < rp[i + 1]; q += 32) {
      const int32_t j = cl[q];
      const double w = (double)cn[q] / (double)rays[transposed ? j : i];
      acc = fma(w, x[j], acc);
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(PR_FULL, acc, o);
    if (lane == 0) y[i] = acc;
  }
}

// Reciprocity defect over the sampled pairs (exchange.py:124-140).
__global__ void __launch_bounds__(256) k_reciprocity(const int64_t* __restrict__ fp, const int32_t* __restrict__ fc,
                                                     const int32_t* __restrict__ fn, const int64_t* __restrict__ rays,
                                                     const double* __restrict__ area, const double* __restrict__ d,
                                                     double delta, int64_t n, double* __restrict__ out) {
  double mdiff = 0.0, mjoint = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    for (int64_t q = fp[i]; q < fp[i + 1]; ++q) {
      const int32_t j = fc[q];
      const double w = (double)fn[q] / (double)rays[i];
      // n_ji by binary search in row j
      int64_t lo = fp[j], hi = fp[j + 1];
      while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (fc[mid] < i) lo = mid + 1;
        else hi = mid;
      }
      const double wr = (lo < fp[j + 1] && fc[lo] == (int32_t)i) ? (double)fn[lo] / (double)rays[j] : 0.0;
      const double Ai = area[i], Aj = area[j];
      double sij = 0.5 * (Ai * w + Aj * wr);
      double sji = 0.5 * (Aj * wr + Ai * w);
      if (j == (int32_t)i) {
        sij += delta * Ai;
        sji += delta * Aj;
      }
      const double jij = Ai * ((d[i] / Ai) * sij * d[j]);
      const double jji = Aj * ((d[j] / Aj) * sji * d[i]);
      mdiff = fmax(mdiff, fabs(jij - jji));
      mjoint = fmax(mjoint, fabs(jij));
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    mdiff = fmax(mdiff, __shfl_xor_sync(PR_FULL, mdiff, o));
    mjoint = fmax(mjoint, __shfl_xor_sync(PR_FULL, mjoint, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomic_max_nonneg(out + 0, mdiff);
    atomic_max_nonneg(out + 1, mjoint);
  }
}

__global__ void k_edges_out(const int64_t* __restrict__ fp, const int32_t* __restrict__ fn,
                            const int64_t* __restrict__ rays, int64_t n, int32_t* __restrict__ origin,
                            double* __restrict__ weight) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t i = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); i < n; i += warps) {
    for (int64_t q = fp[i] + lane; q < fp[i + 1]; q += 32) {
      if (origin) origin[q] = (int32_t)i;
      if (weight) weight[q] = (double)fn[q] / (double)rays[i];
    }
  }
}

// ------------------------------------------------------------------ host side

static int spmv_grid(int64_t rows) { return grid_for(rows * 32, 256, sm_count() * 8); }


// Symmetric eigen-decomposition (cyclic Jacobi) of a k x k matrix, k <= 10.
static void jacobi_eig(int k, double* a, double* v, double* w) {
  for (int i = 0; i < k; ++i)
    for (int j = 0; j < k; ++j) v[i * k + j] = i == j ? 1.0 : 0.0;
  for (int sweep = 0; sweep < 64; ++sweep) {
    double off = 0.0;
    for (int i = 0; i < k; ++i)
      for (int j = i + 1; j < k; ++j) off += a[i * k + j] * a[i * k + j];
    if (off < 1e-300) break;
    for (int p = 0; p < k; ++p)
      for (int q = p + 1; q < k; ++q) {
        const double apq = a[p * k + q];
        if (apq == 0.0) continue;
        const double theta = (a[q * k + q] - a[p * k + p]) / (2.0 * apq);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
        const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
        for (int r = 0; r < k; ++r) {
          const double arp = a[r * k + p], arq = a[r * k + q];
          a[r * k + p] = c * arp - s * arq;
          a[r * k + q] = s * arp + c * arq;
        }
        for (int r = 0; r < k; ++r) {
          const double apr = a[p * k + r], aqr = a[q * k + r];
          a[p * k + r] = c * apr - s * aqr;
          a[q * k + r] = s * apr + c * aqr;
        }
        for (int r = 0; r < k; ++r) {
          const double vrp = v[r * k + p], vrq = v[r * k + q];
          v[r * k + p] = c * vrp - s * vrq;
          v[r * k + q] = s * vrp + c * vrq;
        }
      }
  }
  for (int i = 0; i < k; ++i) w[i] = a[i * k + i];
}

// Least-squares gamma = pinv(H) b for the k x k Gram matrix H.
static void solve_gram(int k, const double* H, const double* b, double* gamma) {
  double a[100], v[100], w[10];
  for (int i = 0; i < k * k; ++i) a[i] = H[i];
  jacobi_eig(k, a, v, w);
  double wmax = 0.0;
  for (int i = 0; i < k; ++i) wmax = fmax(wmax, fabs(w[i]));
  const double cut = 10.0 * 2.220446049250313e-16 * wmax;
  for (int i = 0; i < k; ++i) gamma[i] = 0.0;
  for (int e = 0; e < k; ++e) {
    if (!(fabs(w[e]) > cut)) continue;
    double proj = 0.0;
    for (int i = 0; i < k; ++i) proj += v[i * k + e] * b[i];
    proj /= w[e];
    for (int i = 0; i < k; ++i) gamma[i] += v[i * k + e] * proj;
  }
}

struct BalanceWork {
  int64_t n;
  DevBuf<double> y, y2, d, f, dY, dF, sc, partial, dots;
};

static int balance_eval(pr_operator* op, BalanceWork& w, const double* y, double* dF, int mult, double* y_next,
                        BalanceScalars* out, cudaStream_t s) {
  const int64_t n = w.n;
  PR_CUDA(cudaMemsetAsync(w.sc.ptr, 0, 4 * sizeof(double), s));
  ::pr::launch_mark(), k_exp_scale<<<grid_for(n, 256), 256, 0, s>>>(y, n, w.d.ptr, w.sc.ptr);
  const BalanceEpi epi{op->delta, op->area.ptr, y, w.d.ptr, w.f.ptr, dF, w.sc.ptr, mult, y_next};
  int st = PR_OK;
  ::pr::timer_begin(kTimerBalance, s);
  dispatch_mode(op->S.mode, [&](auto u) { st = launch_spmv<decltype(u)::value, double>(op->S, w.d.ptr, epi, s); });
  ::pr::timer_end(kTimerBalance, s);
  PR_TRY(st);
  op->spmv_calls++;
  PR_CUDA(cudaMemcpyAsync(out, w.sc.ptr, sizeof(BalanceScalars), cudaMemcpyDeviceToHost, s));
  return PR_OK;
}

static int balance_multiplicative(pr_operator* op, BalanceWork& w, double tol, cudaStream_t s);

static int balance_work(BalanceWork& w, int64_t n, cudaStream_t s) {
  const int M = 10;
  w.n = n;
  PR_TRY(w.y.alloc(n, s));
  PR_TRY(w.y2.alloc(n, s));
  PR_TRY(w.d.alloc(n, s));
  PR_TRY(w.f.alloc(n, s));
  PR_TRY(w.dY.alloc((size_t)M * n, s));
  PR_TRY(w.dF.alloc((size_t)M * n, s));
  PR_TRY(w.sc.alloc(4, s));
  PR_TRY(w.partial.alloc((size_t)red_grid() * 20, s));
  PR_TRY(w.dots.alloc(20, s));
  PR_CUDA(cudaMemsetAsync(w.y.ptr, 0, n * sizeof(double), s));
  return PR_OK;
}

static int balance(pr_operator* op, double tol, cudaStream_t s) {
  const int64_t n = op->n;
  const int M = 10;
  const double beta = 0.5;
  BalanceWork w;
  PR_TRY(balance_work(w, n, s));
  const int rg = red_grid();
  BalanceScalars sc;
  PR_TRY(balance_eval(op, w, w.y.ptr, nullptr, 0, nullptr, &sc, s));
  PR_CUDA(cudaStreamSynchronize(s));
  const double eps = 2.220446049250313e-16;
  if (!(sc.bad > 0) && sc.closure <= tol) {  // exchange.py:157-159
    op->method = PR_BALANCE_NONE;
    op->iterations = 0;
    PR_CUDA(cudaMemcpyAsync(op->scale.ptr, w.d.ptr, n * 8, cudaMemcpyDeviceToDevice, s));
    return PR_OK;
  }
  // ---- Anderson acceleration
  bool aa_ok = false;
  int iters = 0;
  if (!(sc.bad > 0)) {
    // History columns live in ring slots 0..cols-1; G and b are indexed by slot.
    double G[10][10] = {{0}}, b[10] = {0};
    int cols = 0, oldest = 0;
    double* y = w.y.ptr;
    double* y_next = w.y2.ptr;
    double max_f = sc.max_f;
    const int maxit = 500;  // scipy.optimize.anderson maxiter of exchange.py:177
    for (int it = 0; it < maxit && max_f > tol; ++it) {
      AAStep st;
      st.cols = cols;
      st.beta = beta;
      double gamma[10] = {0};
      if (cols > 0) {
        double Hf[100];
        for (int i = 0; i < cols; ++i)
          for (int j = 0; j < cols; ++j) Hf[i * cols + j] = G[i][j];
        solve_gram(cols, Hf, b, gamma);
      }
      for (int c = 0; c < 10; ++c) st.gamma[c] = c < cols ? gamma[c] : 0.0;
      int slot;
      if (cols < M) {
        slot = cols;
      } else {
        slot = oldest;
        oldest = (oldest + 1) % M;
      }
      st.slot = slot;
      ::pr::launch_mark(), k_aa_update<<<grid_for(n, 256), 256, 0, s>>>(st, y, w.f.ptr, w.dY.ptr, w.dF.ptr, n, y_next, w.dY.ptr);
      PR_CUDA(cudaGetLastError());
      PR_TRY(balance_eval(op, w, y_next, w.dF.ptr + (size_t)slot * n, 0, nullptr, &sc, s));
      ++iters;
      std::swap(y, y_next);
      if (cols < M) ++cols;
      ::pr::launch_mark(), k_aa_dots<<<rg, 256, 0, s>>>(w.dF.ptr, w.f.ptr, n, cols, slot, w.partial.ptr);
      PR_CUDA(cudaGetLastError());
      PR_TRY(sum_partials(w.partial.ptr, rg, 20, w.dots.ptr, s));
      double hd[20];
      PR_CUDA(cudaMemcpyAsync(hd, w.dots.ptr, sizeof(hd), cudaMemcpyDeviceToHost, s));
      PR_CUDA(cudaStreamSynchronize(s));
      if (sc.bad > 0 || !std::isfinite(sc.max_f)) break;
      for (int c = 0; c < cols; ++c) {
        G[slot][c] = hd[c];
        G[c][slot] = hd[c];
        b[c] = hd[10 + c];
      }
      max_f = sc.max_f;
    }
    if (y != w.y.ptr) PR_CUDA(cudaMemcpyAsync(w.y.ptr, y, n * 8, cudaMemcpyDeviceToDevice, s));
    const double accept = fmin(fmax(10.0 * tol, 10.0 * eps), 1.0e-10);  // exchange.py:180
    if (!(sc.bad > 0) && max_f <= tol && sc.closure <= accept) {
      aa_ok = true;
      // d = exp(y) is in w.d from the last evaluation
      PR_CUDA(cudaMemcpyAsync(op->scale.ptr, w.d.ptr, n * 8, cudaMemcpyDeviceToDevice, s));
      op->method = PR_BALANCE_ANDERSON;
      op->iterations = iters;
    }
  }
  if (aa_ok) return PR_OK;
  return balance_multiplicative(op, w, tol, s);
}

// Damped multiplicative iteration from y = 0 (exchange.py:185-196): the fallback when Anderson
// acceleration does not reach the acceptance tolerance.
static int balance_multiplicative(pr_operator* op, BalanceWork& w, double tol, cudaStream_t s) {
  const int64_t n = op->n;
  BalanceScalars sc;
  PR_CUDA(cudaMemsetAsync(w.y.ptr, 0, n * sizeof(double), s));
  double* y = w.y.ptr;
  double* y_next = w.y2.ptr;
  PR_TRY(balance_eval(op, w, y, nullptr, 1, y_next, &sc, s));
  PR_CUDA(cudaStreamSynchronize(s));
  for (int it = 1; it <= 20000; ++it) {
    if (sc.bad > 0) break;
    std::swap(y, y_next);
    // closure at the updated y, and the next multiplicative step from the same product
    PR_TRY(balance_eval(op, w, y, nullptr, 1, y_next, &sc, s));
    PR_CUDA(cudaStreamSynchronize(s));
    if (sc.bad > 0 || !std::isfinite(sc.closure)) break;
    if (sc.closure <= fmin(tol, 1.0e-10)) {
      PR_CUDA(cudaMemcpyAsync(op->scale.ptr, w.d.ptr, n * 8, cudaMemcpyDeviceToDevice, s));
      op->method = PR_BALANCE_MULTIPLICATIVE;
      op->iterations = it;
      return PR_OK;
    }
  }
  set_error("diagonal balancing of the exchange matrix did not converge");
  return PR_ERR_BALANCE;
}

// Anderson balancing of several operators in lockstep (the iteration of balance(), operator by
// operator the same steps): every iteration makes one product of each operator still iterating,
// all in one launch of the batched blocked product, and takes one host round trip for all of
// them.  A sweep of many small operators then fills the GPU with one grid per iteration instead
// of one operator's grid per stream.  Operators that Anderson does not settle fall back to the
// multiplicative iteration one at a time, as in balance().  Every operator must be blocked and of
// storage mode kMode.
template <int kMode>
static int balance_batch(const std::vector<pr_operator*>& ops, double tol, cudaStream_t s) {
  const int m = (int)ops.size();
  if (m == 0) return PR_OK;
  const int M = 10;
  const double beta = 0.5, eps = 2.220446049250313e-16;
  const double accept = fmin(fmax(10.0 * tol, 10.0 * eps), 1.0e-10);  // exchange.py:180
  struct State {
    BalanceWork w;
    double G[10][10] = {{0}}, b[10] = {0};
    int cols = 0, oldest = 0, iters = 0, slot = 0;
    double* y = nullptr;
    double* y_next = nullptr;
    bool active = false, done = false;
    BalanceScalars sc{};
    double dots[20] = {0};
  };
  std::vector<State> st(m);
  for (int k = 0; k < m; ++k) {
    PR_TRY(balance_work(st[k].w, ops[k]->n, s));
    st[k].y = st[k].w.y.ptr;
    st[k].y_next = st[k].w.y2.ptr;
  }
  DevBuf<BlkItem<double, BalanceEpi>> items;
  PR_TRY(items.alloc(m, s));
  // one product of each listed operator at y[k] (differences into dF_out[k] when given)
  auto products = [&](const std::vector<int>& which, const std::vector<double*>& ys,
                      const std::vector<double*>& dF_out) -> int {
    std::vector<const SymCsr*> mats;
    std::vector<const double*> xs;
    std::vector<BalanceEpi> epis;
    for (size_t j = 0; j < which.size(); ++j) {
      pr_operator* op = ops[which[j]];
      BalanceWork& w = st[which[j]].w;
      PR_CUDA(cudaMemsetAsync(w.sc.ptr, 0, 4 * sizeof(double), s));
      ::pr::launch_mark(), k_exp_scale<<<grid_for(op->n, 256), 256, 0, s>>>(ys[j], op->n, w.d.ptr, w.sc.ptr);
      mats.push_back(&op->S);
      xs.push_back(w.d.ptr);
      epis.push_back(BalanceEpi{op->delta, op->area.ptr, ys[j], w.d.ptr, w.f.ptr, dF_out[j], w.sc.ptr, 0, nullptr});
      op->spmv_calls++;
    }
    PR_CUDA(cudaGetLastError());
    ::pr::timer_begin(kTimerBalance, s);
    const int rc = launch_spmv_batch<kMode, double>(mats, xs, epis, items.ptr, s);
    ::pr::timer_end(kTimerBalance, s);
    PR_TRY(rc);
    for (int k : which) PR_CUDA(cudaMemcpyAsync(&st[k].sc, st[k].w.sc.ptr, sizeof(BalanceScalars),
                                                cudaMemcpyDeviceToHost, s));
    return PR_OK;
  };
  // y = 0 for every operator
  {
    std::vector<int> all(m);
    std::vector<double*> ys(m), none(m, nullptr);
    for (int k = 0; k < m; ++k) {
      all[k] = k;
      ys[k] = st[k].y;
    }
    PR_TRY(products(all, ys, none));
    PR_CUDA(cudaStreamSynchronize(s));
  }
  for (int k = 0; k < m; ++k) {
    pr_operator* op = ops[k];
    if (!(st[k].sc.bad > 0) && st[k].sc.closure <= tol) {  // exchange.py:157-159
      op->method = PR_BALANCE_NONE;
      op->iterations = 0;
      PR_CUDA(cudaMemcpyAsync(op->scale.ptr, st[k].w.d.ptr, op->n * 8, cudaMemcpyDeviceToDevice, s));
      st[k].done = true;
    } else {
      st[k].active = !(st[k].sc.bad > 0) && st[k].sc.max_f > tol;
    }
  }
  const int rg = red_grid();
  for (int it = 0; it < 500; ++it) {  // scipy.optimize.anderson maxiter of exchange.py:177
    std::vector<int> which;
    std::vector<double*> ys, dFs;
    for (int k = 0; k < m; ++k) {
      State& q = st[k];
      if (!q.active) continue;
      const int64_t n = ops[k]->n;
      AAStep step;
      step.cols = q.cols;
      step.beta = beta;
      double gamma[10] = {0};
      if (q.cols > 0) {
        double Hf[100];
        for (int i = 0; i < q.cols; ++i)
          for (int j = 0; j < q.cols; ++j) Hf[i * q.cols + j] = q.G[i][j];
        solve_gram(q.cols, Hf, q.b, gamma);
      }
      for (int c = 0; c < 10; ++c) step.gamma[c] = c < q.cols ? gamma[c] : 0.0;
      if (q.cols < M) {
        q.slot = q.cols;
      } else {
        q.slot = q.oldest;
        q.oldest = (q.oldest + 1) % M;
      }
      step.slot = q.slot;
      ::pr::launch_mark(), k_aa_update<<<grid_for(n, 256), 256, 0, s>>>(step, q.y, q.w.f.ptr, q.w.dY.ptr, q.w.dF.ptr, n,
                                                                      q.y_next, q.w.dY.ptr);
      which.push_back(k);
      ys.push_back(q.y_next);
      dFs.push_back(q.w.dF.ptr + (size_t)q.slot * n);
    }
    if (which.empty()) break;
    PR_CUDA(cudaGetLastError());
    PR_TRY(products(which, ys, dFs));
    for (int k : which) {
      State& q = st[k];
      ++q.iters;
      std::swap(q.y, q.y_next);
      if (q.cols < M) ++q.cols;
      ::pr::launch_mark(), k_aa_dots<<<rg, 256, 0, s>>>(q.w.dF.ptr, q.w.f.ptr, ops[k]->n, q.cols, q.slot,
                                                        q.w.partial.ptr);
      PR_TRY(sum_partials(q.w.partial.ptr, rg, 20, q.w.dots.ptr, s));
      PR_CUDA(cudaMemcpyAsync(q.dots, q.w.dots.ptr, sizeof(q.dots), cudaMemcpyDeviceToHost, s));
    }
    PR_CUDA(cudaGetLastError());
    PR_CUDA(cudaStreamSynchronize(s));
    for (int k : which) {
      State& q = st[k];
      if (q.sc.bad > 0 || !std::isfinite(q.sc.max_f)) {
        q.active = false;
        continue;
      }
      for (int c = 0; c < q.cols; ++c) {
        q.G[q.slot][c] = q.dots[c];
        q.G[c][q.slot] = q.dots[c];
        q.b[c] = q.dots[10 + c];
      }
      if (q.sc.max_f <= tol) q.active = false;
    }
  }
  for (int k = 0; k < m; ++k) {
    State& q = st[k];
    if (q.done) continue;
    pr_operator* op = ops[k];
    if (q.y != q.w.y.ptr) PR_CUDA(cudaMemcpyAsync(q.w.y.ptr, q.y, op->n * 8, cudaMemcpyDeviceToDevice, s));
    if (!(q.sc.bad > 0) && q.sc.max_f <= tol && q.sc.closure <= accept) {
      PR_CUDA(cudaMemcpyAsync(op->scale.ptr, q.w.d.ptr, op->n * 8, cudaMemcpyDeviceToDevice, s));
      op->method = PR_BALANCE_ANDERSON;
      op->iterations = q.iters;
    } else {
      PR_TRY(balance_multiplicative(op, q.w, tol, s));
    }
  }
  return PR_OK;
}

static bool all_equal_i64(const std::vector<int64_t>& v) {
  for (size_t i = 1; i < v.size(); ++i)
    if (v[i] != v[0]) return false;
  return true;
}
static bool all_equal_f64(const std::vector<double>& v) {
  for (size_t i = 1; i < v.size(); ++i)
    if (v[i] != v[0]) return false;
  return true;
}

__global__ void k_pack_words(uint32_t* __restrict__ words, const int32_t* __restrict__ cnt, int64_t m, int bits) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < m; t += (int64_t)gridDim.x * blockDim.x)
    words[t] = (words[t] << bits) | (uint32_t)cnt[t];
}

// S' on the union of the patterns of F and F^T with the pair counts n_ij + n_ji (ranked
// row merge), packed into 32-bit words when the bits fit.
static int sym_union(const CountCsr& F, const CountCsr& T, pr_operator* op, cudaStream_t s) {
  SymCsr& S = op->S;
  const int64_t n = F.n_rows;
  DevBuf<int64_t> len;
  DevBuf<unsigned int> bad;
  PR_TRY(len.alloc(n, s));
  PR_TRY(bad.alloc(1, s));
  PR_CUDA(cudaMemsetAsync(bad.ptr, 0, 4, s));
  ::pr::launch_mark(), k_merge_len<<<grid_for(n * 32, 256), 256, 0, s>>>(F.row_ptr.ptr, F.col.ptr, T.row_ptr.ptr,
                                                                         T.col.ptr, n, len.ptr);
  PR_CUDA(cudaGetLastError());
  PR_TRY(lengths_to_row_ptr(len.ptr, n, S.row_ptr.ptr, s));
  int64_t nnz = 0;
  PR_CUDA(cudaMemcpyAsync(&nnz, S.row_ptr.ptr + n, 8, cudaMemcpyDeviceToHost, s));
  PR_CUDA(cudaStreamSynchronize(s));
  S.nnz = nnz;
  // padded to a whole 16-byte quad: the blocked products read the entries four at a time
  PR_TRY(S.words.alloc((size_t)(nnz + 4) / 4 * 4, s));
  PR_TRY(S.cnt.alloc((size_t)(nnz + 4) / 4 * 4, s));
  ::pr::launch_mark(), k_merge_rank<<<grid_for(n * 32, 256), 256, 0, s>>>(
      F.row_ptr.ptr, F.col.ptr, F.cnt.ptr, T.row_ptr.ptr, T.col.ptr, T.cnt.ptr, n, S.row_ptr.ptr,
      (int32_t*)S.words.ptr, S.cnt.ptr, bad.ptr);
  PR_CUDA(cudaGetLastError());
  if (S.mode == kPacked && nnz > 0) {
    ::pr::launch_mark(), k_pack_words<<<grid_for(nnz, 256), 256, 0, s>>>(S.words.ptr, S.cnt.ptr, nnz, S.bits);
    PR_CUDA(cudaGetLastError());
    S.cnt.release();
  }
  unsigned int hb = 0;
  PR_CUDA(cudaMemcpyAsync(&hb, bad.ptr, 4, cudaMemcpyDeviceToHost, s));
  PR_CUDA(cudaStreamSynchronize(s));
  PR_ARG(!hb, "pair counts exceed 2^31");
  return PR_OK;
}

// CTA row boundaries of a blocked product: boundary c is the first row r whose cost
// row_ptr[r] + r nnz / n reaches c / C of the total, so a CTA holds about 2 nnz / C
// entries plus rows, and fewer than 2 n / C + 1 rows.
__global__ void k_cta_rows(const int64_t* __restrict__ rp, int64_t n, int ctas, int64_t* __restrict__ out) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c > ctas) return;
  if (c == 0 || c == ctas) {
    out[c] = c == 0 ? 0 : n;
    return;
  }
  const double avg = (double)rp[n] / (double)n;
  const double target = (double)c * (2.0 * (double)rp[n] / (double)ctas);
  int64_t lo = 0, hi = n;
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if ((double)rp[mid] + (double)mid * avg < target) lo = mid + 1;
    else hi = mid;
  }
  out[c] = lo;
}

// seg[(b - 1) n + i] = first entry of row i with column >= b W, relative to row_ptr[i]
// (b = 1 .. nb - 1); the words of a row ascend with the column in both union modes.
__global__ void k_block_seg(const int64_t* __restrict__ rp, const uint32_t* __restrict__ words, int64_t n, int nb,
                            int W, int bits, int32_t* __restrict__ seg) {
  const int64_t total = n * (int64_t)(nb - 1);
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = t % n;
    const int b = (int)(t / n) + 1;
    const uint32_t key = (uint32_t)((uint64_t)b * (uint64_t)W) << bits;
    int64_t lo = rp[i], hi = rp[i + 1];
    const int64_t base = lo;
    while (lo < hi) {
      const int64_t mid = (lo + hi) >> 1;
      if (words[mid] < key) lo = mid + 1;
      else hi = mid;
    }
    seg[(int64_t)(b - 1) * n + i] = (int32_t)(lo - base);
  }
}

// Column blocks for the shared-memory products of a union-stored S'.
static int build_col_blocks(SymCsr& S, cudaStream_t s) {
  ColBlocks& B = S.blk;
  B.ready = false;
  const int64_t n = S.n_rows;
  if (n == 0 || S.mode == kValues) return PR_OK;
  const int64_t kRowsCap = 6144;  // binary64 row sums of one CTA: 48 KB of shared memory
  int64_t ctas = std::max<int64_t>(sm_count(), (2 * n + kRowsCap - 1) / kRowsCap);
  if (ctas > n) ctas = std::max<int64_t>(1, n);
  PR_TRY(B.cta_row.alloc(ctas + 1, s));
  ::pr::launch_mark(), k_cta_rows<<<grid_for(ctas + 1, 256), 256, 0, s>>>(S.row_ptr.ptr, n, (int)ctas, B.cta_row.ptr);
  PR_CUDA(cudaGetLastError());
  std::vector<int64_t> h(ctas + 1);
  PR_CUDA(cudaMemcpyAsync(h.data(), B.cta_row.ptr, (ctas + 1) * 8, cudaMemcpyDeviceToHost, s));
  PR_CUDA(cudaStreamSynchronize(s));
  int64_t rows_cap = 1;
  for (int64_t c = 0; c < ctas; ++c) rows_cap = std::max(rows_cap, h[c + 1] - h[c]);
  const int64_t stage_bytes = (int64_t)kBlkSmemMax - rows_cap * 8;
  const int64_t W = stage_bytes / 8 / 64 * 64;
  if (W < 1024) return PR_OK;  // rows too many for one CTA's row sums: warp-per-row products
  B.W = (int)std::min<int64_t>(W, (n + 63) / 64 * 64);
  B.nb = (int)((n + B.W - 1) / B.W);
  B.ctas = (int)ctas;
  B.rows_cap = (int)rows_cap;
  if (B.nb > 1) {
    PR_TRY(B.seg.alloc((size_t)(B.nb - 1) * n, s));
    ::pr::launch_mark(), k_block_seg<<<grid_for(n * (B.nb - 1), 256), 256, 0, s>>>(
        S.row_ptr.ptr, S.words.ptr, n, B.nb, B.W, S.mode == kPacked ? S.bits : 0, B.seg.ptr);
    PR_CUDA(cudaGetLastError());
  }
  B.ready = true;
  return PR_OK;
}

int apply(const pr_operator* op, int which, const double* x_dev, double* y_dev, cudaStream_t s);

// Everything of operator_create before the balancing: accounting, transpose, S', column blocks.
static int operator_assemble(const pr_counts* k, const int64_t* rays, const double* area, double delta,
                             cudaStream_t s, std::unique_ptr<pr_operator>& op) {
  const int64_t n = k->csr->n_rows;
  op.reset(new pr_operator());
  cudaGetDevice(&op->device);
  op->n = n;
  op->F = k->csr;
  op->delta = delta;
  op->last_stream = s;
  PR_TRY(op->rays.alloc(n > 0 ? n : 1, s));
  PR_TRY(op->area.alloc(n > 0 ? n : 1, s));
  PR_TRY(op->scale.alloc(n > 0 ? n : 1, s));
  std::vector<int64_t> h_rays(n);
  std::vector<double> h_area(n);
  if (n > 0) {
    PR_CUDA(cudaMemcpyAsync(h_rays.data(), rays, n * 8, cudaMemcpyDefault, s));
    PR_CUDA(cudaMemcpyAsync(h_area.data(), area, n * 8, cudaMemcpyDefault, s));
    PR_CUDA(cudaStreamSynchronize(s));
    PR_CUDA(cudaMemcpyAsync(op->rays.ptr, h_rays.data(), n * 8, cudaMemcpyHostToDevice, s));
    PR_CUDA(cudaMemcpyAsync(op->area.ptr, h_area.data(), n * 8, cudaMemcpyHostToDevice, s));
  }
  const CountCsr& F = *op->F;
  // accounting (exchange.py:68-71)
  {
    DevBuf<unsigned int> bad;
    PR_TRY(bad.alloc(1, s));
    PR_CUDA(cudaMemsetAsync(bad.ptr, 0, 4, s));
    ::pr::launch_mark(), k_accounting<<<spmv_grid(n), 256, 0, s>>>(F.row_ptr.ptr, F.cnt.ptr, op->rays.ptr, n, bad.ptr);
    PR_CUDA(cudaGetLastError());
    unsigned int hb = 0;
    PR_CUDA(cudaMemcpyAsync(&hb, bad.ptr, 4, cudaMemcpyDeviceToHost, s));
    PR_CUDA(cudaStreamSynchronize(s));
    if (hb) {
      set_error("first-hit counts do not account for every emitted ray");
      return PR_ERR_ACCOUNTING;
    }
  }
  // symmetric matrix: row i = row i of F followed by row i of F^T
  {
    auto T = std::make_shared<CountCsr>();
    PR_TRY(build_transpose(F, *T, s));
    SymCsr& S = op->S;
    S.n_rows = n;
    PR_TRY(S.row_ptr.alloc(n + 1, s));
    const bool uniform = n > 0 && all_equal_i64(h_rays) && all_equal_f64(h_area) && h_rays[0] > 0;
    int64_t max_rays = 0;
    for (int64_t r : h_rays) max_rays = std::max(max_rays, r);
    int cb = 1, kb = 1;
    while (cb < 32 && ((int64_t)1 << cb) < n) ++cb;
    while (kb < 32 && ((int64_t)1 << kb) <= 2 * max_rays) ++kb;  // pair sums n_ij + n_ji <= 2 R
    if (uniform) {
      S.factor = 0.5 * h_area[0] / (double)h_rays[0];
      S.mode = cb + kb <= 32 ? kPacked : kCounts;
      S.bits = S.mode == kPacked ? kb : 0;
    } else {
      S.mode = kValues;
      S.nnz = F.nnz + T->nnz;
      PR_TRY(S.words.alloc(S.nnz > 0 ? S.nnz : 1, s));
      PR_TRY(S.val.alloc(S.nnz > 0 ? S.nnz : 1, s));
    }
    if (n > 0 && S.mode == kValues) {
      ::pr::launch_mark(), k_sym_row_ptr<<<grid_for(n + 1, 256), 256, 0, s>>>(F.row_ptr.ptr, T->row_ptr.ptr, n,
                                                                              S.row_ptr.ptr);
      PR_CUDA(cudaGetLastError());
      ::pr::launch_mark(), k_sym_fill<<<grid_for(n * 32, 256), 256, 0, s>>>(
          F.row_ptr.ptr, F.col.ptr, F.cnt.ptr, T->row_ptr.ptr, T->col.ptr, T->cnt.ptr, op->rays.ptr, op->area.ptr, n,
          S.row_ptr.ptr, S.mode, S.bits, S.words.ptr, S.cnt.ptr, S.val.ptr);
      PR_CUDA(cudaGetLastError());
    } else if (n > 0) {
      // equal areas and ray counts: S'_ij = factor (n_ij + n_ji) on the union of the patterns
      PR_TRY(sym_union(F, *T, op.get(), s));
      PR_TRY(build_col_blocks(op->S, s));
    }
    op->FT = T;  // kept for raw_rmatvec
  }
  return PR_OK;
}

// Row closure of F_p (exchange.py:78-80) after the balancing.
static int operator_closure(pr_operator* op, cudaStream_t s) {
  const int64_t n = op->n;
  if (n > 0) {
    DevBuf<double> ones, r;
    PR_TRY(ones.alloc(n, s));
    PR_TRY(r.alloc(n, s));
    std::vector<double> h1(n, 1.0);
    PR_CUDA(cudaMemcpyAsync(ones.ptr, h1.data(), n * 8, cudaMemcpyHostToDevice, s));
    PR_TRY(apply(op, PR_APPLY_MATVEC, ones.ptr, r.ptr, s));
    std::vector<double> hr(n);
    PR_CUDA(cudaMemcpyAsync(hr.data(), r.ptr, n * 8, cudaMemcpyDeviceToHost, s));
    PR_CUDA(cudaStreamSynchronize(s));
    double e = 0.0;
    for (int64_t i = 0; i < n; ++i) e = fmax(e, fabs(hr[i] - 1.0));
    op->row_sum_error = e;
    if (!(e <= 1.0e-10)) {
      set_error("projected rows do not close: %.3e", e);
      return PR_ERR_NOT_CLOSED;
    }
  }
  PR_CUDA(cudaStreamSynchronize(s));
  return PR_OK;
}

int operator_create(const pr_counts* k, const int64_t* rays, const double* area, double delta, double tol,
                    cudaStream_t s, pr_operator** out) {
  std::unique_ptr<pr_operator> op;
  PR_TRY(operator_assemble(k, rays, area, delta, s, op));
  if (op->n > 0) PR_TRY(balance(op.get(), tol, s));
  PR_TRY(operator_closure(op.get(), s));
  *out = op.release();
  return PR_OK;
}

// Several operators at once: each assembled as operator_create does, then the blocked operators
// of each storage mode balanced together (balance_batch), the others one at a time; out[k] is
// set only when every operator succeeds.
int operators_create_batch(const pr_counts* const* counts, const int64_t* const* rays, const double* const* area,
                           int n_ops, double delta, double tol, cudaStream_t s, pr_operator** out) {
  std::vector<std::unique_ptr<pr_operator>> ops(n_ops);
  for (int k = 0; k < n_ops; ++k) PR_TRY(operator_assemble(counts[k], rays[k], area[k], delta, s, ops[k]));
  std::vector<pr_operator*> packed, counted;
  for (int k = 0; k < n_ops; ++k) {
    pr_operator* op = ops[k].get();
    if (op->n == 0) continue;
    if (op->S.blk.ready && op->S.mode == kPacked) packed.push_back(op);
    else if (op->S.blk.ready && op->S.mode == kCounts) counted.push_back(op);
    else PR_TRY(balance(op, tol, s));
  }
  PR_TRY(balance_batch<kPacked>(packed, tol, s));
  PR_TRY(balance_batch<kCounts>(counted, tol, s));
  for (int k = 0; k < n_ops; ++k) PR_TRY(operator_closure(ops[k].get(), s));
  for (int k = 0; k < n_ops; ++k) out[k] = ops[k].release();
  return PR_OK;
}

// y = product(x) with x, y device vectors of length n.
int apply(const pr_operator* op, int which, const double* x, double* y, cudaStream_t s) {
  const int64_t n = op->n;
  if (n == 0) return PR_OK;
  const CountCsr& F = *op->F;
  if (which == PR_APPLY_RAW || which == PR_APPLY_RAW_T) {
    const CountCsr& M = which == PR_APPLY_RAW ? F : *op->FT;
    ::pr::launch_mark(), k_raw_apply<<<spmv_grid(n), 256, 0, s>>>(M.row_ptr.ptr, M.col.ptr, M.cnt.ptr, op->rays.ptr, n,
                                             which == PR_APPLY_RAW_T, x, y);
    PR_CUDA(cudaGetLastError());
    return PR_OK;
  }
  int mode = which == PR_APPLY_SYM ? 0 : (which == PR_APPLY_MATVEC ? 1 : 2);
  PR_ARG(which >= 0 && which <= PR_APPLY_RMATVEC, "unknown product %d", which);
  DevBuf<double> u;
  if (mode != 0) {
    PR_TRY(u.alloc(n, s));
    ::pr::launch_mark(), k_prep_u<<<grid_for(n, 256), 256, 0, s>>>(op->scale.ptr, op->area.ptr, x, n, mode, u.ptr);
    PR_CUDA(cudaGetLastError());
  }
  const double* v = mode == 0 ? x : u.ptr;
  const ApplyEpi epi{op->delta, op->area.ptr, op->scale.ptr, v, mode, y};
  int st = PR_OK;
  dispatch_mode(op->S.mode, [&](auto un) { st = launch_spmv<decltype(un)::value, double>(op->S, v, epi, s); });
  PR_TRY(st);
  op->spmv_calls++;
  return PR_OK;
}

int reciprocity_error(const pr_operator* op, double* out, cudaStream_t s) {
  const int64_t n = op->n;
  DevBuf<double> r;
  PR_TRY(r.alloc(2, s));
  PR_CUDA(cudaMemsetAsync(r.ptr, 0, 16, s));
  const CountCsr& F = *op->F;
  if (n > 0) {
    ::pr::launch_mark(), k_reciprocity<<<grid_for(n, 256), 256, 0, s>>>(F.row_ptr.ptr, F.col.ptr, F.cnt.ptr, op->rays.ptr, op->area.ptr,
                                                  op->scale.ptr, op->delta, n, r.ptr);
    PR_CUDA(cudaGetLastError());
  }
  double h[2];
  PR_CUDA(cudaMemcpyAsync(h, r.ptr, 16, cudaMemcpyDeviceToHost, s));
  PR_CUDA(cudaStreamSynchronize(s));
  const double tiny = 2.2250738585072014e-308;
  *out = h[0] / fmax(h[1], tiny);
  return PR_OK;
}

int operator_edges(const pr_operator* op, int32_t* origin, int32_t* receiver, double* weight, cudaStream_t s) {
  const CountCsr& F = *op->F;
  const int64_t m = F.nnz, n = op->n;
  if (m == 0) return PR_OK;
  DevBuf<int32_t> o;
  DevBuf<double> w;
  if (origin) PR_TRY(o.alloc(m, s));
  if (weight) PR_TRY(w.alloc(m, s));
  ::pr::launch_mark(), k_edges_out<<<spmv_grid(n), 256, 0, s>>>(F.row_ptr.ptr, F.cnt.ptr, op->rays.ptr, n, origin ? o.ptr : nullptr,
                                           weight ? w.ptr : nullptr);
  PR_CUDA(cudaGetLastError());
  if (origin) PR_CUDA(cudaMemcpyAsync(origin, o.ptr, m * 4, cudaMemcpyDefault, s));
  if (receiver) PR_CUDA(cudaMemcpyAsync(receiver, F.col.ptr, m * 4, cudaMemcpyDefault, s));
  if (weight) PR_CUDA(cudaMemcpyAsync(weight, w.ptr, m * 8, cudaMemcpyDefault, s));
  PR_CUDA(cudaStreamSynchronize(s));
  return PR_OK;
}

}  // namespace pr
