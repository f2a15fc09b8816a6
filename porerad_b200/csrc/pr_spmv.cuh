// Sparse products over the symmetric exchange matrix and deterministic reductions.
//
// S x = S' x + delta A x, S' = 0.5 (A F + F^T A) (porerad/exchange.py:108-112), row i
// stored as row i of F followed by row i of F^T.  One warp owns one row: lanes stride
// over the row's entries (coalesced 32-bit word loads, gathers of x from L2) and the
// partial sums meet in a fixed shuffle tree, so every product is bitwise reproducible.
#pragma once
#include <type_traits>

#include "pr_objects.cuh"

namespace pr {

#define PR_FULL 0xffffffffu

struct SymView {
  const int64_t* __restrict__ row_ptr;
  const uint32_t* __restrict__ words;
  const int32_t* __restrict__ cnt;
  const double* __restrict__ val;
  uint32_t mask;  // count mask of packed words
  int bits;
  double factor;
  int64_t n;
};

inline SymView sym_view(const SymCsr& S) {
  SymView v;
  v.row_ptr = S.row_ptr.ptr;
  v.words = S.words.ptr;
  v.cnt = S.cnt.ptr;
  v.val = S.val.ptr;
  v.bits = S.bits;
  v.mask = S.bits > 0 && S.bits < 32 ? ((1u << S.bits) - 1u) : 0xffffffffu;
  v.factor = S.factor;
  v.n = S.n_rows;
  return v;
}

// sum_j S'_ij x_j in binary64, the full sum on every lane of the warp.
template <int kMode, typename Tx>
__device__ __forceinline__ double sym_row(const SymView& S, int64_t i, const Tx* __restrict__ x, int lane) {
  const int64_t b = S.row_ptr[i], e = S.row_ptr[i + 1];
  double acc = 0.0;
  for (int64_t q = b + lane; q < e; q += 32) {
    const uint32_t w = __ldg(S.words + q);
    if constexpr (kMode == kPacked) {
      acc = fma((double)(w & S.mask), (double)__ldg(x + (w >> S.bits)), acc);
    } else if constexpr (kMode == kCounts) {
      acc = fma((double)__ldg(S.cnt + q), (double)__ldg(x + w), acc);
    } else {
      acc = fma(__ldg(S.val + q), (double)__ldg(x + w), acc);
    }
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(PR_FULL, acc, o);
  return kMode == kValues ? acc : acc * S.factor;
}

// The same sum in binary32 (mixed-precision sweeps).
template <int kMode>
__device__ __forceinline__ float sym_row32(const SymView& S, int64_t i, const float* __restrict__ x, int lane) {
  const int64_t b = S.row_ptr[i], e = S.row_ptr[i + 1];
  float acc = 0.0f;
  for (int64_t q = b + lane; q < e; q += 32) {
    const uint32_t w = __ldg(S.words + q);
    if constexpr (kMode == kPacked) {
      acc = fmaf((float)(w & S.mask), __ldg(x + (w >> S.bits)), acc);
    } else if constexpr (kMode == kCounts) {
      acc = fmaf((float)__ldg(S.cnt + q), __ldg(x + w), acc);
    } else {
      acc = fmaf((float)__ldg(S.val + q), __ldg(x + w), acc);
    }
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(PR_FULL, acc, o);
  return kMode == kValues ? acc : acc * (float)S.factor;
}

// Calls fn(std::integral_constant<int, mode>) for the matrix's storage mode.
template <typename Fn>
inline void dispatch_mode(int mode, Fn&& fn) {
  if (mode == kPacked) fn(std::integral_constant<int, kPacked>());
  else if (mode == kCounts) fn(std::integral_constant<int, kCounts>());
  else fn(std::integral_constant<int, kValues>());
}

// atomic max of a non-negative double (bit patterns of non-negative doubles order as integers)
__device__ __forceinline__ void atomic_max_nonneg(double* addr, double v) {
  if (!(v >= 0.0)) v = __longlong_as_double(0x7ff0000000000000ll);  // NaN -> +inf
  atomicMax((unsigned long long*)addr, (unsigned long long)__double_as_longlong(v));
}

// Block-wide sum of K values per thread into partial[slot * K + k] (fixed tree);
// slot defaults to the block index.
template <int K>
__device__ __forceinline__ void block_sum_store(double (&v)[K], double* __restrict__ partial, int64_t slot = -1) {
  __shared__ double red[32][K];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int k = 0; k < K; ++k)
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(PR_FULL, v[k], o);
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < K; ++k) red[wid][k] = v[k];
  __syncthreads();
  if (threadIdx.x < K) {
    double s = 0.0;
    for (int w = 0; w < nw; ++w) s += red[w][threadIdx.x];
    partial[(slot < 0 ? (int64_t)blockIdx.x : slot) * K + threadIdx.x] = s;
  }
  __syncthreads();
}

// out[k] = sum over blocks of partial[b * K + k], in block order (one thread per k).
__global__ void k_sum_partials(const double* __restrict__ partial, int blocks, int K, double* __restrict__ out);

int sum_partials(const double* partial, int blocks, int K, double* out, cudaStream_t s);

}  // namespace pr
