// Sparse products over the symmetric exchange matrix and deterministic reductions.
//
// S x = S' x + delta A x, S' = 0.5 (A F + F^T A) (porerad/exchange.py:108-112).  A product
// is one kernel: the row sums of S' x followed by a per-row epilogue (the update of the
// solver that consumes the product) and block reductions in a fixed order, so every
// result is bitwise reproducible for a given operator.  Two row-sum schemes:
//  * warp per row (k_spmv_rows): lanes stride over the row's entries (coalesced 32-bit
//    word loads, gathers of x through L1/L2), partial sums meet in a fixed shuffle tree;
//  * column-blocked (k_spmv_blk, union storage only): x is staged in shared memory one
//    block of columns at a time, so the random gathers become shared-memory loads; each
//    row's sum accumulates block by block in shared memory.
#pragma once
#include <algorithm>
#include <mutex>
#include <vector>
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

// Coefficient and column of entry q (storage mode kMode).
template <int kMode, typename Acc>
__device__ __forceinline__ void sym_entry(const SymView& S, int64_t q, Acc& c, uint32_t& col) {
  const uint32_t w = __ldg(S.words + q);
  if constexpr (kMode == kPacked) {
    c = (Acc)(w & S.mask);
    col = w >> S.bits;
  } else if constexpr (kMode == kCounts) {
    c = (Acc)__ldg(S.cnt + q);
    col = w;
  } else {
    c = (Acc)__ldg(S.val + q);
    col = w;
  }
}

// sum_j S'_ij x_j in precision Acc, the full sum on every lane of the warp.  Lane l adds
// entries b + l, b + l + 32, ... in that order; four of them are loaded before the first
// is added, so four word loads and four gathers are in flight per lane (the order of the
// additions, and so the result, does not depend on the unrolling).
template <int kMode, typename Acc, typename Tx>
__device__ __forceinline__ Acc sym_row_acc(const SymView& S, int64_t i, const Tx* __restrict__ x, int lane) {
  const int64_t b = S.row_ptr[i], e = S.row_ptr[i + 1];
  Acc acc = 0;
  int64_t q = b + lane;
  for (; q + 96 < e; q += 128) {
    Acc c0, c1, c2, c3;
    uint32_t j0, j1, j2, j3;
    sym_entry<kMode>(S, q, c0, j0);
    sym_entry<kMode>(S, q + 32, c1, j1);
    sym_entry<kMode>(S, q + 64, c2, j2);
    sym_entry<kMode>(S, q + 96, c3, j3);
    const Acc x0 = (Acc)__ldg(x + j0), x1 = (Acc)__ldg(x + j1), x2 = (Acc)__ldg(x + j2), x3 = (Acc)__ldg(x + j3);
    acc = fma(c0, x0, acc);
    acc = fma(c1, x1, acc);
    acc = fma(c2, x2, acc);
    acc = fma(c3, x3, acc);
  }
  for (; q < e; q += 32) {
    Acc c;
    uint32_t j;
    sym_entry<kMode>(S, q, c, j);
    acc = fma(c, (Acc)__ldg(x + j), acc);
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(PR_FULL, acc, o);
  return kMode == kValues ? acc : acc * (Acc)S.factor;
}

// sum_j S'_ij x_j in binary64.
template <int kMode, typename Tx>
__device__ __forceinline__ double sym_row(const SymView& S, int64_t i, const Tx* __restrict__ x, int lane) {
  return sym_row_acc<kMode, double>(S, i, x, lane);
}

// The same sum in binary32 (mixed-precision sweeps).
template <int kMode>
__device__ __forceinline__ float sym_row32(const SymView& S, int64_t i, const float* __restrict__ x, int lane) {
  return sym_row_acc<kMode, float>(S, i, x, lane);
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

// Sum of a[b * stride + off] over b < count by one warp in a fixed order: lane l adds b = l,
// l + 32, ... in turn, then the lanes meet in a fixed shuffle tree; every lane gets the sum.
__device__ __forceinline__ double warp_sum_partials(const double* __restrict__ a, int count, int stride, int off,
                                                    int lane) {
  double s = 0.0;
  for (int b = lane; b < count; b += 32) s += a[(int64_t)b * stride + off];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(PR_FULL, s, o);
  return s;
}

// out[k] = sum over blocks of partial[b * K + k] (one warp per k, warp_sum_partials order).
__global__ void k_sum_partials(const double* __restrict__ partial, int blocks, int K, double* __restrict__ out);

int sum_partials(const double* partial, int blocks, int K, double* out, cudaStream_t s);


// ------------------------------------------------------------------ generic products

struct BlkView {
  const int32_t* __restrict__ seg;
  const int64_t* __restrict__ cta_row;
  int W, nb;
};

inline BlkView blk_view(const SymCsr& S) { return BlkView{S.blk.seg.ptr, S.blk.cta_row.ptr, S.blk.W, S.blk.nb}; }

// Entries 0..3 of one 16-byte quad of the word array (and of the count array in kCounts mode):
// entry e is summed when lo <= e < hi (the quad's part of the row segment), adding
// coefficient * x[col] to acc in entry order.  xs0 points at x[0] of the staged block's
// coordinates (the shared array shifted back by the block's first column), so x[col] is xs0[col].
// kWhole: the quad lies inside the segment (lo <= 0, hi >= 4), so no entry is tested.
template <int kMode, bool kWhole, typename Acc, typename Tx>
__device__ __forceinline__ void quad_add(const SymView& S, const uint4& w, const int4& c, int lo, int hi,
                                         const Tx* xs0, Acc& acc) {
  const uint32_t ws[4] = {w.x, w.y, w.z, w.w};
  const int32_t cs[4] = {c.x, c.y, c.z, c.w};
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    if (kWhole || (e >= lo && e < hi)) {
      Acc coef;
      uint32_t col;
      if constexpr (kMode == kPacked) {
        coef = (Acc)(ws[e] & S.mask);
        col = ws[e] >> S.bits;
      } else {
        coef = (Acc)cs[e];
        col = ws[e];
      }
      acc = fma(coef, (Acc)xs0[col], acc);
    }
  }
}

// V quads of a group lane, k, k + G, ..., k + (V - 1) G (all below the segment's quad count):
// the loads first, then the entries in quad order.  Only the segment's first and last quads
// are partial, so the per-entry tests run on those alone.
template <int kMode, int G, int V, typename Acc, typename Tx>
__device__ __forceinline__ void seg_quads(const SymView& S, const uint4* __restrict__ w4, const int4* __restrict__ c4,
                                          int k, int lo0, int hi0, const Tx* xs0, Acc& acc) {
  uint4 w[V];
  int4 c[V];
#pragma unroll
  for (int u = 0; u < V; ++u) {
    w[u] = __ldg(w4 + k + u * G);
    c[u] = make_int4(0, 0, 0, 0);
    if constexpr (kMode == kCounts) c[u] = __ldg(c4 + k + u * G);
  }
#pragma unroll
  for (int u = 0; u < V; ++u) {
    const int q = 4 * (k + u * G);  // the quad's first entry, counted from quad 0
    const int lo = lo0 - q, hi = hi0 - q;
    if (lo <= 0 && hi >= 4) quad_add<kMode, true>(S, w[u], c[u], lo, hi, xs0, acc);
    else quad_add<kMode, false>(S, w[u], c[u], lo, hi, xs0, acc);
  }
}

// sum over entries [qb, qe) of a row of coefficient * x[col] (x staged in shared memory, xs0 as
// in quad_add) by a group of G lanes (gl = lane within the group).  The group reads whole
// aligned 16-byte quads of the word array (entries 4a .. 4a + 3 of quad a), from the quad
// holding qb to the one holding qe - 1: lane gl takes quads gl, gl + G, ... of the segment and
// adds the entries of each quad that lie in [qb, qe) in quad order.  Loads go out U quads per
// lane at a time while every lane of the group has U quads left, then two, then one, so no
// lane issues work for quads past the segment.  Indices relative to the segment are 32-bit (a
// segment lies within one column block).  The group's partials meet in a fixed shuffle tree
// (every lane of the warp takes part; lanes of an idle group, qb = qe, add zero).  Reads stay
// inside the word array, padded to a whole quad.
template <int kMode, int G, typename Acc, typename Tx>
__device__ __forceinline__ Acc seg_sum(const SymView& S, int64_t qb, int64_t qe, const Tx* xs0, int gl) {
  constexpr int U = kMode == kCounts ? 2 : 4;  // counts mode loads a second quad per entry quad
  Acc acc = 0;
  if (qe > qb) {
    const int64_t a0 = qb >> 2;
    const int nq = (int)(((qe + 3) >> 2) - a0);  // quads of the segment
    const int lo0 = (int)(qb - 4 * a0);          // first entry of quad 0 in the segment (0..3)
    const int hi0 = (int)(qe - 4 * a0);          // end of the segment, counted from quad 0
    const uint4* __restrict__ w4 = reinterpret_cast<const uint4*>(S.words) + a0;
    const int4* __restrict__ c4 = reinterpret_cast<const int4*>(S.cnt) + a0;
    int k = gl;
    for (; k + (U - 1) * G < nq; k += U * G) seg_quads<kMode, G, U>(S, w4, c4, k, lo0, hi0, xs0, acc);
    if constexpr (U > 2) {
      if (k + G < nq) {
        seg_quads<kMode, G, 2>(S, w4, c4, k, lo0, hi0, xs0, acc);
        k += 2 * G;
      }
    }
    for (; k < nq; k += G) seg_quads<kMode, G, 1>(S, w4, c4, k, lo0, hi0, xs0, acc);
  }
  for (int o = G / 2; o > 0; o >>= 1) acc += __shfl_xor_sync(PR_FULL, acc, o);
  return acc;
}

// An epilogue Epi provides: a Red type of per-thread reduction state (value-initialised),
// bool skip() (the whole product is skipped, e.g. a converged solve), row(i, s, red) with
// s = (S' x)_i, and finish(red), called by every thread of the block once its rows are done.

template <int kMode, typename Acc, typename Tx, class Epi>
__global__ void __launch_bounds__(256) k_spmv_rows(SymView S, const Tx* __restrict__ x, Epi epi) {
  if (epi.skip()) return;
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  typename Epi::Red red{};
  for (int64_t i = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); i < S.n; i += warps) {
    const Acc sum = sym_row_acc<kMode, Acc>(S, i, x, lane);
    if (lane == 0) epi.row(i, sum, red);
  }
  epi.finish(red);
}

constexpr int kBlkThreads = 1024;
constexpr int kBlkSmemMax = 220 * 1024;  // dynamic shared memory of a blocked product

// Stage g covers column blocks [g k, g k + k) (k = 2 for binary32 x, whose blocks are
// half as many bytes), staged with 16-byte loads; groups of G = 8 lanes then take the CTA's
// rows (4 rows in flight per warp: a row's segment of one stage is short).  Eight lanes per
// segment measured faster than four for binary64 x and than sixteen for binary32 x on the
// c2 operators.
// The work of CTA `cta` of a blocked product (its row range B.cta_row[cta] .. B.cta_row[cta + 1]).
template <int kMode, typename Acc, typename Tx, class Epi>
__device__ __forceinline__ void spmv_blk_cta(const SymView& S, const BlkView& B, const Tx* __restrict__ x,
                                             const Epi& epi, int cta) {
  extern __shared__ __align__(16) unsigned char blk_smem[];
  constexpr int k = sizeof(Tx) == 4 ? 2 : 1;
  const int stage_cols = B.W * k;
  Tx* xs = reinterpret_cast<Tx*>(blk_smem);
  Acc* acc = reinterpret_cast<Acc*>(blk_smem + (size_t)stage_cols * sizeof(Tx));
  constexpr int G = 8;  // lanes per row segment
  constexpr int kGroups = 32 / G;
  const int64_t r0 = B.cta_row[cta], r1 = B.cta_row[cta + 1];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int grp = lane / G, gl = lane % G;
  const int stages = (B.nb + k - 1) / k;
  for (int g = 0; g < stages; ++g) {
    const int64_t c0 = (int64_t)g * stage_cols;
    const int64_t cw = min((int64_t)stage_cols, S.n - c0);
    {
      // 16-byte loads when x + c0 is 16-byte aligned (W is a multiple of 64, so only the
      // base of x decides), element loads otherwise
      const int64_t vec = ((uintptr_t)(x + c0) & 15u) ? 0 : cw * (int64_t)sizeof(Tx) / 16;
      const int4* src = reinterpret_cast<const int4*>(x + c0);
      int4* dst = reinterpret_cast<int4*>(xs);
      for (int64_t t = threadIdx.x; t < vec; t += blockDim.x) dst[t] = __ldg(src + t);
      for (int64_t t = vec * 16 / (int64_t)sizeof(Tx) + threadIdx.x; t < cw; t += blockDim.x) xs[t] = __ldg(x + c0 + t);
    }
    __syncthreads();
    const int b0 = g * k, b1 = min(B.nb, b0 + k);
    // entries [qb, qe) of row i in this stage's column blocks (empty past the CTA's rows)
    auto bounds = [&](int64_t i, int64_t& qb, int64_t& qe) {
      qb = qe = 0;
      if (i < r1) {
        const int64_t rb = S.row_ptr[i];
        qb = b0 == 0 ? rb : rb + B.seg[(int64_t)(b0 - 1) * S.n + i];
        qe = b1 == B.nb ? S.row_ptr[i + 1] : rb + B.seg[(int64_t)(b1 - 1) * S.n + i];
      }
    };
    // The group's leader asks L2 for a row segment two iterations before the group sums it, so
    // the sums read L2 instead of waiting on DRAM (a bulk prefetch of the segment's 16-byte
    // quads; the entry arrays are padded to whole quads).
    auto prefetch = [&](int64_t qb, int64_t qe) {
      if (gl != 0 || qe <= qb) return;
      const int64_t a0 = (qb >> 2) << 4, a1 = ((qe + 3) >> 2) << 4;  // byte range of the quads
      asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"((const char*)S.words + a0),
                   "r"((unsigned)(a1 - a0))
                   : "memory");
      if constexpr (kMode == kCounts)
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"((const char*)S.cnt + a0),
                     "r"((unsigned)(a1 - a0))
                     : "memory");
    };
    const int64_t stride = (int64_t)nwarps * kGroups;
    int64_t i = r0 + (int64_t)warp * kGroups + grp;  // warp-uniform loop over base = i - grp
    int64_t qb0, qe0, qb1, qe1;
    bounds(i, qb0, qe0);
    bounds(i + stride, qb1, qe1);
    prefetch(qb0, qe0);
    prefetch(qb1, qe1);
    for (; i - grp < r1; i += stride) {
      int64_t qb2, qe2;
      bounds(i + 2 * stride, qb2, qe2);
      const Acc part = seg_sum<kMode, G, Acc>(S, qb0, qe0, xs - c0, gl);
      if (gl == 0 && i < r1) acc[i - r0] = g == 0 ? part : acc[i - r0] + part;
      prefetch(qb2, qe2);
      qb0 = qb1;
      qe0 = qe1;
      qb1 = qb2;
      qe1 = qe2;
    }
    __syncthreads();
  }
  typename Epi::Red red{};
  for (int64_t i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
    const Acc a = acc[i - r0];
    epi.row(i, kMode == kValues ? a : a * (Acc)S.factor, red);
  }
  epi.finish(red);
}

template <int kMode, typename Acc, typename Tx, class Epi>
__global__ void __launch_bounds__(kBlkThreads, 1) k_spmv_blk(SymView S, BlkView B, const Tx* __restrict__ x, Epi epi) {
  if (epi.skip()) return;
  spmv_blk_cta<kMode, Acc>(S, B, x, epi, blockIdx.x);
}

// One product of each of several operators in one launch: item k owns the CTAs
// [cta_begin_k, cta_begin_{k+1}) of the grid.  The epilogue must not index per-block storage by
// blockIdx (BalanceEpi reduces with atomics only).
template <typename Tx, class Epi>
struct BlkItem {
  SymView S;
  BlkView B;
  const Tx* x;
  Epi epi;
  int cta_begin;
};

template <int kMode, typename Acc, typename Tx, class Epi>
__global__ void __launch_bounds__(kBlkThreads, 1) k_spmv_blk_batch(const BlkItem<Tx, Epi>* __restrict__ items,
                                                                   int n_items) {
  int lo = 0, hi = n_items - 1;  // the last item whose first CTA is at or before this one
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (items[mid].cta_begin <= (int)blockIdx.x) lo = mid;
    else hi = mid - 1;
  }
  const BlkItem<Tx, Epi> it = items[lo];
  if (it.epi.skip()) return;
  spmv_blk_cta<kMode, Acc>(it.S, it.B, it.x, it.epi, (int)blockIdx.x - it.cta_begin);
}

template <int kMode, typename Acc, typename Tx, class Epi>
inline int allow_blk_smem() {
  static std::mutex mu;
  static bool done[64] = {};
  int dev = 0;
  PR_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  if (dev >= 0 && dev < 64 && done[dev]) return PR_OK;
  PR_CUDA(cudaFuncSetAttribute(k_spmv_blk<kMode, Acc, Tx, Epi>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               kBlkSmemMax));
  if (dev >= 0 && dev < 64) done[dev] = true;
  return PR_OK;
}

// Blocks of a product of S (the number of partial-sum slots its block reductions fill).
inline int spmv_slots(const SymCsr& S) {
  if (S.blk.ready) return S.blk.ctas;
  return grid_for(S.n_rows * 32, 256, sm_count() * 8);
}

// One product of S with x (device vector of n entries) and the epilogue epi.
template <int kMode, typename Acc, typename Tx, class Epi>
inline int launch_spmv(const SymCsr& S, const Tx* x, const Epi& epi, cudaStream_t s) {
  const SymView v = sym_view(S);
  if (S.blk.ready && kMode != kValues) {
    constexpr int k = sizeof(Tx) == 4 ? 2 : 1;
    if (((uintptr_t)S.words.ptr & 15u) || (kMode == kCounts && ((uintptr_t)S.cnt.ptr & 15u))) {
      set_error("blocked product: the entry arrays are not 16-byte aligned");
      return PR_ERR_CUDA;
    }
    const size_t smem = (size_t)S.blk.W * k * sizeof(Tx) + (size_t)S.blk.rows_cap * sizeof(Acc);
    if (smem > (size_t)kBlkSmemMax) {
      set_error("blocked product needs %zu bytes of shared memory", smem);
      return PR_ERR_LIMIT;
    }
    PR_TRY((allow_blk_smem<kMode, Acc, Tx, Epi>()));
    ::pr::launch_mark(), k_spmv_blk<kMode, Acc, Tx, Epi><<<S.blk.ctas, kBlkThreads, smem, s>>>(v, blk_view(S), x, epi);
  } else {
    ::pr::launch_mark(), k_spmv_rows<kMode, Acc, Tx, Epi><<<spmv_slots(S), 256, 0, s>>>(v, x, epi);
  }
  PR_CUDA(cudaGetLastError());
  return PR_OK;
}

template <int kMode, typename Acc, typename Tx, class Epi>
inline int allow_blk_batch_smem() {
  static std::mutex mu;
  static bool done[64] = {};
  int dev = 0;
  PR_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  if (dev >= 0 && dev < 64 && done[dev]) return PR_OK;
  PR_CUDA(cudaFuncSetAttribute(k_spmv_blk_batch<kMode, Acc, Tx, Epi>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               kBlkSmemMax));
  if (dev >= 0 && dev < 64) done[dev] = true;
  return PR_OK;
}

// One product of each of the operators mats[k] (blocked, storage mode kMode) with xs[k] and
// epilogue epis[k], all in one launch.  items is device scratch for mats.size() items.
template <int kMode, typename Acc, typename Tx, class Epi>
inline int launch_spmv_batch(const std::vector<const SymCsr*>& mats, const std::vector<const Tx*>& xs,
                             const std::vector<Epi>& epis, BlkItem<Tx, Epi>* items, cudaStream_t s) {
  const int n = (int)mats.size();
  if (n == 0) return PR_OK;
  constexpr int k = sizeof(Tx) == 4 ? 2 : 1;
  std::vector<BlkItem<Tx, Epi>> h(n);
  size_t smem = 0;
  int ctas = 0;
  for (int i = 0; i < n; ++i) {
    const SymCsr& S = *mats[i];
    if (!S.blk.ready || S.mode != kMode) {
      set_error("batched product: operator %d is not a blocked operator of the batch's storage mode", i);
      return PR_ERR_ARG;
    }
    if (((uintptr_t)S.words.ptr & 15u) || (kMode == kCounts && ((uintptr_t)S.cnt.ptr & 15u))) {
      set_error("blocked product: the entry arrays are not 16-byte aligned");
      return PR_ERR_CUDA;
    }
    h[i] = BlkItem<Tx, Epi>{sym_view(S), blk_view(S), xs[i], epis[i], ctas};
    ctas += S.blk.ctas;
    smem = std::max(smem, (size_t)S.blk.W * k * sizeof(Tx) + (size_t)S.blk.rows_cap * sizeof(Acc));
  }
  if (smem > (size_t)kBlkSmemMax) {
    set_error("blocked product needs %zu bytes of shared memory", smem);
    return PR_ERR_LIMIT;
  }
  PR_TRY((allow_blk_batch_smem<kMode, Acc, Tx, Epi>()));
  PR_CUDA(cudaMemcpyAsync(items, h.data(), sizeof(BlkItem<Tx, Epi>) * n, cudaMemcpyHostToDevice, s));
  ::pr::launch_mark(), k_spmv_blk_batch<kMode, Acc, Tx, Epi><<<ctas, kBlkThreads, smem, s>>>(items, n);
  PR_CUDA(cudaGetLastError());
  return PR_OK;
}

}  // namespace pr
