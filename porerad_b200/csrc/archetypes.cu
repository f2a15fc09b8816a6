// Grid work of the benchmark archetype generators (porerad_b200/geometry.py) on the device,
// bit-identical to their host definitions.
//
//  * k_voronoi_field: the open-cell foam's strut field d3 - d1 at every cell centre
//    (i + 1/2, j + 1/2, k + 1/2): distances to the first and third nearest of the periodic seed
//    points.  Per axis the difference c - p is wrapped once into [-N/2, N/2] (below -N/2: + N,
//    above N/2: - N), squares are summed x, y, z in that order and the square roots taken after
//    ranking, the arithmetic of SciPy's periodic k-d tree query for these inputs.
//  * k_stamp_first / k_first_hist / k_first_threshold: a batch of fibers (or holes) stamped at
//    once, each cell keeping the smallest index of one that covers it; the cells each adds (or,
//    within a mask, removes) are then a histogram, so the host finds where its one-at-a-time loop
//    would stop, and the phases follow from "first index <= that one" (the same union).
//  * pr_quantile_threshold: NumPy's default quantile of a device array (the order statistics
//    from a radix sort, the linear interpolation of numpy.quantile on the host) and the
//    threshold field <= q (or >= q) into a phase array.
// Built with -fmad=false.
#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <cmath>
#include <new>
#include <vector>

#include "pr_internal.cuh"

namespace pr {

namespace {

__global__ void __launch_bounds__(256) k_voronoi_field(int N, const double* __restrict__ seeds, int n_seeds,
                                                       double* __restrict__ field) {
  extern __shared__ double sp[];
  for (int q = threadIdx.x; q < 3 * n_seeds; q += blockDim.x) sp[q] = seeds[q];
  __syncthreads();
  const double hb = (double)N / 2.0, fb = (double)N;
  const int64_t n = (int64_t)N * N * N;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(t / ((int64_t)N * N)), j = (int)((t / N) % N), k = (int)(t % N);
    const double c[3] = {(double)i + 0.5, (double)j + 0.5, (double)k + 0.5};
    double d1 = INFINITY, d2 = INFINITY, d3 = INFINITY;
    for (int s = 0; s < n_seeds; ++s) {
      double acc = 0.0;
      for (int a = 0; a < 3; ++a) {
        double x = c[a] - sp[3 * s + a];
        x = x < -hb ? fb + x : (x > hb ? x - fb : x);
        acc = acc + x * x;
      }
      if (acc < d3) {
        if (acc < d2) {
          d3 = d2;
          if (acc < d1) {
            d2 = d1;
            d1 = acc;
          } else {
            d2 = acc;
          }
        } else {
          d3 = acc;
        }
      }
    }
    field[t] = sqrt(d3) - sqrt(d1);
  }
}

__global__ void k_threshold(const double* __restrict__ field, int64_t n, double q, int below,
                            uint8_t* __restrict__ phases, unsigned long long* __restrict__ count) {
  unsigned long long c = 0;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    const uint8_t v = below ? field[t] <= q : field[t] >= q;
    phases[t] = v;
    c += v;
  }
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, c);
}

// Segments of a batch of fibers (fiber f: nodes[node_start[f] .. node_start[f+1]) thickened by
// the shared offsets): each cell keeps the smallest index of a fiber covering it.
__global__ void k_stamp_first(int N, const int* __restrict__ nodes, const int64_t* __restrict__ node_start,
                              const int* __restrict__ offsets, int n_off, int n_fibers, int base,
                              int* __restrict__ first) {
  for (int f = 0; f < n_fibers; ++f) {
    const int64_t nn = node_start[f + 1] - node_start[f];
    const int* nd = nodes + 3 * node_start[f];
    for (int64_t w = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; w < nn * n_off;
         w += (int64_t)gridDim.x * blockDim.x) {
      const int64_t a = w / n_off, b = w - a * n_off;
      int c[3];
      for (int d = 0; d < 3; ++d) {
        const int v = (nd[3 * a + d] + offsets[3 * b + d]) % N;
        c[d] = v < 0 ? v + N : v;
      }
      atomicMin(first + ((int64_t)c[0] * N + c[1]) * N + c[2], base + f);
    }
  }
}

// new[f] = cells whose first covering fiber is base + f (f < K <= 1024), among the cells where
// mask is 1 when a mask is given
__global__ void __launch_bounds__(256) k_first_hist(const int* __restrict__ first, const uint8_t* __restrict__ mask,
                                                    int64_t n, int base, int K, unsigned long long* __restrict__ out) {
  __shared__ unsigned int h[1024];
  for (int q = threadIdx.x; q < K; q += blockDim.x) h[q] = 0;
  __syncthreads();
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    const int v = first[t] - base;
    if (v >= 0 && v < K && (!mask || mask[t] == 1)) atomicAdd(h + v, 1u);
  }
  __syncthreads();
  for (int q = threadIdx.x; q < K; q += blockDim.x)
    if (h[q]) atomicAdd(out + q, (unsigned long long)h[q]);
}

// mode 0: phases = first <= last (the union of the fibers up to last); mode 1: cells covered by a
// hole up to last are cleared
__global__ void k_first_threshold(const int* __restrict__ first, int64_t n, int last, int mode,
                                  uint8_t* __restrict__ phases) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    const bool covered = first[t] <= last;
    if (mode == 0) phases[t] = covered;
    else if (covered) phases[t] = 0;
  }
}

// numpy.quantile(x, q) ("linear"): virtual index v = (n - 1) q between sorted values a and b
static double numpy_lerp_quantile(double a, double b, double v, double lo) {
  const double g = v - lo;
  const double d = b - a;
  return g >= 0.5 ? b - d * (1.0 - g) : a + d * g;
}

}  // namespace

}  // namespace pr

using namespace pr;

extern "C" {

PR_API int pr_voronoi_edge_field(int64_t N, const double* seeds, int n_seeds, double* field, void* stream) {
  PR_ARG(seeds && field, "seeds and field must not be NULL");
  PR_ARG(N > 0 && N <= 1290, "grid size N must be in 1..1290 (N^3 < 2^31)");
  PR_ARG(n_seeds >= 3 && n_seeds <= 2048, "n_seeds must be in 3..2048");
  PR_ARG(is_device_pointer(field), "field must be device memory of N^3 doubles");
  const cudaStream_t s = (cudaStream_t)stream;
  DevBuf<double> dev;
  PR_TRY(dev.alloc((size_t)(3 * n_seeds), s));
  PR_CUDA(cudaMemcpyAsync(dev.ptr, seeds, 24 * (size_t)n_seeds, cudaMemcpyDefault, s));
  const int64_t n = N * N * N;
  k_voronoi_field<<<grid_for(n, 256, sm_count() * 16), 256, 24 * (size_t)n_seeds, s>>>((int)N, dev.ptr, n_seeds,
                                                                                       field);
  launch_mark();
  PR_CUDA(cudaGetLastError());
  PR_CUDA(cudaStreamSynchronize(s));  // the seed array may be host memory the caller frees
  return PR_OK;
}

PR_API int pr_quantile_threshold(const double* field, int64_t n, double quantile, int below, uint8_t* phases,
                                 double* q_out, int64_t* solid_cells, void* stream) {
  PR_ARG(field && phases, "field and phases must not be NULL");
  PR_ARG(n > 0 && n < ((int64_t)1 << 31), "n must be in 1..2^31 - 1");
  PR_ARG(quantile >= 0.0 && quantile <= 1.0, "quantile must be in [0, 1]");
  PR_ARG(is_device_pointer(field) && is_device_pointer(phases), "field and phases must be device memory");
  const cudaStream_t s = (cudaStream_t)stream;
  DevBuf<double> sorted;
  PR_TRY(sorted.alloc((size_t)n, s));
  size_t tmp_bytes = 0;
  PR_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tmp_bytes, field, sorted.ptr, (int)n, 0, 64, s));
  DevBuf<uint8_t> tmp;
  PR_TRY(tmp.alloc(tmp_bytes + 16, s));
  PR_CUDA(cub::DeviceRadixSort::SortKeys(tmp.ptr, tmp_bytes, field, sorted.ptr, (int)n, 0, 64, s));
  const double v = (double)(n - 1) * quantile;
  int64_t lo_i, hi_i;
  double lo;
  if (v >= (double)(n - 1)) {
    lo_i = hi_i = n - 1;
    lo = -1.0;  // numpy marks the index past the top with -1; both values are the largest
  } else if (v < 0.0) {
    lo_i = hi_i = 0;
    lo = 0.0;
  } else {
    lo = std::floor(v);
    lo_i = (int64_t)lo;
    hi_i = lo_i + 1;
  }
  double ab[2];
  PR_CUDA(cudaMemcpyAsync(ab, sorted.ptr + lo_i, 8, cudaMemcpyDeviceToHost, s));
  PR_CUDA(cudaMemcpyAsync(ab + 1, sorted.ptr + hi_i, 8, cudaMemcpyDeviceToHost, s));
  PR_CUDA(cudaStreamSynchronize(s));
  const double q = numpy_lerp_quantile(ab[0], ab[1], v, lo);
  DevBuf<unsigned long long> cnt;
  PR_TRY(cnt.alloc(1, s));
  PR_CUDA(cudaMemsetAsync(cnt.ptr, 0, 8, s));
  k_threshold<<<grid_for(n, 256, sm_count() * 8), 256, 0, s>>>(field, n, q, below, phases, cnt.ptr);
  launch_mark();
  PR_CUDA(cudaGetLastError());
  unsigned long long h = 0;
  PR_CUDA(cudaMemcpyAsync(&h, cnt.ptr, 8, cudaMemcpyDeviceToHost, s));
  PR_CUDA(cudaStreamSynchronize(s));
  if (q_out) *q_out = q;
  if (solid_cells) *solid_cells = (int64_t)h;
  return PR_OK;
}

PR_API int pr_stamp_first(int64_t N, const int32_t* nodes, const int64_t* node_start, const int32_t* offsets,
                          int64_t n_offsets, int n_fibers, int base, int32_t* first, const uint8_t* mask,
                          int64_t* new_cells, void* stream) {
  PR_ARG(node_start && first && new_cells, "node_start, first and new_cells must not be NULL");
  PR_ARG(N > 0 && N <= 1290, "grid size N must be in 1..1290 (N^3 < 2^31)");
  PR_ARG(n_fibers >= 0 && n_fibers <= 1024, "n_fibers must be in 0..1024");
  PR_ARG(base >= 0 && (int64_t)base + n_fibers < INT32_MAX, "fiber indices must stay below 2^31 - 1");
  PR_ARG(n_offsets >= 0 && n_offsets < INT32_MAX, "n_offsets out of range");
  PR_ARG(is_device_pointer(first), "first must be device memory of N^3 int32");
  PR_ARG(!mask || is_device_pointer(mask), "mask must be device memory of N^3 bytes");
  const int64_t n_nodes = node_start[n_fibers];
  PR_ARG(node_start[0] == 0 && n_nodes >= 0, "fiber ranges must start at 0");
  for (int f = 0; f < n_fibers; ++f) PR_ARG(node_start[f + 1] >= node_start[f], "fiber ranges must not decrease");
  PR_ARG((n_nodes == 0 || nodes) && (n_offsets == 0 || offsets), "nodes and offsets must not be NULL");
  const cudaStream_t s = (cudaStream_t)stream;
  const int64_t n = N * N * N;
  DevBuf<unsigned long long> hist;
  PR_TRY(hist.alloc((size_t)(n_fibers > 0 ? n_fibers : 1), s));
  PR_CUDA(cudaMemsetAsync(hist.ptr, 0, 8 * (size_t)(n_fibers > 0 ? n_fibers : 1), s));
  if (n_fibers > 0 && n_nodes > 0 && n_offsets > 0) {
    DevBuf<int> dn, dof;
    DevBuf<int64_t> dn0;
    PR_TRY(dn.alloc((size_t)(3 * n_nodes), s));
    PR_TRY(dof.alloc((size_t)(3 * n_offsets), s));
    PR_TRY(dn0.alloc((size_t)(n_fibers + 1), s));
    PR_CUDA(cudaMemcpyAsync(dn.ptr, nodes, 12 * (size_t)n_nodes, cudaMemcpyDefault, s));
    PR_CUDA(cudaMemcpyAsync(dof.ptr, offsets, 12 * (size_t)n_offsets, cudaMemcpyDefault, s));
    PR_CUDA(cudaMemcpyAsync(dn0.ptr, node_start, 8 * (size_t)(n_fibers + 1), cudaMemcpyDefault, s));
    int64_t most = 0;
    for (int f = 0; f < n_fibers; ++f) most = std::max(most, (node_start[f + 1] - node_start[f]) * n_offsets);
    k_stamp_first<<<grid_for(most, 256, sm_count() * 8), 256, 0, s>>>((int)N, dn.ptr, dn0.ptr, dof.ptr,
                                                                     (int)n_offsets, n_fibers, base, first);
    launch_mark();
    PR_CUDA(cudaGetLastError());
    k_first_hist<<<grid_for(n, 256, sm_count() * 4), 256, 0, s>>>(first, mask, n, base, n_fibers, hist.ptr);
    launch_mark();
    PR_CUDA(cudaGetLastError());
  }
  std::vector<unsigned long long> h((size_t)(n_fibers > 0 ? n_fibers : 1));
  PR_CUDA(cudaMemcpyAsync(h.data(), hist.ptr, 8 * h.size(), cudaMemcpyDeviceToHost, s));
  PR_CUDA(cudaStreamSynchronize(s));  // host inputs may be freed by the caller on return
  for (int f = 0; f < n_fibers; ++f) new_cells[f] = (int64_t)h[f];
  return PR_OK;
}

PR_API int pr_first_threshold(const int32_t* first, int64_t n, int last, int mode, uint8_t* phases, void* stream) {
  PR_ARG(mode == 0 || mode == 1, "mode must be 0 (union) or 1 (clear the covered cells)");
  PR_ARG(first && phases && n > 0, "first and phases must not be NULL; n must be positive");
  PR_ARG(is_device_pointer(first) && is_device_pointer(phases), "first and phases must be device memory");
  const cudaStream_t s = (cudaStream_t)stream;
  k_first_threshold<<<grid_for(n, 256, sm_count() * 8), 256, 0, s>>>(first, n, last, mode, phases);
  launch_mark();
  PR_CUDA(cudaGetLastError());
  PR_CUDA(cudaStreamSynchronize(s));
  return PR_OK;
}

}  // extern "C"
