// Rendering of the reference's digital microstructures (porerad/geometry.py) on the device.
//
//  * k_render_shapes: the union of rotated ellipsoids and cylinders shorter than the cell on
//    the periodic N^3 grid (shape_mask, geometry.py:85-121), cell for cell as the reference's
//    NumPy expression evaluates it: minimum-image offsets ((i - c) + N/2) mod N - N/2 with
//    NumPy's float remainder; local coordinates R^T [x y z] as OpenBLAS's dgemm forms them for
//    three rows (a fused multiply-add chain r0 x, then + r1 y, then + r2 z, each fused);
//    (x_l / r_x)^2 + (y_l / r_y)^2 [+ (z_l / r_z)^2] <= 1 and |z_l| <= r_z.  A cell is tested
//    against a shape only within a conservative bound of the shape's extent.
//  * k_stamp: cylinders longer than the cell (_long_cylinder, geometry.py:59-82): the host
//    gives each fiber's lattice nodes and the offsets of its one-cell-thick disk, the device
//    marks (node + offset) mod N.
//  * k_count_solid: solid cells of the rendered array (the bisection on the radius,
//    geometry.py:124-145, reads phi_s = solid / N^3).
//  * k_lamellar: TL's continuous field (lamellar_field, geometry.py:223-239) from its host
//    parts (the per-x cosine, the per-y sine and per-z cosine of the waviness, the normal noise):
//    the wavy layer term with a correctly rounded sine, the 7-point periodic smoothing of the
//    noise summed in NumPy's order; thresholded by pr_quantile_threshold.
// Built with -fmad=false: every product and sum is rounded where NumPy rounds it.
#include <new>

#include "pr_internal.cuh"
#include "pr_math.cuh"

namespace pr {

namespace {

struct GenShape {
  int kind;
  double c[3];
  double col[3][3];  // col[i] = column i of R = local axis i
  double r[3];
  double bound;      // no cell beyond this offset (per axis) is inside
};

// ((v - c) + half) mod N - half, as NumPy evaluates it for v = 0..N-1 and c in [0, N)
__device__ __forceinline__ double min_image(int v, double c, double half, double nd) {
  const double a = ((double)v - c) + half;
  double m = fmod(a, nd);
  if (m != 0.0) {
    if ((m < 0.0) != (nd < 0.0)) m += nd;
  } else {
    m = copysign(0.0, nd);
  }
  return m - half;
}

__device__ __forceinline__ bool inside(const GenShape& s, double x, double y, double z) {
  const double xl = fma(s.col[0][2], z, fma(s.col[0][1], y, s.col[0][0] * x));
  const double yl = fma(s.col[1][2], z, fma(s.col[1][1], y, s.col[1][0] * x));
  const double zl = fma(s.col[2][2], z, fma(s.col[2][1], y, s.col[2][0] * x));
  const double a = xl / s.r[0], b = yl / s.r[1];
  if (s.kind == PR_SHAPE_ELLIPSOID) {
    const double c = zl / s.r[2];
    return (a * a + b * b) + c * c <= 1.0;
  }
  return a * a + b * b <= 1.0 && fabs(zl) <= s.r[2];
}

__global__ void __launch_bounds__(256) k_render_shapes(int N, const GenShape* __restrict__ shapes, int n_shapes,
                                                       uint8_t* __restrict__ phases) {
  extern __shared__ GenShape sh[];
  for (int q = threadIdx.x; q < n_shapes; q += blockDim.x) sh[q] = shapes[q];
  __syncthreads();
  const double nd = (double)N, half = nd / 2.0;
  const int64_t n = (int64_t)N * N * N;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(t / ((int64_t)N * N)), j = (int)((t / N) % N), k = (int)(t % N);
    uint8_t solid = 0;
    for (int q = 0; q < n_shapes && !solid; ++q) {
      const GenShape& s = sh[q];
      const double x = min_image(i, s.c[0], half, nd);
      if (fabs(x) > s.bound) continue;
      const double y = min_image(j, s.c[1], half, nd);
      if (fabs(y) > s.bound) continue;
      const double z = min_image(k, s.c[2], half, nd);
      if (fabs(z) > s.bound) continue;
      solid = inside(s, x, y, z);
    }
    phases[t] = solid;
  }
}

// fiber f: nodes[node0[f] .. node0[f+1]) and disk offsets[off0[f] .. off0[f+1]), int32 triples
__global__ void k_stamp(int N, const int* __restrict__ nodes, const int64_t* __restrict__ node0,
                        const int* __restrict__ offsets, const int64_t* __restrict__ off0, int n_fibers,
                        uint8_t value, uint8_t* __restrict__ phases) {
  for (int f = 0; f < n_fibers; ++f) {
    const int64_t nn = node0[f + 1] - node0[f], no = off0[f + 1] - off0[f];
    const int* nd = nodes + 3 * node0[f];
    const int* od = offsets + 3 * off0[f];
    for (int64_t w = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; w < nn * no; w += (int64_t)gridDim.x * blockDim.x) {
      const int64_t a = w / no, b = w - a * no;
      int c[3];
      for (int d = 0; d < 3; ++d) {
        int v = (nd[3 * a + d] + od[3 * b + d]) % N;
        c[d] = v < 0 ? v + N : v;
      }
      phases[((int64_t)c[0] * N + c[1]) * N + c[2]] = value;
    }
  }
}

__global__ void __launch_bounds__(256) k_count_solid(const uint8_t* __restrict__ phases, int64_t n, int64_t n16,
                                                     unsigned long long* __restrict__ out) {
  unsigned long long c = 0;
  const uint4* v = reinterpret_cast<const uint4*>(phases);
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n16; t += (int64_t)gridDim.x * blockDim.x) {
    const uint4 w = v[t];
    const unsigned int words[4] = {w.x, w.y, w.z, w.w};
    for (int q = 0; q < 4; ++q) {
      const unsigned int u = words[q];
      // bytes hold 0 or 1 after rendering; count bytes equal to 1
      const unsigned int ones = ~(u ^ 0x01010101u);
      const unsigned int eq = ones & (ones >> 1) & (ones >> 2) & (ones >> 3) & (ones >> 4) & (ones >> 5) &
                              (ones >> 6) & (ones >> 7) & 0x01010101u;
      c += __popc(eq);
    }
  }
  for (int64_t t = n16 * 16 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
       t += (int64_t)gridDim.x * blockDim.x)
    c += phases[t] == 1;
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(out, c);
}

__global__ void __launch_bounds__(256) k_lamellar(int N, const double* __restrict__ base,
                                                  const double* __restrict__ sin_y, const double* __restrict__ cos_z,
                                                  double waviness, double two_pi_layers,
                                                  const double* __restrict__ noise, double* __restrict__ field) {
  const int64_t n = (int64_t)N * N * N;
  const int64_t plane = (int64_t)N * N;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(t / plane), j = (int)((t / N) % N), k = (int)(t % N);
    // wav = waviness * (0.65 sin(.)[y] + 0.35 cos(.)[z]);  arg = (2 pi n (x + wav)) / N
    const double wav = waviness * (0.65 * sin_y[j] + 0.35 * cos_z[k]);
    const double arg = (two_pi_layers * ((double)i + wav)) / (double)N;
    double sv, cv;
    pr_sincos(arg, &sv, &cv);
    const double layer = base[i] + 0.35 * sv;
    const int im = i ? i - 1 : N - 1, ip = i + 1 < N ? i + 1 : 0;
    const int jm = j ? j - 1 : N - 1, jp = j + 1 < N ? j + 1 : 0;
    const int km = k ? k - 1 : N - 1, kp = k + 1 < N ? k + 1 : 0;
    const int64_t ci = (int64_t)i * plane, cj = (int64_t)j * N;
    double w = noise[t];
    w = w + noise[(int64_t)im * plane + cj + k];
    w = w + noise[(int64_t)ip * plane + cj + k];
    w = w + noise[ci + (int64_t)jm * N + k];
    w = w + noise[ci + (int64_t)jp * N + k];
    w = w + noise[ci + cj + km];
    w = w + noise[ci + cj + kp];
    field[t] = layer + w / 7.0;
  }
}

int count_solid(const uint8_t* phases, int64_t n, int64_t* solid, cudaStream_t s) {
  DevBuf<unsigned long long> cnt;
  PR_TRY(cnt.alloc(1, s));
  PR_CUDA(cudaMemsetAsync(cnt.ptr, 0, 8, s));
  const int64_t n16 = ((uintptr_t)phases % 16) ? 0 : n / 16;  // 16-byte loads only from an aligned array
  k_count_solid<<<grid_for(n / 16 + 1, 256, sm_count() * 4), 256, 0, s>>>(phases, n, n16, cnt.ptr);
  launch_mark();
  PR_CUDA(cudaGetLastError());
  unsigned long long h = 0;
  PR_CUDA(cudaMemcpyAsync(&h, cnt.ptr, 8, cudaMemcpyDeviceToHost, s));
  PR_CUDA(cudaStreamSynchronize(s));
  *solid = (int64_t)h;
  return PR_OK;
}

constexpr int kMaxShapes = 48 * 1024 / (int)sizeof(GenShape);  // shapes held in shared memory

}  // namespace

}  // namespace pr

using namespace pr;

extern "C" {

PR_API int pr_render_shapes(int64_t N, const pr_shape* shapes, int n_shapes, uint8_t* phases, int64_t* solid_cells,
                            void* stream) {
  PR_ARG(phases && (shapes || n_shapes == 0), "phases and shapes must not be NULL");
  PR_ARG(N > 0 && N <= 1290, "grid size N must be in 1..1290 (N^3 < 2^31)");
  PR_ARG(n_shapes >= 0, "n_shapes must not be negative");
  PR_ARG(is_device_pointer(phases), "phases must be device memory of N^3 bytes");
  if (n_shapes > kMaxShapes) {
    set_error("%d shapes exceed the %d of one launch", n_shapes, kMaxShapes);
    return PR_ERR_LIMIT;
  }
  const cudaStream_t s = (cudaStream_t)stream;
  GenShape* host = new (std::nothrow) GenShape[n_shapes > 0 ? n_shapes : 1];
  if (!host) {
    set_error("host allocation failed");
    return PR_ERR_OOM;
  }
  for (int q = 0; q < n_shapes; ++q) {
    const pr_shape& a = shapes[q];
    GenShape& g = host[q];
    if (a.kind != PR_SHAPE_ELLIPSOID && a.kind != PR_SHAPE_CYLINDER) {
      delete[] host;
      set_error("shape %d: unknown kind %d", q, a.kind);
      return PR_ERR_ARG;
    }
    g.kind = a.kind;
    for (int d = 0; d < 3; ++d) {
      g.c[d] = a.center[d];
      g.r[d] = a.radii[d];
      for (int e = 0; e < 3; ++e) g.col[d][e] = a.R[3 * e + d];  // column d, row e
    }
    // every inside cell lies within |offset| <= |local| of the centre: the largest semi-axis
    // (ellipsoid) or the half-diagonal (cylinder), with slack for rounding
    const double rmax = fmax(fabs(a.radii[0]), fmax(fabs(a.radii[1]), fabs(a.radii[2])));
    const double ext = a.kind == PR_SHAPE_ELLIPSOID
                           ? rmax
                           : sqrt(fmax(fabs(a.radii[0]), fabs(a.radii[1])) * fmax(fabs(a.radii[0]), fabs(a.radii[1])) +
                                  a.radii[2] * a.radii[2]);
    g.bound = ext * (1.0 + 1e-9) + 1e-6;
  }
  DevBuf<GenShape> dev;
  PR_TRY(dev.alloc((size_t)(n_shapes > 0 ? n_shapes : 1), s));
  cudaError_t e = cudaMemcpyAsync(dev.ptr, host, sizeof(GenShape) * (size_t)n_shapes, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);  // the staging array is freed below
  delete[] host;
  PR_CUDA(e);
  const int64_t n = N * N * N;
  timer_begin(kTimerRender, s);
  k_render_shapes<<<grid_for(n, 256, sm_count() * 16), 256, sizeof(GenShape) * (size_t)n_shapes, s>>>(
      (int)N, dev.ptr, n_shapes, phases);
  timer_end(kTimerRender, s);
  launch_mark();
  PR_CUDA(cudaGetLastError());
  if (solid_cells) PR_TRY(count_solid(phases, n, solid_cells, s));
  return PR_OK;
}

PR_API int pr_stamp_cells(int64_t N, const int32_t* nodes, const int64_t* node_start, const int32_t* offsets,
                          const int64_t* offset_start, int n_fibers, int clear, int value, uint8_t* phases,
                          int64_t* solid_cells, void* stream) {
  PR_ARG(value >= 0 && value <= 255, "value must be a byte");
  PR_ARG(phases && node_start && offset_start, "phases, node_start and offset_start must not be NULL");
  PR_ARG(N > 0 && N <= 1290, "grid size N must be in 1..1290 (N^3 < 2^31)");
  PR_ARG(n_fibers >= 0, "n_fibers must not be negative");
  PR_ARG(is_device_pointer(phases), "phases must be device memory of N^3 bytes");
  const int64_t n_nodes = node_start[n_fibers], n_off = offset_start[n_fibers];
  PR_ARG(node_start[0] == 0 && offset_start[0] == 0 && n_nodes >= 0 && n_off >= 0, "fiber ranges must start at 0");
  for (int f = 0; f < n_fibers; ++f)
    PR_ARG(node_start[f + 1] >= node_start[f] && offset_start[f + 1] >= offset_start[f], "fiber ranges must not decrease");
  PR_ARG((n_nodes == 0 || nodes) && (n_off == 0 || offsets), "nodes and offsets must not be NULL");
  const cudaStream_t s = (cudaStream_t)stream;
  const int64_t n = N * N * N;
  if (clear) PR_CUDA(cudaMemsetAsync(phases, 0, (size_t)n, s));
  if (n_fibers > 0 && n_nodes > 0 && n_off > 0) {
    DevBuf<int> dn, dof;
    DevBuf<int64_t> dn0, do0;
    PR_TRY(dn.alloc((size_t)(3 * n_nodes), s));
    PR_TRY(dof.alloc((size_t)(3 * n_off), s));
    PR_TRY(dn0.alloc((size_t)(n_fibers + 1), s));
    PR_TRY(do0.alloc((size_t)(n_fibers + 1), s));
    PR_CUDA(cudaMemcpyAsync(dn.ptr, nodes, 12 * (size_t)n_nodes, cudaMemcpyDefault, s));
    PR_CUDA(cudaMemcpyAsync(dof.ptr, offsets, 12 * (size_t)n_off, cudaMemcpyDefault, s));
    PR_CUDA(cudaMemcpyAsync(dn0.ptr, node_start, 8 * (size_t)(n_fibers + 1), cudaMemcpyDefault, s));
    PR_CUDA(cudaMemcpyAsync(do0.ptr, offset_start, 8 * (size_t)(n_fibers + 1), cudaMemcpyDefault, s));
    int64_t most = 0;
    for (int f = 0; f < n_fibers; ++f) {
      const int64_t w = (node_start[f + 1] - node_start[f]) * (offset_start[f + 1] - offset_start[f]);
      most = w > most ? w : most;
    }
    timer_begin(kTimerRender, s);
    k_stamp<<<grid_for(most, 256, sm_count() * 8), 256, 0, s>>>((int)N, dn.ptr, dn0.ptr, dof.ptr, do0.ptr, n_fibers,
                                                                (uint8_t)value, phases);
    timer_end(kTimerRender, s);
    launch_mark();
    PR_CUDA(cudaGetLastError());
    PR_CUDA(cudaStreamSynchronize(s));  // the host ranges may be freed by the caller on return
  }
  if (solid_cells) PR_TRY(count_solid(phases, n, solid_cells, s));
  return PR_OK;
}

PR_API int pr_lamellar_field(int64_t N, const double* base_x, const double* sin_y, const double* cos_z,
                             double waviness, double two_pi_layers, const double* noise, double* field,
                             void* stream) {
  PR_ARG(base_x && sin_y && cos_z && noise && field, "arrays must not be NULL");
  PR_ARG(N > 0 && N <= 1290, "grid size N must be in 1..1290 (N^3 < 2^31)");
  PR_ARG(is_device_pointer(field), "field must be device memory of N^3 doubles");
  const cudaStream_t s = (cudaStream_t)stream;
  const int64_t n = N * N * N;
  DevBuf<double> axes, dn;
  PR_TRY(axes.alloc((size_t)(3 * N), s));
  PR_CUDA(cudaMemcpyAsync(axes.ptr, base_x, 8 * (size_t)N, cudaMemcpyDefault, s));
  PR_CUDA(cudaMemcpyAsync(axes.ptr + N, sin_y, 8 * (size_t)N, cudaMemcpyDefault, s));
  PR_CUDA(cudaMemcpyAsync(axes.ptr + 2 * N, cos_z, 8 * (size_t)N, cudaMemcpyDefault, s));
  const double* nz = noise;
  if (!is_device_pointer(noise)) {
    PR_TRY(dn.alloc((size_t)n, s));
    PR_CUDA(cudaMemcpyAsync(dn.ptr, noise, 8 * (size_t)n, cudaMemcpyHostToDevice, s));
    nz = dn.ptr;
  }
  timer_begin(kTimerRender, s);
  k_lamellar<<<grid_for(n, 256, sm_count() * 16), 256, 0, s>>>((int)N, axes.ptr, axes.ptr + N, axes.ptr + 2 * N,
                                                               waviness, two_pi_layers, nz, field);
  timer_end(kTimerRender, s);
  launch_mark();
  PR_CUDA(cudaGetLastError());
  PR_CUDA(cudaStreamSynchronize(s));  // host inputs may be freed by the caller on return
  return PR_OK;
}

PR_API int pr_stamp_fibers(int64_t N, const int32_t* nodes, const int64_t* node_start, const int32_t* offsets,
                           const int64_t* offset_start, int n_fibers, int clear, uint8_t* phases,
                           int64_t* solid_cells, void* stream) {
  return pr_stamp_cells(N, nodes, node_start, offsets, offset_start, n_fibers, clear, 1, phases, solid_cells,
                        stream);
}

}  // extern "C"
