// Gray-diffuse radiosity on the device.
//
// Reflection series (porerad/exchange.py:217-245): flight_0 = E; every reflection
//   incident = F_p^T flight = d * S(d * (flight / A))          (exchange.py:119-122)
//   absorbed += eps * incident;  flight = (1 - eps) * incident
// until sum|flight| <= rtol * max(sum|E|, tiny).  One fused kernel per reflection
// (SpMV + the three vector updates + block partial sums of |flight| and flight)
// and a one-thread finish kernel that sums the partials in a fixed order and sets
// a device flag; reflections launched after convergence return at once, so the
// host checks the flag only once per batch of launches.
//
// Emission (exchange.py:248-271): E = eps sigma A T^4, or with a reference
// temperature the factored eps sigma A ((T - Tr)(T + Tr)(T T + Tr Tr)).
// Prescribed field (coupled.py:138-194): walls at T_m +/- dT/2, internal patches at
// T_h - (i + 0.5) dT / nx of their cell; q_h, q_c, q_i = -sum(net of class) / (ny nz
// (H / nx)^2); coarse source = cell power summed over min(8, n)^3 blocks split as
// numpy.array_split does.
//
// Mixed precision: binary32 Chebyshev sweeps over the same packed matrix (the integer
// counts are exact in binary32) inside binary64 iterative refinement of the radiosity
// J = E + (1 - eps) F_p^T J: the residual r = E - J + (1 - eps) F_p^T J and the absorbed
// power eps F_p^T J are binary64.
#include <cmath>
#include <mutex>
#include <vector>

#include "pr_spmv.cuh"

namespace pr {

#define PR_SIGMA 5.670374419e-8  // porerad/constants.py:3

struct SeriesState {
  int done;        // 0 running, 1 converged, 2 reflection cap reached
  int pad;
  long long iters;
  double residual;  // sum of the power in flight at convergence
  double tol_abs;   // rtol * max(sum|E|, tiny)
};

// One reflection of the series on v = d (flight / A):  inc = d S v;  absorbed += eps inc;
// flight = (1 - eps) inc;  v_out = d (flight / A);  block partials of |flight| and flight.
struct SeriesEpi {
  double delta;
  const double* area;
  const double* d;
  const double* eps;
  const double* v_in;
  double* v_out;
  double* absorbed;
  double* partial;
  const SeriesState* state;
  struct Red {
    double v[2] = {0.0, 0.0};
  };
  __device__ bool skip() const { return state->done != 0; }
  __device__ void row(int64_t i, double sp, Red& r) const {
    const double Ai = area[i];
    const double s = sp + delta * Ai * v_in[i];
    const double inc = d[i] * s;
    const double e = eps[i];
    absorbed[i] += e * inc;
    const double fl = (1.0 - e) * inc;
    v_out[i] = d[i] * (fl / Ai);
    r.v[0] += fabs(fl);
    r.v[1] += fl;
  }
  __device__ void finish(Red& r) const { block_sum_store<2>(r.v, partial); }
};

__global__ void k_series_finish(const double* __restrict__ partial, int blocks, long long max_it,
                                SeriesState* __restrict__ state) {
  if (state->done) return;  // one warp: the same value on every lane
  const int lane = threadIdx.x & 31;
  const double a = warp_sum_partials(partial, blocks, 2, 0, lane);
  const double t = warp_sum_partials(partial, blocks, 2, 1, lane);
  if (lane != 0) return;
  state->iters += 1;
  if (a <= state->tol_abs) {
    state->done = 1;
    state->residual = t;
  } else if (state->iters >= max_it) {
    state->done = 2;
  }
}

// v = d * (x / A) and the block partials of |x|
__global__ void __launch_bounds__(256) k_series_init(const double* __restrict__ x, const double* __restrict__ d,
                                                     const double* __restrict__ area, int64_t n,
                                                     double* __restrict__ v, double* __restrict__ absorbed,
                                                     double* __restrict__ partial) {
  double acc[1] = {0.0};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    v[i] = d[i] * (x[i] / area[i]);
    absorbed[i] = 0.0;
    acc[0] += fabs(x[i]);
  }
  block_sum_store<1>(acc, partial);
}

__global__ void k_series_tol(const double* __restrict__ partial, int blocks, double rtol,
                             SeriesState* __restrict__ state) {
  const double a = warp_sum_partials(partial, blocks, 1, 0, threadIdx.x & 31);
  if (threadIdx.x != 0) return;
  const double tiny = 2.2250738585072014e-308;
  state->done = 0;
  state->iters = 0;
  state->residual = 0.0;
  state->tol_abs = rtol * fmax(a, tiny);
}

static int red_blocks() { return sm_count() * 4; }

// FP64 reflection series on device vectors: emitted (n), eps (n) -> absorbed (n).
int series_fp64(const pr_operator* op, const double* emitted, const double* eps, double rtol, int64_t max_it,
                double* absorbed, double* residual, int64_t* iterations, cudaStream_t s) {
  const int64_t n = op->n;
  const int rb = red_blocks();
  const int sb = spmv_slots(op->S);
  DevBuf<double> va, vb, partial;
  DevBuf<SeriesState> st;
  PR_TRY(va.alloc(n, s));
  PR_TRY(vb.alloc(n, s));
  PR_TRY(partial.alloc((size_t)2 * (sb > rb ? sb : rb), s));
  PR_TRY(st.alloc(1, s));
  PR_CUDA(cudaMemsetAsync(st.ptr, 0, sizeof(SeriesState), s));
  ::pr::launch_mark(), k_series_init<<<rb, 256, 0, s>>>(emitted, op->scale.ptr, op->area.ptr, n, va.ptr, absorbed, partial.ptr);
  PR_CUDA(cudaGetLastError());
  ::pr::launch_mark(), k_series_tol<<<1, 32, 0, s>>>(partial.ptr, rb, rtol, st.ptr);
  PR_CUDA(cudaGetLastError());
  double* vin = va.ptr;
  double* vout = vb.ptr;
  SeriesState h;
  int batch = 4;
  for (int64_t launched = 0;;) {
    for (int b = 0; b < batch; ++b) {
      const SeriesEpi epi{op->delta, op->area.ptr, op->scale.ptr, eps, vin, vout, absorbed, partial.ptr, st.ptr};
      int rc = PR_OK;
      ::pr::timer_begin(kTimerSeries, s);
      dispatch_mode(op->S.mode, [&](auto m) { rc = launch_spmv<decltype(m)::value, double>(op->S, vin, epi, s); });
      ::pr::timer_end(kTimerSeries, s);
      PR_TRY(rc);
      ::pr::launch_mark(), k_series_finish<<<1, 32, 0, s>>>(partial.ptr, sb, (long long)max_it, st.ptr);
      std::swap(vin, vout);
    }
    PR_CUDA(cudaGetLastError());
    launched += batch;
    PR_CUDA(cudaMemcpyAsync(&h, st.ptr, sizeof(h), cudaMemcpyDeviceToHost, s));
    PR_CUDA(cudaStreamSynchronize(s));
    if (h.done) break;
    if (batch < 64) batch *= 2;
  }
  op->spmv_calls += h.iters;
  if (h.done == 2) {
    set_error("radiosity reflection series did not converge");
    return PR_ERR_SERIES;
  }
  *residual = h.residual;
  *iterations = h.iters;
  return PR_OK;
}

// ------------------------------------------------------------------ emission / JVP

__global__ void k_emission(const double* __restrict__ T, const double* __restrict__ eps,
                           const double* __restrict__ area, int64_t n, int has_ref, double ref,
                           double* __restrict__ e) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double t = T[i];
    const double pre = eps[i] * PR_SIGMA * area[i];
    e[i] = has_ref ? pre * ((t - ref) * (t + ref) * (t * t + ref * ref)) : pre * pow(t, 4.0);
  }
}

__global__ void k_emission_derivative(const double* __restrict__ T, const double* __restrict__ dT,
                                      const double* __restrict__ eps, const double* __restrict__ area, int64_t n,
                                      double* __restrict__ e) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    e[i] = 4.0 * eps[i] * PR_SIGMA * area[i] * pow(T[i], 3.0) * dT[i];
}

__global__ void k_sub(const double* __restrict__ a, const double* __restrict__ b, int64_t n, double* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = a[i] - b[i];
}

int net_patch_power(const pr_operator* op, const double* T, const double* eps, const double* area, double rtol,
                    int has_ref, double ref, int64_t max_it, double* emitted, double* absorbed, double* net,
                    double* residual, int64_t* iterations, cudaStream_t s) {
  const int64_t n = op->n;
  DevBuf<double> dT, de, da, dE, dAb;
  PR_TRY(dT.alloc(n, s));
  PR_TRY(de.alloc(n, s));
  PR_TRY(da.alloc(n, s));
  PR_TRY(dE.alloc(n, s));
  PR_TRY(dAb.alloc(n, s));
  PR_CUDA(cudaMemcpyAsync(dT.ptr, T, n * 8, cudaMemcpyDefault, s));
  PR_CUDA(cudaMemcpyAsync(de.ptr, eps, n * 8, cudaMemcpyDefault, s));
  PR_CUDA(cudaMemcpyAsync(da.ptr, area, n * 8, cudaMemcpyDefault, s));
  ::pr::launch_mark(), k_emission<<<grid_for(n, 256), 256, 0, s>>>(dT.ptr, de.ptr, da.ptr, n, has_ref, ref, dE.ptr);
  PR_CUDA(cudaGetLastError());
  double res = 0.0;
  int64_t it = 0;
  PR_TRY(series_fp64(op, dE.ptr, de.ptr, rtol, max_it, dAb.ptr, &res, &it, s));
  if (emitted) PR_CUDA(cudaMemcpyAsync(emitted, dE.ptr, n * 8, cudaMemcpyDefault, s));
  if (absorbed) PR_CUDA(cudaMemcpyAsync(absorbed, dAb.ptr, n * 8, cudaMemcpyDefault, s));
  if (net) {
    ::pr::launch_mark(), k_sub<<<grid_for(n, 256), 256, 0, s>>>(dAb.ptr, dE.ptr, n, dT.ptr);
    PR_CUDA(cudaMemcpyAsync(net, dT.ptr, n * 8, cudaMemcpyDefault, s));
  }
  PR_CUDA(cudaStreamSynchronize(s));
  if (residual) *residual = res;
  if (iterations) *iterations = it;
  return PR_OK;
}

int net_patch_power_jvp(const pr_operator* op, const double* T, const double* dTin, const double* eps,
                        const double* area, double rtol, double* out, cudaStream_t s) {
  const int64_t n = op->n;
  DevBuf<double> dT, dd, de, da, dE, dAb;
  PR_TRY(dT.alloc(n, s));
  PR_TRY(dd.alloc(n, s));
  PR_TRY(de.alloc(n, s));
  PR_TRY(da.alloc(n, s));
  PR_TRY(dE.alloc(n, s));
  PR_TRY(dAb.alloc(n, s));
  PR_CUDA(cudaMemcpyAsync(dT.ptr, T, n * 8, cudaMemcpyDefault, s));
  PR_CUDA(cudaMemcpyAsync(dd.ptr, dTin, n * 8, cudaMemcpyDefault, s));
  PR_CUDA(cudaMemcpyAsync(de.ptr, eps, n * 8, cudaMemcpyDefault, s));
  PR_CUDA(cudaMemcpyAsync(da.ptr, area, n * 8, cudaMemcpyDefault, s));
  ::pr::launch_mark(), k_emission_derivative<<<grid_for(n, 256), 256, 0, s>>>(dT.ptr, dd.ptr, de.ptr, da.ptr, n, dE.ptr);
  PR_CUDA(cudaGetLastError());
  double res = 0.0;
  int64_t it = 0;
  PR_TRY(series_fp64(op, dE.ptr, de.ptr, rtol, 10000, dAb.ptr, &res, &it, s));
  ::pr::launch_mark(), k_sub<<<grid_for(n, 256), 256, 0, s>>>(dAb.ptr, dE.ptr, n, dT.ptr);
  PR_CUDA(cudaMemcpyAsync(out, dT.ptr, n * 8, cudaMemcpyDefault, s));
  PR_CUDA(cudaStreamSynchronize(s));
  return PR_OK;
}

int reflection_series(const pr_operator* op, const double* emitted, const double* eps, double rtol, int64_t max_it,
                      double* absorbed, double* residual, int64_t* iterations, cudaStream_t s) {
  const int64_t n = op->n;
  DevBuf<double> dE, de, dAb;
  PR_TRY(dE.alloc(n, s));
  PR_TRY(de.alloc(n, s));
  PR_TRY(dAb.alloc(n, s));
  PR_CUDA(cudaMemcpyAsync(dE.ptr, emitted, n * 8, cudaMemcpyDefault, s));
  PR_CUDA(cudaMemcpyAsync(de.ptr, eps, n * 8, cudaMemcpyDefault, s));
  PR_TRY(series_fp64(op, dE.ptr, de.ptr, rtol, max_it, dAb.ptr, residual, iterations, s));
  PR_CUDA(cudaMemcpyAsync(absorbed, dAb.ptr, n * 8, cudaMemcpyDefault, s));
  PR_CUDA(cudaStreamSynchronize(s));
  return PR_OK;
}

// ------------------------------------------------------------------ prescribed-field channels

// Patch temperature (coupled.py:45-53 with the linear field of coupled.py:138-143),
// uniform emissivity and the T_ref-subtracted emission (exchange.py:268-270).
// Patch temperature and emission for the channel solves.  T_cells == nullptr: the linear
// prescribed field (walls at T_m +/- dT/2, coupled.py:138-143, 178-184); otherwise the given
// cell field with walls at Th, Tc (coupled.py:45-53).  Emission with a reference
// temperature in the factored form of exchange.py:268-270, else eps sigma A T^4.
struct FieldSpec {
  const double* T_cells;
  double T_m, dT, Th, Tc, eps, ref;
  int has_ref;
};

__global__ void k_field_emission(const int8_t* __restrict__ cls, const int32_t* __restrict__ cell,
                                 const double* __restrict__ area, int64_t n, int64_t nyz, int64_t nx, FieldSpec f,
                                 double* __restrict__ e, double* __restrict__ eps) {
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
    double t;
    const int c = cls[p];
    if (c == 0) t = f.Th;
    else if (c == 1) t = f.Tc;
    else if (f.T_cells) t = f.T_cells[cell[p]];
    else {
      const int64_t i = cell[p] / nyz;
      t = (f.T_m + f.dT / 2.0) - (((double)i + 0.5) * f.dT) / (double)nx;
    }
    const double pre = f.eps * PR_SIGMA * area[p];
    const double r = f.ref;
    e[p] = f.has_ref ? pre * ((t - r) * (t + r) * (t * t + r * r)) : pre * pow(t, 4.0);
    eps[p] = f.eps;
  }
}

// block partial sums of net power per class
__global__ void __launch_bounds__(256) k_class_sums(const int8_t* __restrict__ cls, const double* __restrict__ ab,
                                                    const double* __restrict__ e, int64_t n,
                                                    double* __restrict__ partial) {
  double acc[3] = {0.0, 0.0, 0.0};
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
    const double net = ab[p] - e[p];
    const int c = cls[p];
    acc[0] += c == 0 ? net : 0.0;
    acc[1] += c == 1 ? net : 0.0;
    acc[2] += c == 2 ? net : 0.0;
  }
  block_sum_store<3>(acc, partial);
}

// numpy.array_split(arange(n), b): the first n % b parts have n / b + 1 items.
__device__ __forceinline__ void split_range(int64_t n, int64_t b, int64_t part, int64_t& lo, int64_t& hi) {
  const int64_t q = n / b, r = n % b;
  lo = part * q + (part < r ? part : r);
  hi = lo + q + (part < r ? 1 : 0);
}

// One block per coarse bin: sum of the net power of the internal patches of its cells.
__global__ void __launch_bounds__(256) k_coarse(const int32_t* __restrict__ cfp, const double* __restrict__ ab,
                                                const double* __restrict__ e, int64_t nx, int64_t ny, int64_t nz,
                                                int bx, int by, int bz, double scale, double* __restrict__ out) {
  const int bin = blockIdx.x;
  const int a = bin / (by * bz), b = (bin / bz) % by, c = bin % bz;
  int64_t x0, x1, y0, y1, z0, z1;
  split_range(nx, bx, a, x0, x1);
  split_range(ny, by, b, y0, y1);
  split_range(nz, bz, c, z0, z1);
  const int64_t sy = y1 - y0, sz = z1 - z0;
  const int64_t cells = (x1 - x0) * sy * sz;
  double acc[1] = {0.0};
  for (int64_t t = threadIdx.x; t < cells; t += blockDim.x) {
    const int64_t x = x0 + t / (sy * sz), y = y0 + (t / sz) % sy, z = z0 + t % sz;
    const int64_t cell = (x * ny + y) * nz + z;
    for (int f = 0; f < 6; ++f) {
      const int32_t p = cfp[cell * 6 + f];
      if (p >= 0) acc[0] += ab[p] - e[p];
    }
  }
  __shared__ double part[1];
  block_sum_store<1>(acc, part, 0);
  if (threadIdx.x == 0) out[bin] = part[0] * scale;
}

// ------------------------------------------------------------------ mixed precision

// One Chebyshev step on (I - om G) x = b in binary32 (Saad, Iterative Methods, Alg. 12.1):
//   G d = scale * (S' u + delta A u), u = scale d / A;  x += d;  r -= (I - om G) d;
//   d = c1 d + c2 r;  u_out = scale d / A.
struct ChebEpi {
  float delta;
  const float* scale;
  const float* area;
  const float* om;
  const float* u_in;
  float* u_out;
  float* x;
  float* r;
  float* d;
  float c1, c2;
  struct Red {};
  __device__ bool skip() const { return false; }
  __device__ void row(int64_t i, float sum, Red&) const {
    const float Ai = area[i], sc = scale[i];
    const float gd = sc * (sum + delta * Ai * u_in[i]);
    const float di = d[i];
    const float ad = di - om[i] * gd;
    x[i] += di;
    const float ri = r[i] - ad;
    r[i] = ri;
    const float dn = c1 * di + c2 * ri;
    d[i] = dn;
    u_out[i] = sc * dn / Ai;
  }
  __device__ void finish(Red&) const {}
};

// J += x (when x != nullptr); u = scale J / A; also the binary32 copies of the coefficients.
__global__ void k_refine_prep(double* __restrict__ J, const float* __restrict__ x, const double* __restrict__ scale,
                              const double* __restrict__ area, int64_t n, double* __restrict__ u) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double j = J[i];
    if (x) {
      j += (double)x[i];
      J[i] = j;
    }
    u[i] = scale[i] * (j / area[i]);
  }
}

// Binary64 residual r = E - J + om G J, absorbed = eps G J; block partials of |r| and |E|;
// binary32 start of the next correction solve: x = 0, r32 = d32 = r, u32 = scale r / A.
struct RefineEpi {
  double delta;
  const double* area;
  const double* scale;
  const double* eps;
  const double* E;
  const double* J;
  const double* u;
  double* absorbed;
  double* partial;
  float* x32;
  float* r32;
  float* d32;
  float* u32;
  struct Red {
    double v[2] = {0.0, 0.0};
  };
  __device__ bool skip() const { return false; }
  __device__ void row(int64_t i, double sp, Red& red) const {
    const double Ai = area[i];
    const double s = sp + delta * Ai * u[i];
    const double gj = scale[i] * s;
    const double e = eps[i];
    const double r = E[i] - J[i] + (1.0 - e) * gj;
    absorbed[i] = e * gj;
    red.v[0] += fabs(r);
    red.v[1] += fabs(E[i]);
    x32[i] = 0.0f;
    r32[i] = (float)r;
    d32[i] = (float)r;  // d0 = r0 / theta with theta = 1
    u32[i] = (float)(scale[i] * (r / Ai));
  }
  __device__ void finish(Red& red) const { block_sum_store<2>(red.v, partial); }
};

__global__ void k_to_f32(const double* __restrict__ a, const double* __restrict__ b, const double* __restrict__ c,
                         int64_t n, float* __restrict__ fa, float* __restrict__ fb, float* __restrict__ fc) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    fa[i] = (float)a[i];
    fb[i] = (float)b[i];
    fc[i] = (float)(1.0 - c[i]);
  }
}

// Mixed-precision radiosity: binary64 refinement of J with binary32 Chebyshev
// corrections; absorbed = eps G J from the last binary64 residual.  stats: outer
// refinements, SpMVs (binary64 + binary32), final |r|_1 / |E|_1, binary32 sweeps per
// correction.
int series_mixed(const pr_operator* op, const double* emitted, const double* eps, double rtol, double* absorbed,
                 double* stats, cudaStream_t s) {
  const int64_t n = op->n;
  // spectral bound of om G: max(1 - eps) (F_p is row-stochastic, similar to symmetric)
  std::vector<double> he(n);
  PR_CUDA(cudaMemcpyAsync(he.data(), eps, n * 8, cudaMemcpyDeviceToHost, s));
  PR_CUDA(cudaStreamSynchronize(s));
  double rho = 0.0;
  for (int64_t i = 0; i < n; ++i) rho = fmax(rho, 1.0 - he[i]);
  rho = fmin(fmax(rho, 1e-3), 0.999999);
  const double kappa = (1.0 + rho) / (1.0 - rho);
  const double q = (sqrt(kappa) - 1.0) / (sqrt(kappa) + 1.0);
  const double tol_in = 1.0e-5;
  int k_in = (int)ceil(log(tol_in / 2.0) / log(q));
  if (k_in < 2) k_in = 2;
  if (k_in > 400) k_in = 400;

  DevBuf<double> J, u, partial, sums;
  DevBuf<float> x32, r32, d32, ua, ub, sc32, ar32, om32;
  PR_TRY(J.alloc(n, s));
  PR_TRY(u.alloc(n, s));
  const int sb = spmv_slots(op->S);
  PR_TRY(partial.alloc((size_t)2 * sb, s));
  PR_TRY(sums.alloc(2, s));
  PR_TRY(x32.alloc(n, s));
  PR_TRY(r32.alloc(n, s));
  PR_TRY(d32.alloc(n, s));
  PR_TRY(ua.alloc(n, s));
  PR_TRY(ub.alloc(n, s));
  PR_TRY(sc32.alloc(n, s));
  PR_TRY(ar32.alloc(n, s));
  PR_TRY(om32.alloc(n, s));
  ::pr::launch_mark(), k_to_f32<<<grid_for(n, 256), 256, 0, s>>>(op->scale.ptr, op->area.ptr, eps, n, sc32.ptr, ar32.ptr, om32.ptr);
  PR_CUDA(cudaMemsetAsync(J.ptr, 0, n * 8, s));
  const float c_delta = (float)op->delta;
  const double sigma1 = 1.0 / rho;  // theta / delta with theta = 1, delta = rho
  int outer = 0;
  int64_t sp64 = 0, sp32 = 0;
  double rel = 0.0;
  for (;;) {
    ::pr::launch_mark(), k_refine_prep<<<grid_for(n, 256), 256, 0, s>>>(J.ptr, outer > 0 ? x32.ptr : nullptr, op->scale.ptr,
                                                    op->area.ptr, n, u.ptr);
    {
      const RefineEpi epi{op->delta, op->area.ptr, op->scale.ptr, eps, emitted, J.ptr, u.ptr, absorbed,
                          partial.ptr, x32.ptr, r32.ptr, d32.ptr, ua.ptr};
      int rc = PR_OK;
      ::pr::timer_begin(kTimerRefine, s);
      dispatch_mode(op->S.mode, [&](auto m) { rc = launch_spmv<decltype(m)::value, double>(op->S, u.ptr, epi, s); });
      ::pr::timer_end(kTimerRefine, s);
      PR_TRY(rc);
    }
    ++sp64;
    PR_TRY(sum_partials(partial.ptr, sb, 2, sums.ptr, s));
    double hs[2];
    PR_CUDA(cudaMemcpyAsync(hs, sums.ptr, 16, cudaMemcpyDeviceToHost, s));
    PR_CUDA(cudaStreamSynchronize(s));
    rel = hs[0] / fmax(hs[1], 2.2250738585072014e-308);
    if (rel <= rtol || outer >= 12) break;
    // binary32 Chebyshev correction
    double rho_k = 1.0 / sigma1;
    float* uin = ua.ptr;
    float* uout = ub.ptr;
    for (int k = 0; k < k_in; ++k) {
      const double rho_n = 1.0 / (2.0 * sigma1 - rho_k);
      const float c1 = (float)(rho_n * rho_k), c2 = (float)(2.0 * rho_n / rho);
      const ChebEpi epi{c_delta, sc32.ptr, ar32.ptr, om32.ptr, uin, uout, x32.ptr, r32.ptr, d32.ptr, c1, c2};
      int rc = PR_OK;
      ::pr::timer_begin(kTimerCheb, s);
      dispatch_mode(op->S.mode, [&](auto m) { rc = launch_spmv<decltype(m)::value, float>(op->S, uin, epi, s); });
      ::pr::timer_end(kTimerCheb, s);
      PR_TRY(rc);
      rho_k = rho_n;
      std::swap(uin, uout);
      ++sp32;
    }
    PR_CUDA(cudaGetLastError());
    ++outer;
  }
  op->spmv_calls += sp64 + sp32;
  if (!(rel <= rtol)) {
    set_error("mixed-precision radiosity did not reach the relative residual %.1e (%.1e)", rtol, rel);
    return PR_ERR_SERIES;
  }
  stats[0] = outer;
  stats[1] = (double)(sp64 + sp32);
  stats[2] = rel;
  stats[3] = k_in;
  return PR_OK;
}


static int field_channels(const pr_case* c, const pr_operator* op, const FieldSpec& f, int precision, double rtol,
                          double* q, double* coarse, double* stats, cudaStream_t s) {
  const int64_t n = c->n_patches;
  PR_ARG(op->n == n, "operator has %lld patches, geometry %lld", (long long)op->n, (long long)n);
  DevBuf<double> dE, de, dAb, partial, sums;
  PR_TRY(dE.alloc(n, s));
  PR_TRY(de.alloc(n, s));
  PR_TRY(dAb.alloc(n, s));
  const int rb = red_blocks();
  PR_TRY(partial.alloc((size_t)3 * rb, s));
  PR_TRY(sums.alloc(3, s));
  ::pr::launch_mark(), k_field_emission<<<grid_for(n, 256), 256, 0, s>>>(c->cls.ptr, c->cell.ptr, op->area.ptr, n,
                                                                         c->ny * c->nz, c->nx, f, dE.ptr, de.ptr);
  PR_CUDA(cudaGetLastError());
  double st[4] = {0, 0, 0, 0};
  if (precision == PR_PRECISION_MIXED) {
    PR_TRY(series_mixed(op, dE.ptr, de.ptr, rtol, dAb.ptr, st, s));
  } else {
    double res = 0.0;
    int64_t it = 0;
    const int64_t calls0 = op->spmv_calls;
    PR_TRY(series_fp64(op, dE.ptr, de.ptr, rtol, 10000, dAb.ptr, &res, &it, s));
    st[0] = (double)it;
    st[1] = (double)(op->spmv_calls - calls0);
    st[2] = res;
  }
  ::pr::launch_mark(), k_class_sums<<<rb, 256, 0, s>>>(c->cls.ptr, dAb.ptr, dE.ptr, n, partial.ptr);
  PR_CUDA(cudaGetLastError());
  PR_TRY(sum_partials(partial.ptr, rb, 3, sums.ptr, s));
  const double h = c->H / (double)c->nx;
  const double xs = (double)(c->ny * c->nz) * (h * h);
  DevBuf<double> dco;
  int bx = (int)std::min<int64_t>(8, c->nx), by = (int)std::min<int64_t>(8, c->ny), bz = (int)std::min<int64_t>(8, c->nz);
  if (coarse) {
    PR_TRY(dco.alloc((size_t)bx * by * bz, s));
    ::pr::launch_mark(), k_coarse<<<bx * by * bz, 256, 0, s>>>(c->cfp(), dAb.ptr, dE.ptr, c->nx, c->ny, c->nz, bx, by, bz, 1.0 / xs,
                                           dco.ptr);
    PR_CUDA(cudaGetLastError());
  }
  double hs[3];
  PR_CUDA(cudaMemcpyAsync(hs, sums.ptr, sizeof(hs), cudaMemcpyDeviceToHost, s));
  if (coarse) PR_CUDA(cudaMemcpyAsync(coarse, dco.ptr, dco.bytes(), cudaMemcpyDefault, s));
  PR_CUDA(cudaStreamSynchronize(s));
  const double qh = -hs[0] / xs, qc = -hs[1] / xs, qi = -hs[2] / xs;
  q[0] = qh;
  q[1] = qc;
  q[2] = qi;
  q[3] = fabs(qh + qc + qi) / fmax(fmax(fabs(qh), fabs(qc)), fmax(fabs(qi), 1.0e-30));
  if (stats) for (int k = 0; k < 4; ++k) stats[k] = st[k];
  return PR_OK;
}

int prescribed_channels(const pr_case* c, const pr_operator* op, double T_m, double dT, double epsv, int precision,
                        double rtol, double* q, double* coarse, double* stats, cudaStream_t s) {
  FieldSpec f{nullptr, T_m, dT, T_m + dT / 2.0, T_m - dT / 2.0, epsv, T_m, 1};
  return field_channels(c, op, f, precision, rtol, q, coarse, stats, s);
}

int cell_field_channels(const pr_case* c, const pr_operator* op, const double* T_cells, double Th, double Tc,
                        double epsv, int has_ref, double ref, int precision, double rtol, double* q, double* coarse,
                        double* stats, cudaStream_t s) {
  DevBuf<double> dT;
  PR_TRY(dT.alloc(c->n_cells, s));
  PR_CUDA(cudaMemcpyAsync(dT.ptr, T_cells, c->n_cells * 8, cudaMemcpyDefault, s));
  FieldSpec f{dT.ptr, 0.0, 0.0, Th, Tc, epsv, ref, has_ref};
  return field_channels(c, op, f, precision, rtol, q, coarse, stats, s);
}

}  // namespace pr

// ------------------------------------------------------------------ reflection series without allocation
//
// For callers that cannot call cudaMalloc: a host whose device memory is owned by
// another allocator (a framework pool that reserves the GPU's memory up front), or a
// caller that must not take the allocator's implicit synchronisation in the middle of
// its own stream work.  The scratch of the series (two ping-pong vectors, block
// partial sums and the convergence state) lives in one file-scope device array
// instead, sized for at most kNoAllocMaxPatches patches.
namespace pr {

static constexpr int64_t kNoAllocMaxPatches = 262144;  // 2 x 262144 x 8 B of vectors
// Block partial sums, two values per block.  The series launches at most 8 blocks per SM (the
// products of operators of at most kNoAllocMaxPatches rows: max(SMs, 86) blocked CTAs or 8 per SM
// warp-per-row blocks; 4 per SM for the reductions), so 2 x 8 x 296 values cover GPUs of up to
// 296 SMs (B200: 148).  A launch that would need more is rejected with PR_ERR_LIMIT below.
static constexpr int64_t kNoAllocMaxSms = 296;
static constexpr int64_t kNoAllocPartials = 2 * 8 * kNoAllocMaxSms;
static constexpr int64_t kNoAllocDoubles = 2 * kNoAllocMaxPatches + kNoAllocPartials + 8;

static __device__ __align__(256) double g_series_scratch[kNoAllocDoubles];

// Device address of the scratch array on the current device, looked up once per device.
static int noalloc_scratch(double** out) {
  static std::mutex mu;
  static double* addr[64] = {nullptr};
  int dev = 0;
  PR_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) {
    set_error("device %d outside the supported range", dev);
    return PR_ERR_LIMIT;
  }
  std::lock_guard<std::mutex> lk(mu);
  if (!addr[dev]) {
    void* p = nullptr;
    PR_CUDA(cudaGetSymbolAddress(&p, g_series_scratch));
    addr[dev] = (double*)p;
  }
  *out = addr[dev];
  return PR_OK;
}


static int series_fp64_noalloc(const pr_operator* op, const double* emitted, const double* eps, double rtol,
                               int64_t max_it, double* absorbed, double* residual, int64_t* iterations,
                               cudaStream_t s) {
  const int64_t n = op->n;
  if (n > kNoAllocMaxPatches) {
    set_error("pr_reflection_series_noalloc: %lld patches exceed the %lld of its static scratch; use "
              "pr_reflection_series", (long long)n, (long long)kNoAllocMaxPatches);
    return PR_ERR_LIMIT;
  }
  const int rb = red_blocks();
  const int sb = spmv_slots(op->S);
  if ((int64_t)2 * (sb > rb ? sb : rb) > kNoAllocPartials) {
    set_error("pr_reflection_series_noalloc: %d blocks exceed its partial-sum scratch", sb > rb ? sb : rb);
    return PR_ERR_LIMIT;
  }
  double* base = nullptr;
  PR_TRY(noalloc_scratch(&base));
  double* va = base;
  double* vb = base + kNoAllocMaxPatches;
  double* partial = base + 2 * kNoAllocMaxPatches;
  SeriesState* st = (SeriesState*)(base + 2 * kNoAllocMaxPatches + kNoAllocPartials);
  // the array keeps the previous call's contents: the convergence state must start at zero
  PR_CUDA(cudaMemsetAsync(st, 0, sizeof(SeriesState), s));
  if (n == 0) {
    *residual = 0.0;
    *iterations = 0;
    return PR_OK;
  }
  ::pr::launch_mark(), k_series_init<<<rb, 256, 0, s>>>(emitted, op->scale.ptr, op->area.ptr, n, va, absorbed, partial);
  PR_CUDA(cudaGetLastError());
  ::pr::launch_mark(), k_series_tol<<<1, 32, 0, s>>>(partial, rb, rtol, st);
  PR_CUDA(cudaGetLastError());
  double* vin = va;
  double* vout = vb;
  SeriesState h;
  int batch = 4;
  for (;;) {
    for (int b = 0; b < batch; ++b) {
      const SeriesEpi epi{op->delta, op->area.ptr, op->scale.ptr, eps, vin, vout, absorbed, partial, st};
      int rc = PR_OK;
      dispatch_mode(op->S.mode, [&](auto m) { rc = launch_spmv<decltype(m)::value, double>(op->S, vin, epi, s); });
      PR_TRY(rc);
      ::pr::launch_mark(), k_series_finish<<<1, 32, 0, s>>>(partial, sb, (long long)max_it, st);
      std::swap(vin, vout);
    }
    PR_CUDA(cudaGetLastError());
    PR_CUDA(cudaMemcpyAsync(&h, st, sizeof(h), cudaMemcpyDeviceToHost, s));
    PR_CUDA(cudaStreamSynchronize(s));
    if (h.done) break;
    if (batch < 64) batch *= 2;
  }
  op->spmv_calls += h.iters;
  if (h.done == 2) {
    set_error("radiosity reflection series did not converge");
    return PR_ERR_SERIES;
  }
  *residual = h.residual;
  *iterations = h.iters;
  return PR_OK;
}

}  // namespace pr

extern "C" PR_API int pr_reflection_series_noalloc(const pr_operator* op, const double* emitted,
                                                   const double* emissivity, double relative_tolerance,
                                                   int64_t max_reflections, double* absorbed,
                                                   double* residual_power, int64_t* iterations, void* stream) {
  using namespace pr;
  if (!op || !emitted || !emissivity || !absorbed) {
    set_error("pr_reflection_series_noalloc: operator, emitted, emissivity and absorbed must not be NULL");
    return PR_ERR_ARG;
  }
  if (max_reflections < 1) {
    set_error("max_reflections must be at least 1");
    return PR_ERR_ARG;
  }
  DeviceGuard guard(op->device);
  if (!is_device_pointer_of(emitted, op->device) || !is_device_pointer_of(emissivity, op->device) ||
      !is_device_pointer_of(absorbed, op->device)) {
    set_error("pr_reflection_series_noalloc: emitted, emissivity and absorbed must be device memory of the "
              "operator's device %d", op->device);
    return PR_ERR_ARG;
  }
  double res = 0.0;
  int64_t it = 0;
  const int st = series_fp64_noalloc(op, emitted, emissivity, relative_tolerance, max_reflections, absorbed, &res,
                                     &it, (cudaStream_t)stream);
  if (residual_power) *residual_power = res;
  if (iterations) *iterations = it;
  return st;
}
