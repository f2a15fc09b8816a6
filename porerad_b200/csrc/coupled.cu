// Heat conduction on the voxel grid (porerad/conduction.py) and the strictly coupled
// radiation-conduction solve (porerad/coupled.py:222-447) on the device.
//
// The conduction matrix A is never stored as a general sparse matrix: each cell keeps the
// conductance of its +x, +y and +z face (harmonic mean of the two cells' conductivities
// times dx^2 / dx, conduction.py:55-57, 72-74; y and z periodic, conduction.py:80-83), the
// diagonal accumulated face by face in the order conduction.py:79-91 adds them, and its
// hot/cold wall responses 2 k dx (conduction.py:85-90).  A x is a 7-point stencil.
//
// The Newton-Krylov solve follows coupled.py:340-421: R(T) = A T - b - Q_rad(T);
// corrections by flexible GMRES (restart 30, at most 90 iterations, coupled.py:230-290) on
// the Jacobian-vector product A v - dQ_rad(v) (the radiosity JVP, coupled.py:108-123),
// right-preconditioned by a fixed number of Jacobi-PCG steps on A + diag(emission
// derivative at the initial field) (coupled.py:293-320); a backtracking line search keeps
// every trial field within the wall temperatures (coupled.py:392-408).  All vectors stay on
// the device; the host holds the GMRES Hessenberg (at most 31 x 30) and the scalars.
// Orthogonalisation: two classical Gram-Schmidt passes per column (each one multi-dot, one
// update), the same two projections as the reference's modified Gram-Schmidt with one
// reorthogonalisation; the small least-squares problem is solved by Givens rotations.
// Every reduction is a fixed-order sum of block partials, so a solve is reproducible bit
// for bit on a given device.
#include <cmath>
#include <vector>

#include "pr_spmv.cuh"

namespace pr {

int series_fp64(const pr_operator* op, const double* emitted, const double* eps, double rtol, int64_t max_it,
                double* absorbed, double* residual, int64_t* iterations, cudaStream_t s);

#define PR_SIGMA_C 5.670374419e-8  // porerad/constants.py:3

constexpr int kRedBlocks = 592;  // block partials of every reduction (4 per SM)

// ------------------------------------------------------------------ conduction assembly

__device__ __forceinline__ double harmonic(double lo, double hi) { return 2.0 * lo * hi / (lo + hi + 1.0e-30); }

// Face conductances, wall responses and the diagonal of A, one thread per cell.
__global__ void k_cond_assemble(const double* __restrict__ k, int64_t nx, int64_t ny, int64_t nz, double dx,
                                double* __restrict__ gx, double* __restrict__ gy, double* __restrict__ gz,
                                double* __restrict__ hot, double* __restrict__ cold) {
  const int64_t n = nx * ny * nz, nyz = ny * nz;
  const double area = dx * dx;
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = c / nyz, j = (c / nz) % ny, kk = c % nz;
    const int64_t cyp = j + 1 < ny ? c + nz : c - (ny - 1) * nz;
    const int64_t czp = kk + 1 < nz ? c + 1 : c - (nz - 1);
    gx[c] = i + 1 < nx ? harmonic(k[c], k[c + nyz]) * area / dx : 0.0;
    gy[c] = harmonic(k[c], k[cyp]) * area / dx;
    gz[c] = harmonic(k[c], k[czp]) * area / dx;
    const double face_scale = dx * dx / dx;
    hot[c] = i == 0 ? 2.0 * k[c] * face_scale : 0.0;
    cold[c] = i == nx - 1 ? 2.0 * k[c] * face_scale : 0.0;
  }
}

// diag = the face conductances in the order conduction.py:79-83 adds them (each face to its
// low cell, then to its high cell), then + (hot + cold) (conduction.py:91).
__global__ void k_cond_diagonal(const double* __restrict__ gx, const double* __restrict__ gy,
                                const double* __restrict__ gz, const double* __restrict__ hot,
                                const double* __restrict__ cold, int64_t nx, int64_t ny, int64_t nz,
                                double* __restrict__ diag) {
  const int64_t n = nx * ny * nz, nyz = ny * nz;
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = c / nyz, j = (c / nz) % ny, kk = c % nz;
    double d = 0.0;
    if (i + 1 < nx) d += gx[c];
    if (i > 0) d += gx[c - nyz];
    if (j + 1 < ny) d += gy[c];
    if (j > 0) d += gy[c - nz];
    if (j == ny - 1) d += gy[c];                 // wrap face (j = ny-1 | j = 0), low side
    if (j == 0) d += gy[c + (ny - 1) * nz];      // high side
    if (kk + 1 < nz) d += gz[c];
    if (kk > 0) d += gz[c - 1];
    if (kk == nz - 1) d += gz[c];
    if (kk == 0) d += gz[c + nz - 1];
    diag[c] = d + (hot[c] + cold[c]);
  }
}

struct CondView {
  const double* __restrict__ gx;
  const double* __restrict__ gy;
  const double* __restrict__ gz;
  const double* __restrict__ diag;
  const double* __restrict__ hot;
  const double* __restrict__ cold;
  int64_t nx, ny, nz;
};

inline CondView cond_view(const pr_conduction* A) {
  return CondView{A->gx.ptr, A->gy.ptr, A->gz.ptr, A->diag.ptr, A->hot.ptr, A->cold.ptr, A->nx, A->ny, A->nz};
}

__device__ __forceinline__ double cond_row(const CondView& A, const double* __restrict__ x, int64_t c) {
  const int64_t nyz = A.ny * A.nz;
  const int64_t i = c / nyz, j = (c / A.nz) % A.ny, kk = c % A.nz;
  const int64_t cym = j > 0 ? c - A.nz : c + (A.ny - 1) * A.nz, cyp = j + 1 < A.ny ? c + A.nz : c - (A.ny - 1) * A.nz;
  const int64_t czm = kk > 0 ? c - 1 : c + A.nz - 1, czp = kk + 1 < A.nz ? c + 1 : c - (A.nz - 1);
  double s = A.diag[c] * x[c];
  if (i + 1 < A.nx) s -= A.gx[c] * x[c + nyz];
  if (i > 0) s -= A.gx[c - nyz] * x[c - nyz];
  s -= A.gy[c] * x[cyp];
  s -= A.gy[cym] * x[cym];
  s -= A.gz[c] * x[czp];
  s -= A.gz[czm] * x[czm];
  return s;
}

// y = A x (+ shift x); r = A x - (hot Th + cold Tc) - q when q != nullptr (the Newton residual).
__global__ void k_cond_apply(CondView A, const double* __restrict__ x, const double* __restrict__ shift,
                             double* __restrict__ y) {
  const int64_t n = A.nx * A.ny * A.nz;
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
    double s = cond_row(A, x, c);
    if (shift) s += shift[c] * x[c];
    y[c] = s;
  }
}

__global__ void k_residual(CondView A, const double* __restrict__ T, double Th, double Tc,
                           const double* __restrict__ q, double* __restrict__ r) {
  const int64_t n = A.nx * A.ny * A.nz;
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
    const double b = A.hot[c] * Th + A.cold[c] * Tc;
    r[c] = cond_row(A, T, c) - b - q[c];
  }
}

// ------------------------------------------------------------------ vector kernels

// block partials of a . b
__global__ void __launch_bounds__(256) k_dot(const double* __restrict__ a, const double* __restrict__ b, int64_t n,
                                             double* __restrict__ partial) {
  double acc[1] = {0.0};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    acc[0] = fma(a[i], b[i], acc[0]);
  block_sum_store<1>(acc, partial);
}

// block partials of V_r . w for r < m (V rows of length n, stride n), m <= 32
__global__ void __launch_bounds__(256) k_multidot(const double* __restrict__ V, int m, const double* __restrict__ w,
                                                  int64_t n, double* __restrict__ partial) {
  double acc[32];
#pragma unroll
  for (int r = 0; r < 32; ++r) acc[r] = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double wi = w[i];
#pragma unroll
    for (int r = 0; r < 32; ++r)
      if (r < m) acc[r] = fma(V[(int64_t)r * n + i], wi, acc[r]);
  }
  block_sum_store<32>(acc, partial);
}

// w -= sum_r h[r] V_r (h on the device)
__global__ void k_multi_axpy(const double* __restrict__ V, int m, const double* __restrict__ h, int64_t n,
                             double* __restrict__ w) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double v = w[i];
    for (int r = 0; r < m; ++r) v -= h[r] * V[(int64_t)r * n + i];
    w[i] = v;
  }
}

// y = a x + b y (host scalars)
__global__ void k_axpby(double a, const double* __restrict__ x, double b, double* __restrict__ y, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] = a * x[i] + b * y[i];
}

// out = x + a y
__global__ void k_add_scaled(const double* __restrict__ x, double a, const double* __restrict__ y, int64_t n,
                             double* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = x[i] + a * y[i];
}

__global__ void k_negate(const double* __restrict__ x, int64_t n, double* __restrict__ y) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] = -x[i];
}

// Block partials of (sum x^2, max |x|, min x, max x, number of non-finite entries) of x
// (or of x - y when y != nullptr).
__global__ void __launch_bounds__(256) k_vstats(const double* __restrict__ x, const double* __restrict__ y, int64_t n,
                                                double* __restrict__ partial) {
  double ss = 0.0, ma = 0.0, mn = INFINITY, mx = -INFINITY, bad = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double v = y ? x[i] - y[i] : x[i];
    if (!isfinite(v)) {
      bad += 1.0;
      continue;
    }
    ss = fma(v, v, ss);
    ma = fmax(ma, fabs(v));
    mn = fmin(mn, v);
    mx = fmax(mx, v);
  }
  __shared__ double red[5][8];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int o = 16; o > 0; o >>= 1) {
    ss += __shfl_xor_sync(PR_FULL, ss, o);
    ma = fmax(ma, __shfl_xor_sync(PR_FULL, ma, o));
    mn = fmin(mn, __shfl_xor_sync(PR_FULL, mn, o));
    mx = fmax(mx, __shfl_xor_sync(PR_FULL, mx, o));
    bad += __shfl_xor_sync(PR_FULL, bad, o);
  }
  if (lane == 0) {
    red[0][wid] = ss;
    red[1][wid] = ma;
    red[2][wid] = mn;
    red[3][wid] = mx;
    red[4][wid] = bad;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, b = 0.0, c = INFINITY, d = -INFINITY, e = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      a += red[0][w];
      b = fmax(b, red[1][w]);
      c = fmin(c, red[2][w]);
      d = fmax(d, red[3][w]);
      e += red[4][w];
    }
    double* o = partial + 5 * (int64_t)blockIdx.x;
    o[0] = a;
    o[1] = b;
    o[2] = c;
    o[3] = d;
    o[4] = e;
  }
}

// one warp, fixed order (warp_sum_partials for the sums; min and max do not depend on it)
__global__ void k_vstats_final(const double* __restrict__ partial, int blocks, double* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const double a = warp_sum_partials(partial, blocks, 5, 0, lane);
  const double e = warp_sum_partials(partial, blocks, 5, 4, lane);
  double b = 0.0, c = INFINITY, d = -INFINITY;
  for (int k = lane; k < blocks; k += 32) {
    const double* p = partial + 5 * (int64_t)k;
    b = fmax(b, p[1]);
    c = fmin(c, p[2]);
    d = fmax(d, p[3]);
  }
  for (int o = 16; o > 0; o >>= 1) {
    b = fmax(b, __shfl_xor_sync(PR_FULL, b, o));
    c = fmin(c, __shfl_xor_sync(PR_FULL, c, o));
    d = fmax(d, __shfl_xor_sync(PR_FULL, d, o));
  }
  if (lane != 0) return;
  out[0] = a;
  out[1] = b;
  out[2] = c;
  out[3] = d;
  out[4] = e;
}

// ------------------------------------------------------------------ PCG kernels (device scalars)

// PCG scalars: rz, pAp, rz_new, rr, tol2 (squared stopping norm), done, iterations
struct PcgScalars {
  double rz, pAp, rz_new, rr, tol2;
  int done;
  int pad;
  long long iterations;
};

// Ap = (A + diag(shift)) p and block partials of p . Ap
__global__ void __launch_bounds__(256) k_pcg_apply(CondView A, const double* __restrict__ shift,
                                                   const double* __restrict__ p, double* __restrict__ Ap,
                                                   double* __restrict__ partial, const PcgScalars* __restrict__ st) {
  if (st->done) return;
  const int64_t n = A.nx * A.ny * A.nz;
  double acc[1] = {0.0};
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
    double s = cond_row(A, p, c);
    if (shift) s += shift[c] * p[c];
    Ap[c] = s;
    acc[0] = fma(p[c], s, acc[0]);
  }
  block_sum_store<1>(acc, partial);
}

// alpha = rz / pAp;  x += alpha p;  r -= alpha Ap;  z = r / (diag + shift);  partials of r . z and r . r
__global__ void __launch_bounds__(256) k_pcg_update(const double* __restrict__ diag, const double* __restrict__ shift,
                                                    int64_t n, const double* __restrict__ p,
                                                    const double* __restrict__ Ap, double* __restrict__ x,
                                                    double* __restrict__ r, double* __restrict__ z,
                                                    double* __restrict__ partial, const PcgScalars* __restrict__ st) {
  if (st->done) return;
  const double alpha = st->rz / st->pAp;
  double acc[2] = {0.0, 0.0};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    x[i] += alpha * p[i];
    const double ri = r[i] - alpha * Ap[i];
    r[i] = ri;
    const double zi = ri * (1.0 / (diag[i] + (shift ? shift[i] : 0.0)));
    z[i] = zi;
    acc[0] = fma(ri, zi, acc[0]);
    acc[1] = fma(ri, ri, acc[1]);
  }
  block_sum_store<2>(acc, partial);
}

// one warp: reduce the partials of p . Ap into st->pAp
__global__ void k_pcg_take_pAp(const double* __restrict__ partial, int blocks, PcgScalars* __restrict__ st) {
  if (st->done) return;
  const double a = warp_sum_partials(partial, blocks, 1, 0, threadIdx.x & 31);
  if (threadIdx.x == 0) st->pAp = a;
}

// one warp: r . z and r . r of the step; the convergence test (when tol2 > 0)
__global__ void k_pcg_take_rz(const double* __restrict__ partial, int blocks, PcgScalars* __restrict__ st) {
  if (st->done) return;
  const int lane = threadIdx.x & 31;
  const double a = warp_sum_partials(partial, blocks, 2, 0, lane);
  const double b = warp_sum_partials(partial, blocks, 2, 1, lane);
  if (lane != 0) return;
  st->rz_new = a;
  st->rr = b;
  st->iterations += 1;
  if (st->tol2 > 0.0 && b <= st->tol2) st->done = 1;
}

// p = z + (rz_new / rz) p;  rz = rz_new
__global__ void k_pcg_direction(const double* __restrict__ z, int64_t n, double* __restrict__ p,
                                PcgScalars* __restrict__ st) {
  if (st->done) return;
  const double beta = st->rz_new / st->rz;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    p[i] = z[i] + beta * p[i];
}

__global__ void k_pcg_roll(PcgScalars* __restrict__ st) {
  if (threadIdx.x == 0 && !st->done) st->rz = st->rz_new;
}

// start: r = rhs - A x (x given) or r = rhs (x = 0); z = r / (diag + shift); p = z; partials of r . z, r . r
__global__ void __launch_bounds__(256) k_pcg_start(CondView A, const double* __restrict__ shift,
                                                   const double* __restrict__ rhs, double* __restrict__ x, int zero_x,
                                                   double* __restrict__ r, double* __restrict__ z,
                                                   double* __restrict__ p, double* __restrict__ partial) {
  const int64_t n = A.nx * A.ny * A.nz;
  double acc[2] = {0.0, 0.0};
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
    double ri;
    if (zero_x) {
      x[c] = 0.0;
      ri = rhs[c];
    } else {
      double s = cond_row(A, x, c);
      if (shift) s += shift[c] * x[c];
      ri = rhs[c] - s;
    }
    r[c] = ri;
    const double zi = ri * (1.0 / (A.diag[c] + (shift ? shift[c] : 0.0)));
    z[c] = zi;
    p[c] = zi;
    acc[0] = fma(ri, zi, acc[0]);
    acc[1] = fma(ri, ri, acc[1]);
  }
  block_sum_store<2>(acc, partial);
}

__global__ void k_pcg_init_scalars(const double* __restrict__ partial, int blocks, double tol2,
                                   PcgScalars* __restrict__ st) {
  const int lane = threadIdx.x & 31;
  const double a = warp_sum_partials(partial, blocks, 2, 0, lane);
  const double b = warp_sum_partials(partial, blocks, 2, 1, lane);
  if (lane != 0) return;
  st->rz = a;
  st->rr = b;
  st->tol2 = tol2;
  st->iterations = 0;
  st->done = (tol2 > 0.0 && b <= tol2) ? 1 : 0;
}

// ------------------------------------------------------------------ radiation on cells

// Patch temperatures (coupled.py:45-53): walls at Th / Tc, internal patches at their cell.
__global__ void k_patch_temperature(const int8_t* __restrict__ cls, const int32_t* __restrict__ cell,
                                    const double* __restrict__ T_cells, double Th, double Tc, int64_t n,
                                    double* __restrict__ Tp) {
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
    const int c = cls[p];
    Tp[p] = c == 0 ? Th : (c == 1 ? Tc : T_cells[cell[p]]);
  }
}

// eps sigma A T^4 (exchange.py:266-267)
__global__ void k_emission_t4(const double* __restrict__ Tp, double eps, const double* __restrict__ area, int64_t n,
                              double* __restrict__ e) {
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x)
    e[p] = eps * PR_SIGMA_C * area[p] * pow(Tp[p], 4.0);
}

// 4 eps sigma A T^3 dT with dT of internal patches from their cell, 0 on walls (coupled.py:116-118,
// exchange.py:285)
__global__ void k_emission_jvp(const int8_t* __restrict__ cls, const int32_t* __restrict__ cell,
                               const double* __restrict__ Tp, const double* __restrict__ dT_cells, double eps,
                               const double* __restrict__ area, int64_t n, double* __restrict__ e) {
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
    const double d = cls[p] == 2 ? dT_cells[cell[p]] : 0.0;
    e[p] = 4.0 * eps * PR_SIGMA_C * area[p] * pow(Tp[p], 3.0) * d;
  }
}

// cell power = sum over the cell's internal patches (faces in order) of absorbed - emitted
// (coupled.py:56-62; patch ids of a cell ascend with the face, as np.add.at visits them)
__global__ void k_cell_power(const int32_t* __restrict__ cfp, const double* __restrict__ ab,
                             const double* __restrict__ e, int64_t n_cells, double* __restrict__ q) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n_cells; c += (int64_t)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int f = 0; f < 6; ++f) {
      const int32_t p = cfp[c * 6 + f];
      if (p >= 0) s += ab[p] - e[p];
    }
    q[c] = s;
  }
}

// emission derivative of every cell: sum over its internal patches of 4 eps sigma A_p T_c^3 (coupled.py:65-73)
__global__ void k_emission_diagonal(const int32_t* __restrict__ cfp, const double* __restrict__ area,
                                    const double* __restrict__ T_cells, double eps, int64_t n_cells,
                                    double* __restrict__ out) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n_cells; c += (int64_t)gridDim.x * blockDim.x) {
    double s = 0.0;
    const double t3 = pow(T_cells[c], 3.0);
    for (int f = 0; f < 6; ++f) {
      const int32_t p = cfp[c * 6 + f];
      if (p >= 0) s += 4.0 * eps * PR_SIGMA_C * area[p] * t3;
    }
    out[c] = s;
  }
}

// net = ab - e per patch; block partials of the class sums (hot, cold, internal) and of the total
__global__ void __launch_bounds__(256) k_net_sums(const int8_t* __restrict__ cls, const double* __restrict__ ab,
                                                  const double* __restrict__ e, int64_t n, double* __restrict__ net,
                                                  double* __restrict__ partial) {
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
    const double v = ab[p] - e[p];
    if (net) net[p] = v;
    const int c = cls[p];
    acc[c == 0 ? 0 : (c == 1 ? 1 : 2)] += v;
    acc[3] += v;
  }
  block_sum_store<4>(acc, partial);
}

// mean over (j, k) of the conductive wall fluxes 2 k (Th - T[0]) / dx and 2 k (T[-1] - Tc) / dx
// (conduction.py:43-50): block partials of the two sums
__global__ void __launch_bounds__(256) k_wall_flux(const double* __restrict__ k, const double* __restrict__ T,
                                                   int64_t nx, int64_t nyz, double dx, double Th, double Tc,
                                                   double* __restrict__ partial) {
  double acc[2] = {0.0, 0.0};
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nyz; t += (int64_t)gridDim.x * blockDim.x) {
    acc[0] += 2.0 * k[t] * (Th - T[t]) / dx;
    const int64_t c = (nx - 1) * nyz + t;
    acc[1] += 2.0 * k[c] * (T[c] - Tc) / dx;
  }
  block_sum_store<2>(acc, partial);
}

// linear profile between the walls (conduction.py:109-110)
__global__ void k_linear_profile(int64_t nx, int64_t nyz, double Th, double Tc, double* __restrict__ T) {
  const int64_t n = nx * nyz;
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = c / nyz;
    T[c] = Th + (Tc - Th) * (((double)i + 0.5) / (double)nx);
  }
}

// block partials of the number of entries outside [lo, hi]
__global__ void __launch_bounds__(256) k_count_outside(const double* __restrict__ x, int64_t n, double lo, double hi,
                                                       double* __restrict__ partial) {
  double acc[1] = {0.0};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    acc[0] += (x[i] < lo || x[i] > hi) ? 1.0 : 0.0;
  block_sum_store<1>(acc, partial);
}

__global__ void k_fill(double* __restrict__ x, int64_t n, double v) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) x[i] = v;
}

// ------------------------------------------------------------------ host helpers

static int grid_n(int64_t n) { return grid_for(n, 256, sm_count() * 16); }

// Fixed-order reductions with the result copied to the host.
struct Reducer {
  DevBuf<double> partial, out;
  std::vector<double> host;
  int init(cudaStream_t s) {
    PR_TRY(partial.alloc((size_t)kRedBlocks * 32, s));
    PR_TRY(out.alloc(32, s));
    host.assign(32, 0.0);
    return PR_OK;
  }
  int dot(const double* a, const double* b, int64_t n, double* r, cudaStream_t s) {
    ::pr::launch_mark(), k_dot<<<kRedBlocks, 256, 0, s>>>(a, b, n, partial.ptr);
    PR_CUDA(cudaGetLastError());
    PR_TRY(sum_partials(partial.ptr, kRedBlocks, 1, out.ptr, s));
    PR_CUDA(cudaMemcpyAsync(r, out.ptr, 8, cudaMemcpyDeviceToHost, s));
    PR_CUDA(cudaStreamSynchronize(s));
    return PR_OK;
  }
  // (sum of squares, max |.|, min, max, non-finite count) of x (- y)
  int stats(const double* x, const double* y, int64_t n, double* r5, cudaStream_t s) {
    ::pr::launch_mark(), k_vstats<<<kRedBlocks, 256, 0, s>>>(x, y, n, partial.ptr);
    PR_CUDA(cudaGetLastError());
    ::pr::launch_mark(), k_vstats_final<<<1, 32, 0, s>>>(partial.ptr, kRedBlocks, out.ptr);
    PR_CUDA(cudaGetLastError());
    PR_CUDA(cudaMemcpyAsync(r5, out.ptr, 5 * 8, cudaMemcpyDeviceToHost, s));
    PR_CUDA(cudaStreamSynchronize(s));
    return PR_OK;
  }
  // V_r . w, r < m, into device h (m doubles) and the host copy
  int multidot(const double* V, int m, const double* w, int64_t n, double* h_dev, double* h_host, cudaStream_t s) {
    ::pr::launch_mark(), k_multidot<<<kRedBlocks, 256, 0, s>>>(V, m, w, n, partial.ptr);
    PR_CUDA(cudaGetLastError());
    PR_TRY(sum_partials(partial.ptr, kRedBlocks, 32, h_dev, s));
    PR_CUDA(cudaMemcpyAsync(h_host, h_dev, (size_t)m * 8, cudaMemcpyDeviceToHost, s));
    PR_CUDA(cudaStreamSynchronize(s));
    return PR_OK;
  }
};

// A CUDA graph captured on a private stream (capture is not allowed on the legacy default
// stream) and launched on the caller's stream; rebuilt when its key changes.
struct CapturedGraph {
  cudaGraphExec_t exec = nullptr;
  cudaStream_t cap = nullptr;
  long long key = -1;
  ~CapturedGraph() {
    if (exec) cudaGraphExecDestroy(exec);
    if (cap) cudaStreamDestroy(cap);
  }
  template <class F>
  int ensure(long long k, F&& record) {
    if (exec && key == k) return PR_OK;
    if (exec) {
      cudaGraphExecDestroy(exec);
      exec = nullptr;
    }
    if (!cap) PR_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    PR_CUDA(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
    const int st = record(cap);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(cap, &g);
    if (st != PR_OK) {
      if (g) cudaGraphDestroy(g);
      return st;
    }
    PR_CUDA(e);
    const cudaError_t ei = cudaGraphInstantiate(&exec, g, 0);
    cudaGraphDestroy(g);
    PR_CUDA(ei);
    key = k;
    return PR_OK;
  }
  int launch(cudaStream_t s) {
    PR_CUDA(cudaGraphLaunch(exec, s));
    return PR_OK;
  }
};

// Jacobi-preconditioned CG on (A + diag(shift)) x = rhs.  steps > 0: exactly that many steps
// from x = 0, no convergence test (coupled.py:293-320).  steps == 0: from the given x until
// ||r||_2 <= tol (checked on the device, polled by the host), at most max_it steps.  Both run
// as CUDA graphs of their fixed launch sequences (a preconditioner application is about 60
// small launches).
struct Pcg {
  DevBuf<double> r, z, p, Ap, partial, gin, gout;
  DevBuf<PcgScalars> st;
  CapturedGraph fixed_graph, batch_graph;
  int64_t n = 0;
  int init(int64_t n_, cudaStream_t s) {
    n = n_;
    PR_TRY(r.alloc(n, s));
    PR_TRY(z.alloc(n, s));
    PR_TRY(p.alloc(n, s));
    PR_TRY(Ap.alloc(n, s));
    PR_TRY(gin.alloc(n, s));
    PR_TRY(gout.alloc(n, s));
    PR_TRY(partial.alloc((size_t)kRedBlocks * 2, s));
    PR_TRY(st.alloc(1, s));
    return PR_OK;
  }
  int step(const CondView& A, const double* shift, double* x, cudaStream_t s, bool direction) {
    const int g = grid_n(n);
    ::pr::launch_mark(), k_pcg_apply<<<kRedBlocks, 256, 0, s>>>(A, shift, p.ptr, Ap.ptr, partial.ptr, st.ptr);
    ::pr::launch_mark(), k_pcg_take_pAp<<<1, 32, 0, s>>>(partial.ptr, kRedBlocks, st.ptr);
    ::pr::launch_mark(), k_pcg_update<<<kRedBlocks, 256, 0, s>>>(A.diag, shift, n, p.ptr, Ap.ptr, x, r.ptr, z.ptr,
                                                                 partial.ptr, st.ptr);
    ::pr::launch_mark(), k_pcg_take_rz<<<1, 32, 0, s>>>(partial.ptr, kRedBlocks, st.ptr);
    if (direction) {
      ::pr::launch_mark(), k_pcg_direction<<<g, 256, 0, s>>>(z.ptr, n, p.ptr, st.ptr);
      ::pr::launch_mark(), k_pcg_roll<<<1, 32, 0, s>>>(st.ptr);
    }
    PR_CUDA(cudaGetLastError());
    return PR_OK;
  }
  int fixed_seq(const CondView& A, const double* shift, const double* rhs, int steps, double* x, cudaStream_t s) {
    ::pr::launch_mark(), k_pcg_start<<<kRedBlocks, 256, 0, s>>>(A, shift, rhs, x, 1, r.ptr, z.ptr, p.ptr, partial.ptr);
    ::pr::launch_mark(), k_pcg_init_scalars<<<1, 32, 0, s>>>(partial.ptr, kRedBlocks, 0.0, st.ptr);
    PR_CUDA(cudaGetLastError());
    for (int k = 0; k < steps; ++k) PR_TRY(step(A, shift, x, s, k + 1 < steps));
    return PR_OK;
  }
  // x = (steps of PCG from 0)(rhs): the captured sequence between a copy in and a copy out
  int fixed(const CondView& A, const double* shift, const double* rhs, int steps, double* x, cudaStream_t s) {
    PR_TRY(fixed_graph.ensure(((long long)steps << 1) ^ (long long)(uintptr_t)shift, [&](cudaStream_t c) -> int {
      return fixed_seq(A, shift, gin.ptr, steps, gout.ptr, c);
    }));
    PR_CUDA(cudaMemcpyAsync(gin.ptr, rhs, n * 8, cudaMemcpyDeviceToDevice, s));
    PR_TRY(fixed_graph.launch(s));
    PR_CUDA(cudaMemcpyAsync(x, gout.ptr, n * 8, cudaMemcpyDeviceToDevice, s));
    return PR_OK;
  }
  int solve(const CondView& A, const double* shift, const double* rhs, double tol, int64_t max_it, double* x,
            PcgScalars* out, cudaStream_t s) {
    ::pr::launch_mark(), k_pcg_start<<<kRedBlocks, 256, 0, s>>>(A, shift, rhs, x, 0, r.ptr, z.ptr, p.ptr, partial.ptr);
    ::pr::launch_mark(), k_pcg_init_scalars<<<1, 32, 0, s>>>(partial.ptr, kRedBlocks, tol * tol, st.ptr);
    PR_CUDA(cudaGetLastError());
    // graphs of 32 steps (steps after convergence return at once), polled every 1, 2, 4, 8 graphs
    constexpr int kGraphSteps = 32;
    PR_TRY(batch_graph.ensure((long long)(uintptr_t)x ^ ((long long)(uintptr_t)shift << 1), [&](cudaStream_t c) -> int {
      for (int k = 0; k < kGraphSteps; ++k) PR_TRY(step(A, shift, x, c, true));
      return PR_OK;
    }));
    int graphs = 1;
    for (int64_t done = 0; done < max_it;) {
      for (int g = 0; g < graphs && done < max_it; ++g, done += kGraphSteps) PR_TRY(batch_graph.launch(s));
      PR_CUDA(cudaMemcpyAsync(out, st.ptr, sizeof(PcgScalars), cudaMemcpyDeviceToHost, s));
      PR_CUDA(cudaStreamSynchronize(s));
      if (out->done) return PR_OK;
      if (graphs < 8) graphs *= 2;
    }
    PR_CUDA(cudaMemcpyAsync(out, st.ptr, sizeof(PcgScalars), cudaMemcpyDeviceToHost, s));
    PR_CUDA(cudaStreamSynchronize(s));
    return PR_OK;
  }
};

// ------------------------------------------------------------------ conduction entry points

int conduction_create(const double* conductivity, int64_t nx, int64_t ny, int64_t nz, double H, cudaStream_t s,
                      pr_conduction** out) {
  std::unique_ptr<pr_conduction> A(new pr_conduction());
  cudaGetDevice(&A->device);
  A->nx = nx;
  A->ny = ny;
  A->nz = nz;
  A->n = nx * ny * nz;
  A->H = H;
  A->dx = H / (double)nx;
  A->last_stream = s;
  const int64_t n = A->n;
  PR_TRY(A->k.alloc(n, s));
  PR_TRY(A->gx.alloc(n, s));
  PR_TRY(A->gy.alloc(n, s));
  PR_TRY(A->gz.alloc(n, s));
  PR_TRY(A->diag.alloc(n, s));
  PR_TRY(A->hot.alloc(n, s));
  PR_TRY(A->cold.alloc(n, s));
  PR_CUDA(cudaMemcpyAsync(A->k.ptr, conductivity, n * 8, cudaMemcpyDefault, s));
  ::pr::launch_mark(), k_cond_assemble<<<grid_n(n), 256, 0, s>>>(A->k.ptr, nx, ny, nz, A->dx, A->gx.ptr, A->gy.ptr,
                                                                A->gz.ptr, A->hot.ptr, A->cold.ptr);
  ::pr::launch_mark(), k_cond_diagonal<<<grid_n(n), 256, 0, s>>>(A->gx.ptr, A->gy.ptr, A->gz.ptr, A->hot.ptr,
                                                                A->cold.ptr, nx, ny, nz, A->diag.ptr);
  PR_CUDA(cudaGetLastError());
  PR_CUDA(cudaStreamSynchronize(s));
  *out = A.release();
  return PR_OK;
}

int conduction_apply(const pr_conduction* A, const double* x, double* y, cudaStream_t s) {
  const int64_t n = A->n;
  DevBuf<double> dx_, dy_;
  PR_TRY(dx_.alloc(n, s));
  PR_TRY(dy_.alloc(n, s));
  PR_CUDA(cudaMemcpyAsync(dx_.ptr, x, n * 8, cudaMemcpyDefault, s));
  ::pr::launch_mark(), k_cond_apply<<<grid_n(n), 256, 0, s>>>(cond_view(A), dx_.ptr, nullptr, dy_.ptr);
  PR_CUDA(cudaGetLastError());
  PR_CUDA(cudaMemcpyAsync(y, dy_.ptr, n * 8, cudaMemcpyDefault, s));
  PR_CUDA(cudaStreamSynchronize(s));
  return PR_OK;
}

static int wall_fluxes_dev(const pr_conduction* A, const double* T, double Th, double Tc, Reducer& red, double* qh,
                           double* qc, cudaStream_t s) {
  const int64_t nyz = A->ny * A->nz;
  ::pr::launch_mark(), k_wall_flux<<<kRedBlocks, 256, 0, s>>>(A->k.ptr, T, A->nx, nyz, A->dx, Th, Tc, red.partial.ptr);
  PR_CUDA(cudaGetLastError());
  PR_TRY(sum_partials(red.partial.ptr, kRedBlocks, 2, red.out.ptr, s));
  double h[2];
  PR_CUDA(cudaMemcpyAsync(h, red.out.ptr, 16, cudaMemcpyDeviceToHost, s));
  PR_CUDA(cudaStreamSynchronize(s));
  *qh = h[0] / (double)nyz;
  *qc = h[1] / (double)nyz;
  return PR_OK;
}

int conduction_wall_fluxes(const pr_conduction* A, const double* T, double Th, double Tc, double* qh, double* qc,
                           cudaStream_t s) {
  DevBuf<double> dT;
  PR_TRY(dT.alloc(A->n, s));
  PR_CUDA(cudaMemcpyAsync(dT.ptr, T, A->n * 8, cudaMemcpyDefault, s));
  Reducer red;
  PR_TRY(red.init(s));
  return wall_fluxes_dev(A, dT.ptr, Th, Tc, red, qh, qc, s);
}

// Pure-conduction field (conduction.py:95-120): Jacobi-PCG from the linear profile until
// ||A T - b||_2 <= rtol ||b||_2; then the true relative residual must be <= 1e-9.
static int conduction_solve_dev(const pr_conduction* A, double Th, double Tc, double rtol, double* T, int64_t* iters,
                                double* relative, cudaStream_t s) {
  const int64_t n = A->n;
  DevBuf<double> b, r;
  PR_TRY(b.alloc(n, s));
  PR_TRY(r.alloc(n, s));
  const CondView V = cond_view(A);
  DevBuf<double> zero;
  PR_TRY(zero.alloc(n, s));
  PR_CUDA(cudaMemsetAsync(zero.ptr, 0, n * 8, s));
  // b = hot Th + cold Tc: the residual kernel with T = 0 and q = 0 gives -b
  ::pr::launch_mark(), k_residual<<<grid_n(n), 256, 0, s>>>(V, zero.ptr, Th, Tc, zero.ptr, b.ptr);
  ::pr::launch_mark(), k_negate<<<grid_n(n), 256, 0, s>>>(b.ptr, n, b.ptr);
  ::pr::launch_mark(), k_linear_profile<<<grid_n(n), 256, 0, s>>>(A->nx, A->ny * A->nz, Th, Tc, T);
  PR_CUDA(cudaGetLastError());
  Reducer red;
  PR_TRY(red.init(s));
  double bb = 0.0;
  PR_TRY(red.dot(b.ptr, b.ptr, n, &bb, s));
  const double bnorm = sqrt(bb);
  Pcg pcg;
  PR_TRY(pcg.init(n, s));
  PcgScalars st{};
  const int64_t max_it = std::max<int64_t>(50000, 20 * A->nx);  // conduction.py:114
  PR_TRY(pcg.solve(V, nullptr, b.ptr, rtol * bnorm, max_it, T, &st, s));
  ::pr::launch_mark(), k_residual<<<grid_n(n), 256, 0, s>>>(V, T, Th, Tc, zero.ptr, r.ptr);
  PR_CUDA(cudaGetLastError());
  double rr = 0.0;
  PR_TRY(red.dot(r.ptr, r.ptr, n, &rr, s));
  *relative = sqrt(rr) / bnorm;
  *iters = st.iterations;
  if (!st.done || !(*relative <= 1.0e-9)) {
    set_error("conduction solve did not converge: %lld iterations, residual=%.3e", (long long)st.iterations,
              *relative);
    return PR_ERR_SERIES;
  }
  return PR_OK;
}

int conduction_solve(const pr_conduction* A, double Th, double Tc, double rtol, double* T_out, int64_t* iters,
                     double* relative, cudaStream_t s) {
  DevBuf<double> T;
  PR_TRY(T.alloc(A->n, s));
  PR_TRY(conduction_solve_dev(A, Th, Tc, rtol, T.ptr, iters, relative, s));
  PR_CUDA(cudaMemcpyAsync(T_out, T.ptr, A->n * 8, cudaMemcpyDefault, s));
  PR_CUDA(cudaStreamSynchronize(s));
  return PR_OK;
}

// ------------------------------------------------------------------ the coupled solve

namespace {

constexpr int kNewtonMax = 8;          // coupled.py:29
constexpr double kNewtonResidual = 1.0e-13;
constexpr double kNewtonStep = 1.0e-10;
constexpr int kRestart = 30;
constexpr int kGmresMax = 90;
constexpr double kGmresRtol = 1.0e-8;
constexpr double kGmresAtol = 1.0e-13;
constexpr double kRtolNewton = 1.0e-8;
constexpr double kRtolFinal = 1.0e-13;

struct RadState {
  DevBuf<double> Tp, E, ab, q;  // patch temperature, emission, absorbed; cell net power
  double residual_power = 0.0;
  int64_t iterations = 0;
};

struct Coupled {
  const pr_case* c;
  const pr_operator* op;
  const pr_conduction* A;
  double Th, Tc, eps;
  cudaStream_t s;
  int64_t n, np;
  CondView V;
  Reducer red;
  Pcg pcg;
  DevBuf<double> epsv, shift, w, Ew, abw, tmp;
  DevBuf<double> basis, zbasis, hdev;

  int init(cudaStream_t s_) {
    s = s_;
    n = A->n;
    np = op->n;
    V = cond_view(A);
    PR_TRY(red.init(s));
    PR_TRY(pcg.init(n, s));
    PR_TRY(epsv.alloc(np, s));
    ::pr::launch_mark(), k_fill<<<grid_n(np), 256, 0, s>>>(epsv.ptr, np, eps);
    PR_CUDA(cudaGetLastError());
    PR_TRY(shift.alloc(n, s));
    PR_TRY(w.alloc(n, s));
    PR_TRY(tmp.alloc(n, s));
    PR_TRY(Ew.alloc(np, s));
    PR_TRY(abw.alloc(np, s));
    PR_TRY(basis.alloc((size_t)(kRestart + 1) * n, s));
    PR_TRY(zbasis.alloc((size_t)kRestart * n, s));
    PR_TRY(hdev.alloc(32, s));
    return PR_OK;
  }

  int alloc_state(RadState& st) {
    PR_TRY(st.Tp.alloc(np, s));
    PR_TRY(st.E.alloc(np, s));
    PR_TRY(st.ab.alloc(np, s));
    PR_TRY(st.q.alloc(n, s));
    return PR_OK;
  }

  // evaluate_radiation (coupled.py:86-105) at cell field T, radiosity to rtol
  int radiation(const double* T, double rtol, RadState& st) {
    ::pr::launch_mark(), k_patch_temperature<<<grid_n(np), 256, 0, s>>>(c->cls.ptr, c->cell.ptr, T, Th, Tc, np,
                                                                        st.Tp.ptr);
    ::pr::launch_mark(), k_emission_t4<<<grid_n(np), 256, 0, s>>>(st.Tp.ptr, eps, op->area.ptr, np, st.E.ptr);
    PR_CUDA(cudaGetLastError());
    PR_TRY(series_fp64(op, st.E.ptr, epsv.ptr, rtol, 10000, st.ab.ptr, &st.residual_power, &st.iterations, s));
    ::pr::launch_mark(), k_cell_power<<<grid_n(n), 256, 0, s>>>(c->cfp(), st.ab.ptr, st.E.ptr, n, st.q.ptr);
    PR_CUDA(cudaGetLastError());
    return PR_OK;
  }

  // out = A v - radiation_jvp(T_patch, v) (coupled.py:108-123, 371-374)
  int jacobian(const double* Tp, const double* v, double* out) {
    ::pr::launch_mark(), k_emission_jvp<<<grid_n(np), 256, 0, s>>>(c->cls.ptr, c->cell.ptr, Tp, v, eps, op->area.ptr,
                                                                   np, Ew.ptr);
    PR_CUDA(cudaGetLastError());
    double res = 0.0;
    int64_t it = 0;
    PR_TRY(series_fp64(op, Ew.ptr, epsv.ptr, kRtolNewton, 10000, abw.ptr, &res, &it, s));
    ::pr::launch_mark(), k_cell_power<<<grid_n(n), 256, 0, s>>>(c->cfp(), abw.ptr, Ew.ptr, n, tmp.ptr);
    ::pr::launch_mark(), k_cond_apply<<<grid_n(n), 256, 0, s>>>(V, v, nullptr, out);
    ::pr::launch_mark(), k_axpby<<<grid_n(n), 256, 0, s>>>(-1.0, tmp.ptr, 1.0, out, n);
    PR_CUDA(cudaGetLastError());
    return PR_OK;
  }

  double norm2(const double* x) {
    double st[5];
    if (red.stats(x, nullptr, n, st, s) != PR_OK) return NAN;
    return sqrt(st[0]);
  }

  // Flexible GMRES (coupled.py:230-290) on J x = b, right-preconditioned by `steps` fixed
  // Jacobi-PCG steps on A + diag(shift); x = 0 at the start.
  int fgmres(const double* Tp, const double* b, int steps, double* x, bool* converged, int* iterations,
             double* true_rel) {
    DevBuf<double> rres, cand;
    PR_TRY(rres.alloc(n, s));
    PR_TRY(cand.alloc(n, s));
    PR_CUDA(cudaMemsetAsync(x, 0, n * 8, s));
    const double b_norm = std::max(norm2(b), 2.2250738585072014e-308);
    const double threshold = std::max(kGmresAtol, kGmresRtol * b_norm);
    const double eps64 = 2.220446049250313e-16;
    int total = 0;
    double* Vb = basis.ptr;
    double* Zb = zbasis.ptr;
    while (total < kGmresMax) {
      // residual = b - J x
      PR_TRY(jacobian(Tp, x, rres.ptr));
      ::pr::launch_mark(), k_axpby<<<grid_n(n), 256, 0, s>>>(1.0, b, -1.0, rres.ptr, n);
      PR_CUDA(cudaGetLastError());
      const double beta = norm2(rres.ptr);
      if (beta <= threshold) {
        *converged = true;
        *iterations = total;
        *true_rel = beta / b_norm;
        return PR_OK;
      }
      const int width = std::min(kRestart, kGmresMax - total);
      std::vector<double> H((size_t)(width + 1) * width, 0.0), g(width + 1, 0.0), cs(width, 0.0), sn(width, 0.0);
      std::vector<double> R((size_t)(width + 1) * width, 0.0);  // rotated H
      ::pr::launch_mark(), k_axpby<<<grid_n(n), 256, 0, s>>>(1.0 / beta, rres.ptr, 0.0, Vb, n);
      PR_CUDA(cudaGetLastError());
      g[0] = beta;
      bool restart_from = false;
      int used = 0;
      for (int col = 0; col < width; ++col) {
        double* vcol = Vb + (size_t)col * n;
        double* zcol = Zb + (size_t)col * n;
        PR_TRY(pcg.fixed(V, shift.ptr, vcol, steps, zcol, s));
        PR_TRY(jacobian(Tp, zcol, w.ptr));
        double h[32];
        for (int pass = 0; pass < 2; ++pass) {
          PR_TRY(red.multidot(Vb, col + 1, w.ptr, n, hdev.ptr, h, s));
          ::pr::launch_mark(), k_multi_axpy<<<grid_n(n), 256, 0, s>>>(Vb, col + 1, hdev.ptr, n, w.ptr);
          PR_CUDA(cudaGetLastError());
          for (int r = 0; r <= col; ++r) H[(size_t)r * width + col] += h[r];
        }
        const double next_norm = norm2(w.ptr);
        H[(size_t)(col + 1) * width + col] = next_norm;
        if (next_norm > eps64 * beta) {
          ::pr::launch_mark(), k_axpby<<<grid_n(n), 256, 0, s>>>(1.0 / next_norm, w.ptr, 0.0, Vb + (size_t)(col + 1) * n,
                                                                 n);
          PR_CUDA(cudaGetLastError());
        } else {
          PR_CUDA(cudaMemsetAsync(Vb + (size_t)(col + 1) * n, 0, n * 8, s));
        }
        // least squares min ||g - H y|| by Givens rotations on the new column
        for (int r = 0; r <= col + 1; ++r) R[(size_t)r * width + col] = H[(size_t)r * width + col];
        for (int r = 0; r < col; ++r) {
          const double a = R[(size_t)r * width + col], bb = R[(size_t)(r + 1) * width + col];
          R[(size_t)r * width + col] = cs[r] * a + sn[r] * bb;
          R[(size_t)(r + 1) * width + col] = -sn[r] * a + cs[r] * bb;
        }
        {
          const double a = R[(size_t)col * width + col], bb = R[(size_t)(col + 1) * width + col];
          const double rr = hypot(a, bb);
          cs[col] = rr > 0.0 ? a / rr : 1.0;
          sn[col] = rr > 0.0 ? bb / rr : 0.0;
          R[(size_t)col * width + col] = rr;
          R[(size_t)(col + 1) * width + col] = 0.0;
          const double g0 = g[col];
          g[col] = cs[col] * g0;
          g[col + 1] = -sn[col] * g0;
        }
        const double estimate = fabs(g[col + 1]);
        ++total;
        used = col + 1;
        if (estimate <= threshold || next_norm <= eps64 * beta) {
          // candidate = x + Z y
          std::vector<double> y(col + 1, 0.0);
          for (int r = col; r >= 0; --r) {
            double v = g[r];
            for (int k = r + 1; k <= col; ++k) v -= R[(size_t)r * width + k] * y[k];
            const double d = R[(size_t)r * width + r];
            y[r] = d != 0.0 ? v / d : 0.0;
          }
          PR_CUDA(cudaMemcpyAsync(cand.ptr, x, n * 8, cudaMemcpyDeviceToDevice, s));
          for (int r = 0; r <= col; ++r) {
            ::pr::launch_mark(), k_axpby<<<grid_n(n), 256, 0, s>>>(y[r], Zb + (size_t)r * n, 1.0, cand.ptr, n);
          }
          PR_CUDA(cudaGetLastError());
          PR_TRY(jacobian(Tp, cand.ptr, rres.ptr));
          ::pr::launch_mark(), k_axpby<<<grid_n(n), 256, 0, s>>>(1.0, b, -1.0, rres.ptr, n);
          PR_CUDA(cudaGetLastError());
          const double true_norm = norm2(rres.ptr);
          PR_CUDA(cudaMemcpyAsync(x, cand.ptr, n * 8, cudaMemcpyDeviceToDevice, s));
          if (true_norm <= threshold) {
            *converged = true;
            *iterations = total;
            *true_rel = true_norm / b_norm;
            return PR_OK;
          }
          restart_from = true;
          break;
        }
      }
      if (restart_from) continue;
      // x += Z y over the whole cycle
      std::vector<double> y(used, 0.0);
      for (int r = used - 1; r >= 0; --r) {
        double v = g[r];
        for (int k = r + 1; k < used; ++k) v -= R[(size_t)r * width + k] * y[k];
        const double d = R[(size_t)r * width + r];
        y[r] = d != 0.0 ? v / d : 0.0;
      }
      for (int r = 0; r < used; ++r)
        ::pr::launch_mark(), k_axpby<<<grid_n(n), 256, 0, s>>>(y[r], Zb + (size_t)r * n, 1.0, x, n);
      PR_CUDA(cudaGetLastError());
    }
    PR_TRY(jacobian(Tp, x, rres.ptr));
    ::pr::launch_mark(), k_axpby<<<grid_n(n), 256, 0, s>>>(1.0, b, -1.0, rres.ptr, n);
    PR_CUDA(cudaGetLastError());
    const double true_norm = norm2(rres.ptr);
    *converged = true_norm <= threshold;
    *iterations = total;
    *true_rel = true_norm / b_norm;
    return PR_OK;
  }
};

}  // namespace

// One Newton-Krylov solve (coupled.py:340-421) with `steps` preconditioner steps.
static int newton_krylov(Coupled& K, const double* T_init, int steps, double* T, RadState& final_state,
                         pr_coupled_result* res) {
  const int64_t n = K.n;
  cudaStream_t s = K.s;
  memset(res, 0, sizeof(*res));
  res->preconditioner_steps = steps;
  // preconditioner shift: the emission derivative at the initial field (coupled.py:353)
  ::pr::launch_mark(), k_emission_diagonal<<<grid_n(n), 256, 0, s>>>(K.c->cfp(), K.op->area.ptr, T_init, K.eps, n,
                                                                     K.shift.ptr);
  PR_CUDA(cudaGetLastError());
  PR_CUDA(cudaMemcpyAsync(T, T_init, n * 8, cudaMemcpyDeviceToDevice, s));
  RadState state, trial_state;
  PR_TRY(K.alloc_state(state));
  PR_TRY(K.alloc_state(trial_state));
  DevBuf<double> resid, trial_resid, step, cand, rhs;
  PR_TRY(resid.alloc(n, s));
  PR_TRY(trial_resid.alloc(n, s));
  PR_TRY(step.alloc(n, s));
  PR_TRY(cand.alloc(n, s));
  PR_TRY(rhs.alloc(n, s));
  PR_TRY(K.radiation(T, kRtolNewton, state));
  ::pr::launch_mark(), k_residual<<<grid_n(n), 256, 0, s>>>(K.V, T, K.Th, K.Tc, state.q.ptr, resid.ptr);
  PR_CUDA(cudaGetLastError());
  double st5[5];
  PR_TRY(K.red.stats(resid.ptr, nullptr, n, st5, s));
  double last_step = std::max(st5[1], 2.2250738585072014e-308) <= kNewtonResidual ? 0.0 : INFINITY;
  int failure = PR_COUPLED_MAX_NEWTON;
  bool converged = false;
  for (int it = 0; it < kNewtonMax; ++it) {
    PR_TRY(K.red.stats(resid.ptr, nullptr, n, st5, s));
    const double residual_norm = st5[1];
    const double residual_l2 = sqrt(st5[0]);
    if (residual_norm <= kNewtonResidual && last_step <= kNewtonStep) {
      converged = true;
      failure = PR_COUPLED_OK;
      break;
    }
    // FGMRES on J step = -R at the state's patch temperatures
    ::pr::launch_mark(), k_axpby<<<grid_n(n), 256, 0, s>>>(-1.0, resid.ptr, 0.0, rhs.ptr, n);
    PR_CUDA(cudaGetLastError());
    bool gconv = false;
    int giters = 0;
    double grel = 0.0;
    PR_TRY(K.fgmres(state.Tp.ptr, rhs.ptr, steps, step.ptr, &gconv, &giters, &grel));
    // true residual of the linear solve: || J step + R ||
    PR_TRY(K.jacobian(state.Tp.ptr, step.ptr, cand.ptr));
    ::pr::launch_mark(), k_axpby<<<grid_n(n), 256, 0, s>>>(1.0, resid.ptr, 1.0, cand.ptr, n);
    PR_CUDA(cudaGetLastError());
    const double true_l2 = K.norm2(cand.ptr);
    if (res->n_linear < PR_COUPLED_MAX_LINEAR) {
      pr_coupled_linear& L = res->linear[res->n_linear++];
      L.converged = gconv ? 1 : 0;
      L.gmres_iterations = giters;
      L.rhs_l2_W = residual_l2;
      L.true_residual_l2_W = true_l2;
      L.true_residual_relative = grel;
    }
    if (!gconv) {
      failure = PR_COUPLED_LINEAR;
      break;
    }
    PR_TRY(K.red.stats(step.ptr, nullptr, n, st5, s));
    if (residual_norm <= kNewtonResidual && st5[1] <= kNewtonStep) {
      converged = true;
      failure = PR_COUPLED_OK;
      break;
    }
    // backtracking line search within [Tc, Th] (coupled.py:392-408)
    double alpha = 1.0, trial_norm = 0.0;
    bool accepted = false;
    while (alpha >= 0x1p-20) {
      ::pr::launch_mark(), k_add_scaled<<<grid_n(n), 256, 0, s>>>(T, alpha, step.ptr, n, cand.ptr);
      PR_CUDA(cudaGetLastError());
      PR_TRY(K.red.stats(cand.ptr, nullptr, n, st5, s));
      if (st5[4] == 0.0 && st5[2] >= K.Tc && st5[3] <= K.Th) {
        PR_TRY(K.radiation(cand.ptr, kRtolNewton, trial_state));
        ::pr::launch_mark(), k_residual<<<grid_n(n), 256, 0, s>>>(K.V, cand.ptr, K.Th, K.Tc, trial_state.q.ptr,
                                                                  trial_resid.ptr);
        PR_CUDA(cudaGetLastError());
        PR_TRY(K.red.stats(trial_resid.ptr, nullptr, n, st5, s));
        trial_norm = st5[1];
        if (trial_norm <= (1.0 - 1.0e-4 * alpha) * residual_norm) {
          accepted = true;
          break;
        }
      }
      alpha *= 0.5;
    }
    if (!accepted) {
      failure = PR_COUPLED_LINE_SEARCH;
      break;
    }
    PR_TRY(K.red.stats(cand.ptr, T, n, st5, s));
    last_step = st5[1];
    PR_CUDA(cudaMemcpyAsync(T, cand.ptr, n * 8, cudaMemcpyDeviceToDevice, s));
    std::swap(state, trial_state);
    std::swap(resid, trial_resid);
    res->newton_iterations += 1;
    if (trial_norm <= kNewtonResidual && last_step <= kNewtonStep) {
      converged = true;
      failure = PR_COUPLED_OK;
      break;
    }
  }
  // final state at the tight radiosity tolerance (coupled.py:364-368)
  PR_TRY(K.radiation(T, kRtolFinal, final_state));
  ::pr::launch_mark(), k_residual<<<grid_n(n), 256, 0, s>>>(K.V, T, K.Th, K.Tc, final_state.q.ptr, resid.ptr);
  PR_CUDA(cudaGetLastError());
  PR_TRY(K.red.stats(resid.ptr, nullptr, n, st5, s));
  res->final_residual_inf_W = st5[1];
  res->converged = converged ? 1 : 0;
  res->failure = failure;
  return PR_OK;
}

static bool linear_residuals_pass(const pr_coupled_result* r) {  // coupled.py:333-337
  if (r->n_linear == 0) return false;
  for (int k = 0; k < r->n_linear; ++k) {
    const pr_coupled_linear& L = r->linear[k];
    if (!L.converged || !(L.true_residual_l2_W <= std::max(1.0e-13, 1.0e-8 * L.rhs_l2_W))) return false;
  }
  return true;
}

int coupled_solve(const pr_case* c, const pr_operator* op, const pr_conduction* A, double Th, double Tc, double eps,
                  const double* T_initial, int preconditioner_steps, double* T_out, double* patch_temperature,
                  double* patch_emitted, double* patch_absorbed, double* cell_net_power, pr_coupled_result* res,
                  cudaStream_t s) {
  PR_ARG(A->nx == c->nx && A->ny == c->ny && A->nz == c->nz, "conduction grid and geometry differ");
  PR_ARG(op->n == c->n_patches, "operator and geometry differ in the number of patches");
  Coupled K{c, op, A, Th, Tc, eps};
  PR_TRY(K.init(s));
  const int64_t n = A->n, np = op->n;
  DevBuf<double> T0, T;
  PR_TRY(T0.alloc(n, s));
  PR_TRY(T.alloc(n, s));
  PR_CUDA(cudaMemcpyAsync(T0.ptr, T_initial, n * 8, cudaMemcpyDefault, s));
  RadState fin;
  PR_TRY(K.alloc_state(fin));
  const int attempts[2] = {10, 20};  // coupled.py:37, 423-440
  const int n_att = preconditioner_steps > 0 ? 1 : 2;
  for (int a = 0; a < n_att; ++a) {
    const int steps = preconditioner_steps > 0 ? preconditioner_steps : attempts[a];
    PR_TRY(newton_krylov(K, T0.ptr, steps, T.ptr, fin, res));
    if (res->converged && linear_residuals_pass(res)) break;
  }
  res->linear_residuals_pass = linear_residuals_pass(res) ? 1 : 0;
  // wall-flux metrics (coupled.py:443-472)
  double qh = 0.0, qc = 0.0;
  PR_TRY(wall_fluxes_dev(A, T.ptr, Th, Tc, K.red, &qh, &qc, s));
  ::pr::launch_mark(), k_net_sums<<<kRedBlocks, 256, 0, s>>>(c->cls.ptr, fin.ab.ptr, fin.E.ptr, np, nullptr,
                                                             K.red.partial.ptr);
  PR_CUDA(cudaGetLastError());
  PR_TRY(sum_partials(K.red.partial.ptr, kRedBlocks, 4, K.red.out.ptr, s));
  double sums[4];
  PR_CUDA(cudaMemcpyAsync(sums, K.red.out.ptr, 32, cudaMemcpyDeviceToHost, s));
  double st5[5];
  PR_TRY(K.red.stats(T.ptr, nullptr, n, st5, s));
  const double cell = A->H / (double)A->nx;
  const double area = (double)(A->ny * A->nz) * cell * cell;
  res->q_cond_hot_W_m2 = qh;
  res->q_cond_cold_W_m2 = qc;
  res->q_rad_hot_W_m2 = -sums[0] / area;
  res->q_rad_cold_W_m2 = sums[1] / area;
  res->q_total_hot_W_m2 = qh + res->q_rad_hot_W_m2;
  res->q_total_cold_W_m2 = qc + res->q_rad_cold_W_m2;
  const double scale = std::max(std::max(fabs(res->q_total_hot_W_m2), fabs(res->q_total_cold_W_m2)),
                                2.2250738585072014e-308);
  res->radiative_fraction_hot = res->q_rad_hot_W_m2 / res->q_total_hot_W_m2;
  res->k_eff_apparent_W_mK = res->q_total_hot_W_m2 * A->H / (Th - Tc);
  res->wall_flux_mismatch_rel = fabs(res->q_total_hot_W_m2 - res->q_total_cold_W_m2) / scale;
  res->global_energy_residual_W = sums[3] + fin.residual_power;
  res->energy_residual_rel = fabs(res->global_energy_residual_W) / std::max(scale * area, 2.2250738585072014e-308);
  res->residual_power_W = fin.residual_power;
  res->series_iterations = fin.iterations;
  res->T_min_K = st5[2];
  res->T_max_K = st5[3];
  {
    // cells outside [Tc, Th] (coupled.py:470)
    ::pr::launch_mark(), k_count_outside<<<kRedBlocks, 256, 0, s>>>(T.ptr, n, Tc, Th, K.red.partial.ptr);
    PR_CUDA(cudaGetLastError());
    PR_TRY(sum_partials(K.red.partial.ptr, kRedBlocks, 1, K.red.out.ptr, s));
    double cnt = 0.0;
    PR_CUDA(cudaMemcpyAsync(&cnt, K.red.out.ptr, 8, cudaMemcpyDeviceToHost, s));
    PR_CUDA(cudaStreamSynchronize(s));
    res->temperature_bound_violations = (int64_t)cnt;
  }
  if (T_out) PR_CUDA(cudaMemcpyAsync(T_out, T.ptr, n * 8, cudaMemcpyDefault, s));
  if (patch_temperature) PR_CUDA(cudaMemcpyAsync(patch_temperature, fin.Tp.ptr, np * 8, cudaMemcpyDefault, s));
  if (patch_emitted) PR_CUDA(cudaMemcpyAsync(patch_emitted, fin.E.ptr, np * 8, cudaMemcpyDefault, s));
  if (patch_absorbed) PR_CUDA(cudaMemcpyAsync(patch_absorbed, fin.ab.ptr, np * 8, cudaMemcpyDefault, s));
  if (cell_net_power) PR_CUDA(cudaMemcpyAsync(cell_net_power, fin.q.ptr, n * 8, cudaMemcpyDefault, s));
  PR_CUDA(cudaStreamSynchronize(s));
  return PR_OK;
}

}  // namespace pr

// ------------------------------------------------------------------ C-ABI

using namespace pr;

#define PR_CHECK_NULL_C(p, name)                \
  do {                                          \
    if (!(p)) {                                 \
      set_error("%s must not be NULL", name);   \
      return PR_ERR_ARG;                        \
    }                                           \
  } while (0)

extern "C" {

PR_API int pr_conduction_create(const double* conductivity, int64_t nx, int64_t ny, int64_t nz, double H_m,
                                void* stream, pr_conduction** out) {
  PR_CHECK_NULL_C(out, "out");
  *out = nullptr;
  PR_CHECK_NULL_C(conductivity, "conductivity");
  PR_ARG(nx > 0 && ny > 0 && nz > 0 && nx * ny * nz < ((int64_t)1 << 33), "grid dimensions out of range");
  PR_ARG(H_m > 0.0, "H_m must be positive");
  return conduction_create(conductivity, nx, ny, nz, H_m, (cudaStream_t)stream, out);
}

PR_API void pr_conduction_destroy(pr_conduction* A) {
  if (!A) return;
  DeviceGuard g(A->device);
  delete A;
}

PR_API int pr_conduction_arrays(const pr_conduction* A, double* gx, double* gy, double* gz, double* diag,
                                double* hot_rhs, double* cold_rhs, void* stream) {
  PR_CHECK_NULL_C(A, "conduction");
  DeviceGuard g(A->device);
  cudaStream_t s = (cudaStream_t)stream;
  const size_t b = (size_t)A->n * 8;
  if (gx) PR_CUDA(cudaMemcpyAsync(gx, A->gx.ptr, b, cudaMemcpyDefault, s));
  if (gy) PR_CUDA(cudaMemcpyAsync(gy, A->gy.ptr, b, cudaMemcpyDefault, s));
  if (gz) PR_CUDA(cudaMemcpyAsync(gz, A->gz.ptr, b, cudaMemcpyDefault, s));
  if (diag) PR_CUDA(cudaMemcpyAsync(diag, A->diag.ptr, b, cudaMemcpyDefault, s));
  if (hot_rhs) PR_CUDA(cudaMemcpyAsync(hot_rhs, A->hot.ptr, b, cudaMemcpyDefault, s));
  if (cold_rhs) PR_CUDA(cudaMemcpyAsync(cold_rhs, A->cold.ptr, b, cudaMemcpyDefault, s));
  PR_CUDA(cudaStreamSynchronize(s));
  return PR_OK;
}

PR_API int pr_conduction_apply(const pr_conduction* A, const double* x, double* y, void* stream) {
  PR_CHECK_NULL_C(A, "conduction");
  PR_CHECK_NULL_C(x, "x");
  PR_CHECK_NULL_C(y, "y");
  DeviceGuard g(A->device);
  return conduction_apply(A, x, y, (cudaStream_t)stream);
}

PR_API int pr_conduction_solve(const pr_conduction* A, double T_hot_K, double T_cold_K, double rtol, double* T_out,
                               int64_t* iterations, double* relative_residual, void* stream) {
  PR_CHECK_NULL_C(A, "conduction");
  PR_CHECK_NULL_C(T_out, "T_out");
  PR_ARG(rtol > 0.0, "rtol must be positive");
  DeviceGuard g(A->device);
  int64_t it = 0;
  double rel = 0.0;
  const int st = conduction_solve(A, T_hot_K, T_cold_K, rtol, T_out, &it, &rel, (cudaStream_t)stream);
  if (iterations) *iterations = it;
  if (relative_residual) *relative_residual = rel;
  return st;
}

PR_API int pr_conduction_wall_fluxes(const pr_conduction* A, const double* T, double T_hot_K, double T_cold_K,
                                     double* q_hot, double* q_cold, void* stream) {
  PR_CHECK_NULL_C(A, "conduction");
  PR_CHECK_NULL_C(T, "T");
  DeviceGuard g(A->device);
  double qh = 0.0, qc = 0.0;
  PR_TRY(conduction_wall_fluxes(A, T, T_hot_K, T_cold_K, &qh, &qc, (cudaStream_t)stream));
  if (q_hot) *q_hot = qh;
  if (q_cold) *q_cold = qc;
  return PR_OK;
}

PR_API int pr_coupled_solve(const pr_case* c, const pr_operator* op, const pr_conduction* A, double T_hot_K,
                            double T_cold_K, double epsilon, const double* T_initial, int preconditioner_steps,
                            double* T_out, double* patch_temperature, double* patch_emitted, double* patch_absorbed,
                            double* cell_net_power, pr_coupled_result* result, void* stream) {
  PR_CHECK_NULL_C(c, "case");
  PR_CHECK_NULL_C(op, "operator");
  PR_CHECK_NULL_C(A, "conduction");
  PR_CHECK_NULL_C(T_initial, "T_initial");
  PR_CHECK_NULL_C(result, "result");
  PR_ARG(c->device == op->device && c->device == A->device, "objects live on different devices");
  PR_ARG(T_hot_K > T_cold_K, "T_hot_K must exceed T_cold_K");
  PR_ARG(preconditioner_steps >= 0, "preconditioner_steps must not be negative");
  DeviceGuard g(c->device);
  return coupled_solve(c, op, A, T_hot_K, T_cold_K, epsilon, T_initial, preconditioner_steps, T_out,
                       patch_temperature, patch_emitted, patch_absorbed, cell_net_power, result,
                       (cudaStream_t)stream);
}

}  // extern "C"
