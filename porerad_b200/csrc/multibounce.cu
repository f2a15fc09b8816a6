// Multi-bounce ray statistics of a slab (porerad/properties.py, porerad/penetration.py) on the
// device: equivalent radiative properties (extinction from the first path segment, albedo and
// asymmetry from the surface interactions) and the penetration response (reflected,
// transmitted and absorbed fractions).
//
// Both follow the reference's Taichi kernels ray for ray: the same 32-bit hash generator
// (properties.py:83-96), the same cell traversal with its start-cell rule, tie tolerance,
// surface normals and step cap (properties.py:98-197), the same Lambertian sampling about the
// surface normal (properties.py:200-226), and both restart rules of a reflected ray.  One
// thread follows one ray; tallies accumulate per thread in ray order and meet in fixed-order
// warp reductions, one partial per warp, then one fixed-order sum over the warps (the reference
// adds them with atomics in whatever order its threads run).
// Built with -fmad=false; the azimuth's sin and cos are correctly rounded (pr_sincos).
#include "pr_math.cuh"
#include "pr_spmv.cuh"

namespace pr {

namespace {

__device__ __forceinline__ uint32_t mb_hash(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7FEB352Du;
  x ^= x >> 15;
  x *= 0x846CA68Bu;
  x ^= x >> 16;
  return x;
}

// next uniform in [0, 1) with 24 bits (properties.py:92-96)
__device__ __forceinline__ double mb_rand(uint32_t& state) {
  state = mb_hash(state + 0x9E3779B9u);
  return (double)(state & 0x00FFFFFFu) / (double)0x01000000u;
}

struct MbGrid {
  const uint32_t* __restrict__ occ;  // flat occupancy bits, cell (i ny + j) nz + k
  int sx, sy, sz;
};

__device__ __forceinline__ int pymod(int a, int m) {
  const int r = a % m;
  return r < 0 ? r + m : r;
}

struct Hit {
  int fate;  // 0 solid, 1 exit at x = 0, 2 exit at x = N, 3 step cap
  double t, nx, ny, nz;
};

// Cell traversal from o along d (normalised here) until a solid cell, an x wall or the step
// cap; the normal is that of the last face crossed (properties.py:98-197).
__device__ Hit mb_trace(const MbGrid& g, double ox, double oy, double oz, double dx0, double dy0, double dz0) {
  const double norm = sqrt(pr_add(pr_add(pr_mul(dx0, dx0), pr_mul(dy0, dy0)), pr_mul(dz0, dz0)));
  const double dx = pr_div(dx0, norm), dy = pr_div(dy0, norm), dz = pr_div(dz0, norm);
  int i = (int)floor(ox), j = (int)floor(oy), k = (int)floor(oz);
  if (dx < 0.0 && fabs(pr_sub(ox, floor(pr_add(ox, 0.5)))) <= 1.0e-12) i -= 1;
  if (dy < 0.0 && fabs(pr_sub(oy, floor(pr_add(oy, 0.5)))) <= 1.0e-12) j -= 1;
  if (dz < 0.0 && fabs(pr_sub(oz, floor(pr_add(oz, 0.5)))) <= 1.0e-12) k -= 1;
  int stx = 0, sty = 0, stz = 0;
  double tmx = 1.0e300, tmy = 1.0e300, tmz = 1.0e300, tdx = 1.0e300, tdy = 1.0e300, tdz = 1.0e300;
  const double sdx = fabs(dx) > 0.0 ? dx : 1.0, sdy = fabs(dy) > 0.0 ? dy : 1.0, sdz = fabs(dz) > 0.0 ? dz : 1.0;
  if (dx > 0.0) {
    stx = 1;
    tmx = pr_div(pr_sub((double)(i + 1), ox), sdx);
    tdx = pr_div(1.0, sdx);
  } else if (dx < 0.0) {
    stx = -1;
    tmx = pr_div(pr_sub((double)i, ox), sdx);
    tdx = pr_div(-1.0, sdx);
  }
  if (dy > 0.0) {
    sty = 1;
    tmy = pr_div(pr_sub((double)(j + 1), oy), sdy);
    tdy = pr_div(1.0, sdy);
  } else if (dy < 0.0) {
    sty = -1;
    tmy = pr_div(pr_sub((double)j, oy), sdy);
    tdy = pr_div(-1.0, sdy);
  }
  if (dz > 0.0) {
    stz = 1;
    tmz = pr_div(pr_sub((double)(k + 1), oz), sdz);
    tdz = pr_div(1.0, sdz);
  } else if (dz < 0.0) {
    stz = -1;
    tmz = pr_div(pr_sub((double)k, oz), sdz);
    tdz = pr_div(-1.0, sdz);
  }
  Hit h{-1, 0.0, 0.0, 0.0, 0.0};
  const long long max_steps = 10LL * g.sx * g.sy * g.sz + 10;
  for (long long steps = 0; h.fate == -1 && steps < max_steps;) {
    ++steps;
    if (i < 0) {
      h.fate = 1;
    } else if (i >= g.sx) {
      h.fate = 2;
    } else {
      const int cell = (i * g.sy + pymod(j, g.sy)) * g.sz + pymod(k, g.sz);
      if ((__ldg(g.occ + (cell >> 5)) >> (cell & 31)) & 1u) {
        h.fate = 0;
      } else {
        const double tn = fmin(tmx, fmin(tmy, tmz));
        const bool cx = fabs(pr_sub(tmx, tn)) <= 1.0e-12;
        const bool cy = fabs(pr_sub(tmy, tn)) <= 1.0e-12;
        const bool cz = fabs(pr_sub(tmz, tn)) <= 1.0e-12;
        if (cx) {
          i += stx;
          tmx = pr_add(tmx, tdx);
          h.nx = -(double)stx;
          h.ny = 0.0;
          h.nz = 0.0;
        }
        if (cy) {
          j += sty;
          tmy = pr_add(tmy, tdy);
          if (!cx) {
            h.nx = 0.0;
            h.ny = -(double)sty;
            h.nz = 0.0;
          }
        }
        if (cz) {
          k += stz;
          tmz = pr_add(tmz, tdz);
          if (!cx && !cy) {
            h.nx = 0.0;
            h.ny = 0.0;
            h.nz = -(double)stz;
          }
        }
        h.t = tn;
      }
    }
  }
  if (h.fate == -1) h.fate = 3;
  return h;
}

#define MB_TWO_PI 0x1.921fb54442d18p+2  // the binary64 product 2.0 * math.pi

// Lambertian direction about the unit normal n (properties.py:200-226): an orthonormal
// frame from a helper axis, radius sqrt(xi1), azimuth 2 pi xi2, elevation sqrt(1 - xi1).
__device__ void mb_lambertian(uint32_t& state, double nx, double ny, double nz, double& dx, double& dy, double& dz) {
  const double xi1 = mb_rand(state), xi2 = mb_rand(state);
  double hx = 1.0, hy = 0.0, hz = 0.0;
  if (fabs(nx) > 0.9) {
    hx = 0.0;
    hy = 1.0;
    hz = 0.0;
  }
  double ux = pr_sub(pr_mul(hy, nz), pr_mul(hz, ny));
  double uy = pr_sub(pr_mul(hz, nx), pr_mul(hx, nz));
  double uz = pr_sub(pr_mul(hx, ny), pr_mul(hy, nx));
  const double un = sqrt(pr_add(pr_add(pr_mul(ux, ux), pr_mul(uy, uy)), pr_mul(uz, uz)));
  ux = pr_div(ux, un);
  uy = pr_div(uy, un);
  uz = pr_div(uz, un);
  const double vx = pr_sub(pr_mul(ny, uz), pr_mul(nz, uy));
  const double vy = pr_sub(pr_mul(nz, ux), pr_mul(nx, uz));
  const double vz = pr_sub(pr_mul(nx, uy), pr_mul(ny, ux));
  const double radius = sqrt(xi1);
  const double phi = pr_mul(MB_TWO_PI, xi2);
  double s, c;
  pr_sincos(phi, &s, &c);
  const double cx = pr_mul(radius, c), cy = pr_mul(radius, s);
  const double cz = sqrt(fmax(0.0, pr_sub(1.0, xi1)));
  dx = pr_add(pr_add(pr_mul(cx, ux), pr_mul(cy, vx)), pr_mul(cz, nx));
  dy = pr_add(pr_add(pr_mul(cx, uy), pr_mul(cy, vy)), pr_mul(cz, ny));
  dz = pr_add(pr_add(pr_mul(cx, uz), pr_mul(cy, vz)), pr_mul(cz, nz));
}

// Tallies of one thread: properties (0 events, 1 sum of event lengths, 2 censored, 3 sum of
// censored lengths, 4 interactions, 5 scattered, 6 sum of mu, 7 sum of mu^2) or penetration
// (0 reflected, 1 transmitted, 2 absorbed, 3 stopped at a cap).  Counts are exact in binary64.
constexpr int kMbThreads = 64;  // small blocks: a block's registers return as soon as its two warps end

template <bool kPenetration>
__global__ void __launch_bounds__(kMbThreads) k_multibounce(MbGrid g, int64_t n, uint32_t seed, double eps, int max_bounces,
                                                     int hit_point, double* __restrict__ partial) {
  double acc[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  for (int64_t ray = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; ray < n; ray += (int64_t)gridDim.x * blockDim.x) {
    uint32_t state = mb_hash(seed + (uint32_t)(ray + 1) * 747796405u);
    const double ry = mb_rand(state), rz = mb_rand(state);
    double ox = 0.0, oy = pr_mul(ry, (double)g.sy), oz = pr_mul(rz, (double)g.sz);
    double dx = 1.0, dy = 0.0, dz = 0.0;
    if (kPenetration) mb_lambertian(state, 1.0, 0.0, 0.0, dx, dy, dz);
    Hit h = mb_trace(g, ox, oy, oz, dx, dy, dz);
    if (h.fate != 0) {
      if (kPenetration) {
        acc[h.fate == 1 ? 0 : (h.fate == 2 ? 1 : 3)] += 1.0;
      } else {
        acc[2] += 1.0;
        acc[3] += h.t;
      }
      continue;
    }
    double nx = h.nx, ny = h.ny, nz = h.nz, dist = h.t;
    if (pr_add(pr_add(pr_mul(nx, nx), pr_mul(ny, ny)), pr_mul(nz, nz)) <= 1.0e-24) {
      nx = -dx;
      ny = -dy;
      nz = -dz;
    }
    if (!kPenetration) {
      acc[0] += 1.0;
      acc[1] += dist;
    }
    if (hit_point) {
      ox = pr_add(ox, pr_mul(dx, dist));
      oy = pr_add(oy, pr_mul(dy, dist));
      oz = pr_add(oz, pr_mul(dz, dist));
    }
    for (int bounces = 0;;) {
      if (!kPenetration) acc[4] += 1.0;
      const double u = mb_rand(state);
      if (u < eps) {
        if (kPenetration) acc[2] += 1.0;
        break;
      }
      const double px = dx, py = dy, pz = dz;
      mb_lambertian(state, nx, ny, nz, dx, dy, dz);
      if (!kPenetration) {
        const double mu = pr_add(pr_add(pr_mul(px, dx), pr_mul(py, dy)), pr_mul(pz, dz));
        acc[5] += 1.0;
        acc[6] += mu;
        acc[7] += pr_mul(mu, mu);
      }
      if (++bounces >= max_bounces) {
        if (kPenetration) acc[3] += 1.0;
        break;
      }
      if (hit_point) {
        ox = pr_add(ox, pr_mul(nx, 1.0e-9));
        oy = pr_add(oy, pr_mul(ny, 1.0e-9));
        oz = pr_add(oz, pr_mul(nz, 1.0e-9));
      } else {
        ox = pr_add(pr_add(ox, pr_mul(px, dist)), pr_mul(nx, 1.0e-9));
        oy = pr_add(pr_add(oy, pr_mul(py, dist)), pr_mul(ny, 1.0e-9));
        oz = pr_add(pr_add(oz, pr_mul(pz, dist)), pr_mul(nz, 1.0e-9));
      }
      h = mb_trace(g, ox, oy, oz, dx, dy, dz);
      if (h.fate != 0) {
        if (kPenetration) acc[h.fate == 1 ? 0 : (h.fate == 2 ? 1 : 3)] += 1.0;
        break;
      }
      nx = h.nx;
      ny = h.ny;
      nz = h.nz;
      dist = h.t;
      if (pr_add(pr_add(pr_mul(nx, nx), pr_mul(ny, ny)), pr_mul(nz, nz)) <= 1.0e-24) {
        nx = -dx;
        ny = -dy;
        nz = -dz;
      }
      ox = pr_add(ox, pr_mul(dx, dist));
      oy = pr_add(oy, pr_mul(dy, dist));
      oz = pr_add(oz, pr_mul(dz, dist));
    }
  }
  // one partial per warp (no block barrier: a warp whose rays have ended does not wait for the others)
#pragma unroll
  for (int k = 0; k < 8; ++k)
    for (int o = 16; o > 0; o >>= 1) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], o);
  if ((threadIdx.x & 31) == 0) {
    const int64_t slot = (int64_t)blockIdx.x * (kMbThreads / 32) + (threadIdx.x >> 5);
#pragma unroll
    for (int k = 0; k < 8; ++k) partial[slot * 8 + k] = acc[k];
  }
}

}  // namespace

int sum_partials(const double* partial, int blocks, int K, double* out, cudaStream_t s);

// One run of n rays of one seed: the 8 tallies (properties) or 4 counts (penetration).
int multibounce(const pr_case* c, bool penetration, double eps, int64_t n, uint32_t seed, int max_bounces,
                int hit_point, double* out8, cudaStream_t s) {
  const int blocks = (int)std::min<int64_t>((n + kMbThreads - 1) / kMbThreads, (int64_t)sm_count() * 64);
  const int warps = blocks * (kMbThreads / 32);
  DevBuf<double> partial, out;
  PR_TRY(partial.alloc((size_t)warps * 8, s));
  PR_TRY(out.alloc(8, s));
  const MbGrid g{c->occ.ptr, (int)c->nx, (int)c->ny, (int)c->nz};
  if (penetration)
    ::pr::launch_mark(), k_multibounce<true><<<blocks, kMbThreads, 0, s>>>(g, n, seed, eps, max_bounces, hit_point, partial.ptr);
  else
    ::pr::launch_mark(), k_multibounce<false><<<blocks, kMbThreads, 0, s>>>(g, n, seed, eps, max_bounces, hit_point, partial.ptr);
  PR_CUDA(cudaGetLastError());
  PR_TRY(sum_partials(partial.ptr, warps, 8, out.ptr, s));
  PR_CUDA(cudaMemcpyAsync(out8, out.ptr, 64, cudaMemcpyDeviceToHost, s));
  PR_CUDA(cudaStreamSynchronize(s));
  return PR_OK;
}

}  // namespace pr

using namespace pr;

extern "C" {

PR_API int pr_radiative_properties(const pr_case* c, double epsilon, int64_t n_rays, uint32_t seed, int restart,
                                   int max_bounces, pr_properties_tally* out, void* stream) {
  if (!c || !out) {
    set_error("case and out must not be NULL");
    return PR_ERR_ARG;
  }
  PR_ARG(n_rays > 0 && max_bounces > 0, "n_rays and max_bounces must be positive");
  PR_ARG(restart == PR_RESTART_ARTICLE || restart == PR_RESTART_HIT_POINT, "unknown restart rule %d", restart);
  DeviceGuard guard(c->device);
  double t[8];
  PR_TRY(multibounce(c, false, epsilon, n_rays, seed, max_bounces, restart == PR_RESTART_HIT_POINT, t,
                     (cudaStream_t)stream));
  out->events = (int64_t)t[0];
  out->event_length = t[1];
  out->censored = (int64_t)t[2];
  out->censored_length = t[3];
  out->interactions = (int64_t)t[4];
  out->scattered = (int64_t)t[5];
  out->sum_mu = t[6];
  out->sum_mu2 = t[7];
  return PR_OK;
}

PR_API int pr_penetration(const pr_case* c, double epsilon, int64_t n_rays, uint32_t seed, int restart,
                          int max_bounces, int64_t* counts, void* stream) {
  if (!c || !counts) {
    set_error("case and counts must not be NULL");
    return PR_ERR_ARG;
  }
  PR_ARG(n_rays > 0 && max_bounces > 0, "n_rays and max_bounces must be positive");
  PR_ARG(restart == PR_RESTART_ARTICLE || restart == PR_RESTART_HIT_POINT, "unknown restart rule %d", restart);
  DeviceGuard guard(c->device);
  double t[8];
  PR_TRY(multibounce(c, true, epsilon, n_rays, seed, max_bounces, restart == PR_RESTART_HIT_POINT, t,
                     (cudaStream_t)stream));
  for (int k = 0; k < 4; ++k) counts[k] = (int64_t)t[k];
  return PR_OK;
}

}  // extern "C"
