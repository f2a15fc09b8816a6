// Ray generation, first-hit traversal and per-patch count reduction on sm_100a.
//
// Ray stream (generate_rays, porerad/view_factors.py:135-182): ray r of patch p in
// the block of seed s takes draws (p*R + r)*4 + c, c = 0..3, of that block's PCG64
// stream.  Each thread jumps its stream there with the power-of-two affine maps of
// the LCG, so rays are generated on the fly in any order and never stored.
//   c = 0, 1: origin offsets clip(u, 1e-12, 1 - 1e-12) - 0.5 along the two face
//             tangents, then y, z wrapped with NumPy's float remainder;
//   c = 2, 3: radius = sqrt(u2), azimuth = (2 pi) u3, cos(theta) = sqrt(1 - u2);
//             the direction is divided by sqrt((dx^2 + dy^2) + dz^2).
// Traversal (_trace_kernel, view_factors.py:202-258): Amanatides-Woo cell walk in
// binary64 with the 1e-12 tie tolerance, periodic y/z, exits through x < 0 (hot
// wall) or x >= nx (cold wall), step cap max(10 N^3 + 10, min(8 nx (1 + (|dy|+|dz|)
// /|dx|) + 100, 1e8)).  Every operation is an explicit round-to-nearest intrinsic,
// so the arithmetic is the reference's operation for operation.  The occupancy
// probe reads one bit of the packed grid (L1/L2 resident).
#include <cub/device/device_scan.cuh>

#include <map>
#include <mutex>
#include <tuple>

#include "pr_math.cuh"
#include "pr_objects.cuh"

namespace pr {

// Per-seed table of LCG jump maps (A, C): state -> A state + C.
//   [0, 128):   the maps of 2^i steps, i = 0..63
//   [128, 192): the maps of 4 l steps, l = 0..31 (lane offsets inside a batch of 32 rays)
//   [192, 194): the map of 128 steps (one batch of 32 rays)
static constexpr int kMapStride = 256;
static constexpr int kMapSmall = 128;
static constexpr int kMapBatch = 192;

#define PR_TIE 1.0e-12
#ifndef PR_FULL
#define PR_FULL 0xffffffffu
#endif
#define PR_FAR 1.0e300
#define PR_TWO_PI 0x1.921fb54442d18p+2  // the binary64 product 2.0 * numpy.pi

struct Geom {
  const uint32_t* __restrict__ occ;
  const int32_t* __restrict__ cfp;
  const int32_t* __restrict__ hot;
  const int32_t* __restrict__ cold;
  int32_t nx, ny, nz;
  int64_t n_cells;
};

struct RaySrc {
  const double* __restrict__ origin;  // (P, 3)
  const int8_t* __restrict__ code;    // emission normal 0..5
  const pr_u128* __restrict__ maps;   // per seed: kMapStride entries, see SeedTables
  const pr_u128* __restrict__ state;  // per seed
  const pr_u128* __restrict__ inc;    // per seed
  double ny_d, nz_d;
};

__device__ __forceinline__ double clip_edge(double u) {
  const double lo = 1.0e-12, hi = 1.0 - 1.0e-12;
  return u < lo ? lo : (u > hi ? hi : u);
}

// NumPy's float remainder by b > 0 for the origins, whose values lie in (-b, 2b):
// a - b is exact there (Sterbenz), a + b is the single rounded add NumPy makes for a
// negative fmod result, and a zero result is +0.0.  Other values take the general path.
__device__ __forceinline__ double wrap_origin(double a, double b) {
  if (a > -b && a < 2.0 * b) {
    if (a >= b) return pr_sub(a, b);
    if (a < 0.0) return pr_add(a, b);
    return a == 0.0 ? 0.0 : a;
  }
  return pr_pymod_pos(a, b);
}

// Origin and unit direction of ray r of patch p, block s (view_factors.py:148-181).
// Tangent axes (first, second) of a normal along x, y, z: (y, z), (x, z), (x, y).
__device__ __forceinline__ void make_ray(const RaySrc& src, int64_t p, int64_t r, int64_t R, int s,
                                         double& ox, double& oy, double& oz, double& dx, double& dy, double& dz) {
  const pr_u128* maps = src.maps + (int64_t)s * kMapStride;
  pr_u128 st = pr_pcg_jump(src.state[s], (uint64_t)((p * R + r) * 4), maps);
  const pr_u128 inc = src.inc[s];
  const double u0 = pr_pcg_next_double(&st, inc);
  const double u1 = pr_pcg_next_double(&st, inc);
  const double u2 = pr_pcg_next_double(&st, inc);
  const double u3 = pr_pcg_next_double(&st, inc);
  const int code = src.code[p];
  const int ax = code >> 1;
  const double sign = (code & 1) ? -1.0 : 1.0;
  ox = src.origin[3 * p];
  oy = src.origin[3 * p + 1];
  oz = src.origin[3 * p + 2];
  const double ta = pr_sub(clip_edge(u0), 0.5);
  const double tb = pr_sub(clip_edge(u1), 0.5);
  if (ax == 0) {
    oy = pr_add(oy, ta);
    oz = pr_add(oz, tb);
  } else if (ax == 1) {
    ox = pr_add(ox, ta);
    oz = pr_add(oz, tb);
  } else {
    ox = pr_add(ox, ta);
    oy = pr_add(oy, tb);
  }
  oy = wrap_origin(oy, src.ny_d);
  oz = wrap_origin(oz, src.nz_d);
  const double radius = pr_sqrt(u2);
  double sn, cs;
  pr_sincos(pr_mul(PR_TWO_PI, u3), &sn, &cs);
  const double la = pr_mul(radius, cs);
  const double lb = sign * pr_mul(radius, sn);
  const double dn = sign * pr_sqrt(pr_sub(1.0, u2));
  if (ax == 0) {
    dx = dn; dy = la; dz = lb;
  } else if (ax == 1) {
    dx = la; dy = dn; dz = lb;
  } else {
    dx = la; dy = lb; dz = dn;
  }
  const double len = pr_sqrt(pr_add(pr_add(pr_mul(dx, dx), pr_mul(dy, dy)), pr_mul(dz, dz)));
  dx = pr_div(dx, len);
  dy = pr_div(dy, len);
  dz = pr_div(dz, len);
}

__device__ __forceinline__ int64_t first_cell(double pos, double dir) {
  int64_t idx = (int64_t)floor(pos);
  if (dir < 0.0 && fabs(pr_sub(pos, rint(pos))) <= PR_TIE) idx -= 1;
  return idx;
}

__device__ __forceinline__ void axis_setup(double pos, double dir, int64_t idx, int& step, double& tmax,
                                           double& tdel) {
  if (dir > 0.0) {
    step = 1;
    tmax = pr_div(pr_sub(pr_add((double)idx, 1.0), pos), dir);
    tdel = pr_div(1.0, dir);
  } else if (dir < 0.0) {
    step = -1;
    tmax = pr_div(pr_sub((double)idx, pos), dir);
    tdel = pr_div(-1.0, dir);
  } else {
    step = 0;
    tmax = PR_FAR;
    tdel = PR_FAR;
  }
}

__device__ __forceinline__ int64_t imod(int64_t a, int64_t n) {
  int64_t m = a % n;
  return m < 0 ? m + n : m;
}

// imod for a value given as a binary64 integer (a floor) and n < 2^31: 32-bit arithmetic when
// the value fits in 32 bits (every wrap of a ray's coordinate in practice), else imod.
__device__ __forceinline__ int imod_floor(double f, int n) {
  if (fabs(f) < 2147483647.0) {
    const int m = (int)f % n;
    return m < 0 ? m + n : m;
  }
  return (int)imod((int64_t)f, (int64_t)n);
}

// First patch hit by the ray, or -1 when it resolves none (the reference's
// failed flag); *steps counts the cells visited.
__device__ int32_t dda_first_hit(const Geom& g, double ox, double oy, double oz, double dx, double dy,
                                 double dz, int64_t* steps) {
  *steps = 0;
  if (dx == 0.0) return -1;
  int64_t i = first_cell(ox, dx);
  const int64_t j0 = first_cell(oy, dy), k0 = first_cell(oz, dz);
  int sx, sy, sz;
  double tx, ty, tz, ddx, ddy, ddz;
  axis_setup(ox, dx, i, sx, tx, ddx);
  axis_setup(oy, dy, j0, sy, ty, ddy);
  axis_setup(oz, dz, k0, sz, tz, ddz);
  int jj = (int)imod(j0, g.ny), kk = (int)imod(k0, g.nz);
  double t = 0.0;
  int face = -1;
  double scale = pr_add(pr_mul(pr_mul(8.0, (double)g.nx),
                               pr_add(1.0, pr_div(pr_add(fabs(dy), fabs(dz)), fabs(dx)))), 100.0);
  if (scale > 100000000.0) scale = 100000000.0;
  int64_t cap = 10 * g.n_cells + 10;
  if ((int64_t)scale > cap) cap = (int64_t)scale;
  int64_t it = 0;
  for (; it < cap; ++it) {
    if (i < 0 || i >= g.nx) {
      const int64_t wj = imod((int64_t)floor(pr_add(oy, pr_mul(dy, t))), g.ny);
      const int64_t wk = imod((int64_t)floor(pr_add(oz, pr_mul(dz, t))), g.nz);
      *steps = it + 1;
      return i < 0 ? g.hot[wj * g.nz + wk] : g.cold[wj * g.nz + wk];
    }
    const int64_t row = i * g.ny + jj;
    const int64_t cell = row * g.nz + kk;
    const uint32_t word = __ldg(g.occ + (cell >> 5));
    if ((word >> (cell & 31)) & 1u) {
      *steps = it + 1;
      return face >= 0 ? __ldg(g.cfp + (row * g.nz + kk) * 6 + face) : -1;
    }
    double tn = tx;
    if (ty < tn) tn = ty;
    if (tz < tn) tn = tz;
    const bool cx = fabs(pr_sub(tx, tn)) <= PR_TIE;
    const bool cy = fabs(pr_sub(ty, tn)) <= PR_TIE;
    const bool cz = fabs(pr_sub(tz, tn)) <= PR_TIE;
    if (cx) {
      i += sx;
      tx = pr_add(tx, ddx);
      face = sx > 0 ? 1 : 0;
    }
    if (cy) {
      jj += sy;
      if (jj == g.ny) jj = 0;
      else if (jj < 0) jj = g.ny - 1;
      ty = pr_add(ty, ddy);
      if (!cx) face = sy > 0 ? 3 : 2;
    }
    if (cz) {
      kk += sz;
      if (kk == g.nz) kk = 0;
      else if (kk < 0) kk = g.nz - 1;
      tz = pr_add(tz, ddz);
      if (!cx && !cy) face = sz > 0 ? 5 : 4;
    }
    t = tn;
  }
  *steps = it;
  return -1;
}

__device__ __forceinline__ void block_add_i64(int64_t v, unsigned long long* target) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0 && v) atomicAdd(target, (unsigned long long)v);
}

__global__ void k_generate(RaySrc src, int64_t p0, int64_t np, int64_t R, double* __restrict__ origins,
                           double* __restrict__ dirs) {
  const int64_t n = np * R;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
    double ox, oy, oz, dx, dy, dz;
    make_ray(src, p0 + q / R, q % R, R, 0, ox, oy, oz, dx, dy, dz);
    origins[3 * q] = ox;
    origins[3 * q + 1] = oy;
    origins[3 * q + 2] = oz;
    dirs[3 * q] = dx;
    dirs[3 * q + 1] = dy;
    dirs[3 * q + 2] = dz;
  }
}

__global__ void __launch_bounds__(256) k_trace_given(Geom g, const double* __restrict__ origins,
                                                     const double* __restrict__ dirs, int64_t n,
                                                     int32_t* __restrict__ recv,
                                                     unsigned long long* __restrict__ counters) {
  int64_t my_steps = 0, my_fail = 0;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
    int64_t st = 0;
    const int32_t hit = dda_first_hit(g, origins[3 * q], origins[3 * q + 1], origins[3 * q + 2], dirs[3 * q],
                                      dirs[3 * q + 1], dirs[3 * q + 2], &st);
    my_steps += st;
    my_fail += hit < 0;
    recv[q] = hit;
  }
  block_add_i64(my_steps, counters + 0);
  block_add_i64(my_fail, counters + 1);
}

// ---------------------------------------------------------------------------
// Pooled traversal.  A chunk of rays is numbered seed-major, g = (s * np + (p - p0)) * R + r,
// so inside one seed block consecutive rays are 4 draws apart in their PCG64 stream.
// Each warp grabs units of kUnit consecutive rays from a global counter, generates
// them 32 at a time with all lanes converged (one 128-step map advances the batch base,
// one small map per lane), runs the DDA setup there too, and parks the ready states
// in a warp-private shared-memory pool.  Idle lanes take rays from the pool between
// bursts of kBurst DDA steps, so the warp no longer waits for its longest ray.
static constexpr int kPool = 64;   // pool slots per warp (two batches)
static constexpr int kWarps = 4;   // warps per block
static constexpr int kUnit = 512;  // rays per work grab

struct WarpPool {
  double tx[kPool], ty[kPool], tz[kPool], ddx[kPool], ddy[kPool], ddz[kPool];
  double oy[kPool], oz[kPool], dy[kPool], dz[kPool];
  int i[kPool], jj[kPool], kk[kPool], meta[kPool], cap[kPool], q[kPool];
  double eoy[32], eoz[32], edy[32], edz[32];  // wall-exit data of each lane's current ray
};

// One chunk of a launch: the rays of patches [p0, p0 + np) of one case, numbered seed-major
// inside the chunk (g = (s * np + p - p0) * R + r) and placed at global ray indices
// [start, start + n) of the launch, start a multiple of kUnit.  A launch (a wave) may hold
// chunks of many cases of different sizes.  Its rays' hit codes go to recv[start + g].
struct WaveChunk {
  const uint32_t* occ;
  const double* origin;
  const int8_t* code;
  const pr_u128* maps;   // kMapStride maps per seed of this case
  const pr_u128* state;  // per seed
  const pr_u128* inc;    // per seed
  int64_t n, np, p0, R, start, n_cells;
  int32_t nx, ny, nz;
  double ny_d, nz_d;
};

// Ray (origin, direction) of patch p from a positioned stream (view_factors.py:148-181).
__device__ __forceinline__ void ray_from_stream(const WaveChunk& src, pr_u128 st, pr_u128 inc, int64_t p, double& ox,
                                                double& oy, double& oz, double& dx, double& dy, double& dz) {
  const double u0 = pr_pcg_next_double(&st, inc);
  const double u1 = pr_pcg_next_double(&st, inc);
  const double u2 = pr_pcg_next_double(&st, inc);
  const double u3 = pr_pcg_next_double(&st, inc);
  const int code = src.code[p];
  const int ax = code >> 1;
  const double sign = (code & 1) ? -1.0 : 1.0;
  ox = src.origin[3 * p];
  oy = src.origin[3 * p + 1];
  oz = src.origin[3 * p + 2];
  const double ta = pr_sub(clip_edge(u0), 0.5);
  const double tb = pr_sub(clip_edge(u1), 0.5);
  if (ax == 0) {
    oy = pr_add(oy, ta);
    oz = pr_add(oz, tb);
  } else if (ax == 1) {
    ox = pr_add(ox, ta);
    oz = pr_add(oz, tb);
  } else {
    ox = pr_add(ox, ta);
    oy = pr_add(oy, tb);
  }
  oy = wrap_origin(oy, src.ny_d);
  oz = wrap_origin(oz, src.nz_d);
  const double radius = pr_sqrt(u2);
  double sn, cs;
  pr_sincos(pr_mul(PR_TWO_PI, u3), &sn, &cs);
  const double la = pr_mul(radius, cs);
  const double lb = sign * pr_mul(radius, sn);
  const double dn = sign * pr_sqrt(pr_sub(1.0, u2));
  if (ax == 0) {
    dx = dn; dy = la; dz = lb;
  } else if (ax == 1) {
    dx = la; dy = dn; dz = lb;
  } else {
    dx = la; dy = lb; dz = dn;
  }
  const double len = pr_sqrt(pr_add(pr_add(pr_mul(dx, dx), pr_mul(dy, dy)), pr_mul(dz, dz)));
  dx = pr_div(dx, len);
  dy = pr_div(dy, len);
  dz = pr_div(dz, len);
}

__device__ __forceinline__ void flush_chunk_counters(long long& steps, long long& fails,
                                                     unsigned long long* __restrict__ ctr, int lane) {
  for (int o = 16; o > 0; o >>= 1) {
    steps += __shfl_xor_sync(PR_FULL, steps, o);
    fails += __shfl_xor_sync(PR_FULL, fails, o);
  }
  if (lane == 0) {
    if (steps) atomicAdd(ctr, (unsigned long long)steps);
    if (fails) atomicAdd(ctr + 1, (unsigned long long)fails);
  }
  steps = 0;
  fails = 0;
}

// chunk holding global ray index u (chunks sorted by start)
__device__ __forceinline__ int find_chunk(const WaveChunk* __restrict__ chunks, int n_chunks, int64_t u) {
  int lo = 0, hi = n_chunks - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (chunks[mid].start <= u) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// The pooled traversal over a table of chunks.  A warp works on one chunk at a time: when
// its next work unit belongs to another chunk it stops generating, drains its lanes and
// pool, flushes the chunk's step/failure counters (chunk_ctr[2 c], [2 c + 1]) and switches.
template <int kMinBlocks, int kBurst, int kLook>
__global__ void __launch_bounds__(kWarps * 32, kMinBlocks) k_trace_pool(const WaveChunk* __restrict__ chunks,
                                                                        int n_chunks, int64_t total,
                                                                        int32_t* __restrict__ recv,
                                                                        unsigned long long* __restrict__ work,
                                                                        unsigned long long* __restrict__ chunk_ctr) {
  __shared__ WarpPool pools[kWarps];
  WarpPool& pool = pools[threadIdx.x >> 5];
  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;

  int64_t unit_next = 0, unit_end = 0;  // warp-uniform: the work unit being generated
  int unit_chunk = -1, cur = -1;        // warp-uniform: its chunk, and the chunk of the rays in flight
  const uint32_t* occ = nullptr;        // warp-uniform geometry of chunk cur
  int nx = 0, ny = 0, nz = 0;
  int head = 0, tail = 0;               // warp-uniform pool cursors
  bool more = true;                     // warp-uniform
  pr_u128 base_st{0, 0};
  int base_s = -1;
  uint64_t base_m = 0;

  bool active = false;
  double tx = 0, ty = 0, tz = 0, ddx = 0, ddy = 0, ddz = 0, t = 0;
  int i = 0, jj = 0, kk = 0, sx = 0, sy = 0, sz = 0, face = -1, it = 0, cap = 0, q = 0;
  long long my_steps = 0, my_fail = 0;

  for (;;) {
    // ---- switch to the chunk of the pending unit once nothing of the previous one is in flight
    if (unit_chunk != cur && unit_next < unit_end && head == tail && !__any_sync(PR_FULL, active)) {
      if (cur >= 0) flush_chunk_counters(my_steps, my_fail, chunk_ctr + 2 * cur, lane);
      cur = unit_chunk;
      occ = chunks[cur].occ;
      nx = chunks[cur].nx;
      ny = chunks[cur].ny;
      nz = chunks[cur].nz;
      base_s = -1;
    }
    // ---- generate one batch of 32 rays when the pool has room for it
    if (more && tail - head <= kPool - 32) {
      if (unit_next >= unit_end) {
        unsigned long long u = 0;
        if (lane == 0) u = atomicAdd(work, (unsigned long long)kUnit);
        u = __shfl_sync(PR_FULL, u, 0);
        if ((int64_t)u >= total) {
          more = false;
        } else {
          unit_chunk = find_chunk(chunks, n_chunks, (int64_t)u);
          unit_next = (int64_t)u;
          unit_end = min((int64_t)u + kUnit, chunks[unit_chunk].start + chunks[unit_chunk].n);
        }
      }
      if (more && unit_chunk == cur && unit_next < unit_end) {
        const WaveChunk& C = chunks[cur];
        const int64_t npR = C.np * C.R;
        const uint64_t base_draw = (uint64_t)C.p0 * (uint64_t)C.R;  // stream ray index of the chunk's first ray
        const int64_t g0 = unit_next - C.start;                      // chunk-local index of the batch
        const int cnt = (int)min((int64_t)32, unit_end - unit_next);
        unit_next += cnt;
        // batch base stream (warp-uniform)
        const int s0 = (int)(g0 / npR);
        const uint64_t m0 = (base_draw + (uint64_t)(g0 - (int64_t)s0 * npR)) * 4u;
        const pr_u128* maps0 = C.maps + (int64_t)s0 * kMapStride;
        if (base_s == s0 && m0 == base_m + 128u) {
          base_st = pr_u128_affine(maps0[kMapBatch], maps0[kMapBatch + 1], base_st);
        } else {
          base_st = pr_pcg_jump(C.state[s0], m0, maps0);
        }
        base_s = s0;
        base_m = m0;
        if (lane < cnt) {
          const int64_t gq = g0 + lane;
          // seed block and patch of ray gq without 64-bit divisions per lane: from the batch's
          // (s0, rem0), at most a few seed blocks further (32 rays per batch)
          int sq = s0;
          int64_t rem = (g0 - (int64_t)s0 * npR) + lane;
          while (rem >= npR) {
            rem -= npR;
            ++sq;
          }
          const int64_t p = C.p0 + (rem < (int64_t)UINT32_MAX && C.R < (int64_t)UINT32_MAX
                                        ? (int64_t)((uint32_t)rem / (uint32_t)C.R)
                                        : rem / C.R);
          pr_u128 st;
          if (sq == s0) {
            st = pr_u128_affine(maps0[kMapSmall + 2 * lane], maps0[kMapSmall + 2 * lane + 1], base_st);
          } else {
            const pr_u128* mq = C.maps + (int64_t)sq * kMapStride;
            st = pr_pcg_jump(C.state[sq], (base_draw + (uint64_t)rem) * 4u, mq);
          }
          double ox, oy, oz, dx, dy, dz;
          ray_from_stream(C, st, C.inc[sq], p, ox, oy, oz, dx, dy, dz);
          // DDA setup (view_factors.py:213-224)
          const int slot = (tail + lane) & (kPool - 1);
          int c = 0, si = 0, sj = 0, sk = 0, ci = 0, cj = 0, ck = 0;
          double a = 0, b = 0, e = 0, da = 0, db = 0, de = 0;
          if (dx != 0.0) {
            const int64_t i0 = first_cell(ox, dx), j0 = first_cell(oy, dy), k0 = first_cell(oz, dz);
            axis_setup(ox, dx, i0, si, a, da);
            axis_setup(oy, dy, j0, sj, b, db);
            axis_setup(oz, dz, k0, sk, e, de);
            ci = (int)max((int64_t)-1, min(i0, (int64_t)nx));
            cj = imod_floor((double)j0, ny);
            ck = imod_floor((double)k0, nz);
            double scale = pr_add(pr_mul(pr_mul(8.0, (double)nx),
                                         pr_add(1.0, pr_div(pr_add(fabs(dy), fabs(dz)), fabs(dx)))), 100.0);
            if (scale > 100000000.0) scale = 100000000.0;
            c = (int)min((int64_t)INT32_MAX, 10 * C.n_cells + 10);
            if ((int64_t)scale > (int64_t)c) c = (int)scale;
          }
          pool.tx[slot] = a; pool.ty[slot] = b; pool.tz[slot] = e;
          pool.ddx[slot] = da; pool.ddy[slot] = db; pool.ddz[slot] = de;
          pool.oy[slot] = oy; pool.oz[slot] = oz; pool.dy[slot] = dy; pool.dz[slot] = dz;
          pool.i[slot] = ci; pool.jj[slot] = cj; pool.kk[slot] = ck;
          pool.meta[slot] = (si + 1) | ((sj + 1) << 2) | ((sk + 1) << 4);
          pool.cap[slot] = c;
          pool.q[slot] = (int)(C.start + gq);  // wave-wide ray index (< 2^31)
        }
        tail += cnt;
        __syncwarp();
      }
    }
    // ---- idle lanes take ready rays
    const unsigned idle = __ballot_sync(PR_FULL, !active);
    const int avail = tail - head;
    if (!active) {
      const int rank = __popc(idle & lt);
      if (rank < avail) {
        const int slot = (head + rank) & (kPool - 1);
        tx = pool.tx[slot]; ty = pool.ty[slot]; tz = pool.tz[slot];
        ddx = pool.ddx[slot]; ddy = pool.ddy[slot]; ddz = pool.ddz[slot];
        i = pool.i[slot]; jj = pool.jj[slot]; kk = pool.kk[slot];
        const int meta = pool.meta[slot];
        sx = (meta & 3) - 1;
        sy = ((meta >> 2) & 3) - 1;
        sz = ((meta >> 4) & 3) - 1;
        cap = pool.cap[slot];
        q = pool.q[slot];
        pool.eoy[lane] = pool.oy[slot];
        pool.eoz[lane] = pool.oz[slot];
        pool.edy[lane] = pool.dy[slot];
        pool.edz[lane] = pool.dz[slot];
        t = 0.0;
        face = -1;
        it = 0;
        active = true;
      }
    }
    head += min(__popc(idle), avail);
    __syncwarp();
    if (!more && head == tail && !__any_sync(PR_FULL, active)) break;
    // ---- DDA steps (view_factors.py:225-255), kBurst rounds per refill
    if constexpr (kLook == 0) {
  #pragma unroll 1
      for (int b = 0; b < kBurst; ++b) {
        if (!active) continue;
        int32_t hit = -2;
        if (it >= cap) {
          hit = -1;
        } else {
          ++it;
          if ((unsigned)i >= (unsigned)nx) {
            // hit code of a wall: 6 n_cells + (0 hot | ny nz cold) + j nz + k
            const int wj = imod_floor(floor(pr_add(pool.eoy[lane], pr_mul(pool.edy[lane], t))), ny);
            const int wk = imod_floor(floor(pr_add(pool.eoz[lane], pr_mul(pool.edz[lane], t))), nz);
            hit = 6 * nx * ny * nz + (i < 0 ? 0 : ny * nz) + wj * nz + wk;
          } else {
            const int row = i * ny + jj;
            const int cell = row * nz + kk;
            const uint32_t word = __ldg(occ + (cell >> 5));
            if ((word >> (cell & 31)) & 1u) {
              // hit code of a cell face: its cell_face_patch index
              hit = face >= 0 ? cell * 6 + face : -1;
            } else {
              double tn = tx;
              if (ty < tn) tn = ty;
              if (tz < tn) tn = tz;
              const bool cx = fabs(pr_sub(tx, tn)) <= PR_TIE;
              const bool cy = fabs(pr_sub(ty, tn)) <= PR_TIE;
              const bool cz = fabs(pr_sub(tz, tn)) <= PR_TIE;
              if (cx) {
                i += sx;
                tx = pr_add(tx, ddx);
                face = sx > 0 ? 1 : 0;
              }
              if (cy) {
                jj += sy;
                jj = jj == ny ? 0 : (jj < 0 ? ny - 1 : jj);
                ty = pr_add(ty, ddy);
                if (!cx) face = sy > 0 ? 3 : 2;
              }
              if (cz) {
                kk += sz;
                kk = kk == nz ? 0 : (kk < 0 ? nz - 1 : kk);
                tz = pr_add(tz, ddz);
                if (!cx && !cy) face = sz > 0 ? 5 : 4;
              }
              t = tn;
            }
          }
        }
        if (hit != -2) {
          recv[q] = hit;  // no load on this path: the RLE pass maps codes to patches
          my_steps += it;
          my_fail += hit < 0;
          active = false;
        }
      }
    } else {
      // Lookahead rounds: the DDA state advances through up to kLook cells without waiting
      // for their occupancy (the arithmetic does not depend on it), recording each cell's
      // occupancy bit and hit code; the kLook occupancy words are then loaded together and
      // the first solid cell decides.  A wall or the step cap ends the round early.  Step
      // counts and hit codes are those of the one-cell-at-a-time loop: cells are visited in
      // the same order with the same arithmetic, and the state past a solid cell is dropped.
#pragma unroll 1
      for (int b = 0; b < kBurst; ++b) {
        if (!active) continue;
        int32_t cell[kLook], code[kLook];  // each recorded cell and its hit code
        int m = 0;      // cells recorded
        int stop = 0;   // 0 none, 1 wall at position m, 2 step cap at position m
        int32_t wall_code = -1;
        const int left = cap - it;  // steps left before the ray's step cap
#pragma unroll
        for (int p = 0; p < kLook; ++p) {
          cell[p] = 0;
          code[p] = -1;
          if (stop == 0) {  // while no stop is recorded, m == p
            if (p >= left) {
              stop = 2;
            } else if ((unsigned)i >= (unsigned)nx) {
              stop = 1;  // the wall's hit code is formed after the round (i and t stay as they are)
            } else {
              cell[p] = (i * ny + jj) * nz + kk;
              code[p] = face >= 0 ? cell[p] * 6 + face : -1;
              m = p + 1;
              double tn = tx;
              if (ty < tn) tn = ty;
              if (tz < tn) tn = tz;
              const bool cx = fabs(pr_sub(tx, tn)) <= PR_TIE;
              const bool cy = fabs(pr_sub(ty, tn)) <= PR_TIE;
              const bool cz = fabs(pr_sub(tz, tn)) <= PR_TIE;
              if (cx) {
                i += sx;
                tx = pr_add(tx, ddx);
                face = sx > 0 ? 1 : 0;
              }
              if (cy) {
                jj += sy;
                jj = jj == ny ? 0 : (jj < 0 ? ny - 1 : jj);
                ty = pr_add(ty, ddy);
                if (!cx) face = sy > 0 ? 3 : 2;
              }
              if (cz) {
                kk += sz;
                kk = kk == nz ? 0 : (kk < 0 ? nz - 1 : kk);
                tz = pr_add(tz, ddz);
                if (!cx && !cy) face = sz > 0 ? 5 : 4;
              }
              t = tn;
            }
          }
        }
        // A wall exit's hit code, formed once per round outside the unrolled cells: one copy of
        // its floor/modulo code instead of kLook (measured 7 % faster on the c2 traversal).
        if (stop == 1) {
          const int wj = (int)imod((int64_t)floor(pr_add(pool.eoy[lane], pr_mul(pool.edy[lane], t))), ny);
          const int wk = (int)imod((int64_t)floor(pr_add(pool.eoz[lane], pr_mul(pool.edz[lane], t))), nz);
          wall_code = 6 * nx * ny * nz + (i < 0 ? 0 : ny * nz) + wj * nz + wk;
        }
        uint32_t word[kLook];
#pragma unroll
        for (int p = 0; p < kLook; ++p) word[p] = p < m ? __ldg(occ + (cell[p] >> 5)) : 0u;
        int32_t hit = -2;
        int used = m;
#pragma unroll
        for (int p = kLook - 1; p >= 0; --p) {
          if (p < m && ((word[p] >> (cell[p] & 31)) & 1u)) {
            hit = code[p];  // the cell_face_patch index
            used = p + 1;
          }
        }
        if (hit == -2) {
          if (stop == 1) {
            hit = wall_code;
            used = m + 1;
          } else if (stop == 2) {
            hit = -1;
            used = m;
          }
        }
        it += used;
        if (hit != -2) {
          recv[q] = hit;
          my_steps += it;
          my_fail += hit < 0;
          active = false;
        }
      }
    }
  }
  if (cur >= 0) flush_chunk_counters(my_steps, my_fail, chunk_ctr + 2 * cur, lane);
}

// Per origin patch: gather its L = S * R receivers (seed-major chunk layout), sort them
// in shared memory (bitonic), run-length encode into (receiver, count) pairs at
// out[(p - p0) * L ...], nnz[p - p0].
struct RleChunk {
  const int32_t* recv;  // hit codes of the chunk (seed-major)
  const int32_t* ftab;  // face table of its case: hit code -> receiving patch
  unsigned long long* fail;  // the chunk's failed-ray counter
  int64_t np;           // patches
  int64_t patch0;       // index of its first patch among the wave's patches
  int64_t ray0;         // offset of its rays (and stage entries) in the wave's buffers
};

__global__ void __launch_bounds__(512) k_patch_rle(const RleChunk* __restrict__ rc, int n_chunks,
                                                   int64_t total_patches, int L, int R, int Lpad,
                                                   int32_t* __restrict__ st_col, int32_t* __restrict__ st_cnt,
                                                   int32_t* __restrict__ nnz) {
  extern __shared__ int32_t sm[];
  int32_t* key = sm;          // Lpad
  int32_t* head = sm + Lpad;  // Lpad (positions of run heads)
  __shared__ int32_t warp_tot[16];
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int64_t gp = blockIdx.x; gp < total_patches; gp += gridDim.x) {
    int c = 0;
    {
      int lo = 0, hi = n_chunks - 1;
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (rc[mid].patch0 <= gp) lo = mid;
        else hi = mid - 1;
      }
      c = lo;
    }
    const int64_t p = gp - rc[c].patch0, np = rc[c].np;
    const int32_t* recv = rc[c].recv;
    const int32_t* ftab = rc[c].ftab;
    for (int i = tid; i < Lpad; i += nt) {
      if (i < L) {
        const int sd = i / R;
        const int32_t code = recv[((int64_t)sd * np + p) * R + (i - sd * R)];
        const int32_t r = code >= 0 ? __ldg(ftab + code) : -1;
        if (code >= 0 && r < 0) atomicAdd(rc[c].fail, 1ull);  // a face without a patch
        key[i] = r;
      } else {
        key[i] = INT32_MAX;
      }
    }
    __syncthreads();
    for (int k = 2; k <= Lpad; k <<= 1) {
      for (int j = k >> 1; j > 0; j >>= 1) {
        for (int t = tid; t < (Lpad >> 1); t += nt) {
          const int a = ((t / j) * 2 * j) + (t % j);
          const int b = a + j;
          const bool up = (a & k) == 0;
          const int32_t x = key[a], y = key[b];
          if ((x > y) == up) {
            key[a] = y;
            key[b] = x;
          }
        }
        __syncthreads();
      }
    }
    // heads: contiguous chunk per thread, then a block-wide exclusive scan
    const int per = (L + nt - 1) / nt;
    const int lo = tid * per, hi = min(L, lo + per);
    int mine = 0;
    for (int i = lo; i < hi; ++i) mine += (i == 0 || key[i] != key[i - 1]);
    int incl = mine;
    const int lane = tid & 31, wid = tid >> 5;
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    if (lane == 31) warp_tot[wid] = incl;
    __syncthreads();
    int base = 0, total = 0;
    for (int w = 0; w < (nt >> 5); ++w) {
      if (w < wid) base += warp_tot[w];
      total += warp_tot[w];
    }
    int u = base + incl - mine;
    for (int i = lo; i < hi; ++i)
      if (i == 0 || key[i] != key[i - 1]) head[u++] = i;
    __syncthreads();
    int32_t* oc = st_col + rc[c].ray0 + p * L;
    int32_t* on = st_cnt + rc[c].ray0 + p * L;
    for (int v = tid; v < total; v += nt) {
      const int h = head[v];
      const int e = v + 1 < total ? head[v + 1] : L;
      oc[v] = key[h];
      on[v] = e - h;
    }
    if (tid == 0) nnz[gp] = total;
    __syncthreads();
  }
}

// The same reduction with one warp per origin patch, for Lpad = 32 K <= 1024: the patch's
// keys sit in registers, element e = r * 32 + lane in register r of lane `lane`, and are
// sorted by the bitonic network (partners e ^ j: across lanes by shuffles for j < 32,
// across registers for j >= 32); run heads and tails come from neighbour shuffles and
// ballots, head positions go through the warp's shared row, and every tail writes its
// (receiver, count).  Output layout as k_patch_rle.
template <int K>
__global__ void __launch_bounds__(128) k_patch_rle_warp(const RleChunk* __restrict__ rc, int n_chunks,
                                                        int64_t total_patches, int L, int R,
                                                        int32_t* __restrict__ st_col, int32_t* __restrict__ st_cnt,
                                                        int32_t* __restrict__ nnz) {
  constexpr int N = 32 * K;
  __shared__ int32_t heads[4][N];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const unsigned lt = (1u << lane) - 1u;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t gp = blockIdx.x * (int64_t)(blockDim.x >> 5) + wid; gp < total_patches; gp += warps) {
    int c = 0;
    {
      int lo = 0, hi = n_chunks - 1;
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (rc[mid].patch0 <= gp) lo = mid;
        else hi = mid - 1;
      }
      c = lo;
    }
    const int64_t p = gp - rc[c].patch0, np = rc[c].np;
    const int32_t* recv = rc[c].recv;
    const int32_t* ftab = rc[c].ftab;
    int32_t x[K];
    int bad = 0;
#pragma unroll
    for (int r = 0; r < K; ++r) {
      const int e = r * 32 + lane;
      int32_t v = INT32_MAX;
      if (e < L) {
        const int sd = e / R;
        const int32_t code = recv[((int64_t)sd * np + p) * R + (e - sd * R)];
        v = code >= 0 ? __ldg(ftab + code) : -1;
        bad += code >= 0 && v < 0;  // a face without a patch
      }
      x[r] = v;
    }
    if (bad) atomicAdd(rc[c].fail, (unsigned long long)bad);
    // bitonic sort, ascending
#pragma unroll
    for (int k = 2; k <= N; k <<= 1) {
#pragma unroll
      for (int j = k >> 1; j > 0; j >>= 1) {
        if (j >= 32) {
          const int jr = j >> 5;
#pragma unroll
          for (int r = 0; r < K; ++r) {
            if ((r & jr) == 0) {
              const bool up = ((r * 32) & k) == 0;  // k >= 64 here: bit of r
              const int32_t a = x[r], b = x[r | jr];
              const bool sw = up ? (a > b) : (a < b);
              x[r] = sw ? b : a;
              x[r | jr] = sw ? a : b;
            }
          }
        } else {
          const bool lower = (lane & j) == 0;
#pragma unroll
          for (int r = 0; r < K; ++r) {
            const bool up = (k < 32 ? (lane & k) : ((r * 32) & k)) == 0;
            const int32_t y = __shfl_xor_sync(PR_FULL, x[r], j);
            const int32_t lo_v = min(x[r], y), hi_v = max(x[r], y);
            x[r] = (lower == up) ? lo_v : hi_v;
          }
        }
      }
    }
    // run heads (key differs from its predecessor) and tails (differs from its successor)
    int32_t* hrow = heads[wid];
    int base = 0;
#pragma unroll
    for (int r = 0; r < K; ++r) {
      const int e = r * 32 + lane;
      int32_t prev = __shfl_up_sync(PR_FULL, x[r], 1);
      const int32_t last_prev = __shfl_sync(PR_FULL, x[r > 0 ? r - 1 : 0], 31);
      if (lane == 0) prev = last_prev;
      const bool head = e < L && (e == 0 || x[r] != prev);
      const unsigned hb = __ballot_sync(PR_FULL, head);
      if (head) hrow[base + __popc(hb & lt)] = e;
      base += __popc(hb);
    }
    __syncwarp();
    int32_t* oc = st_col + rc[c].ray0 + p * L;
    int32_t* on = st_cnt + rc[c].ray0 + p * L;
    int runs = 0;  // heads at positions < e
#pragma unroll
    for (int r = 0; r < K; ++r) {
      const int e = r * 32 + lane;
      int32_t prev = __shfl_up_sync(PR_FULL, x[r], 1);
      const int32_t last_prev = __shfl_sync(PR_FULL, x[r > 0 ? r - 1 : 0], 31);
      if (lane == 0) prev = last_prev;
      int32_t next = __shfl_down_sync(PR_FULL, x[r], 1);
      const int32_t first_next = __shfl_sync(PR_FULL, x[r + 1 < K ? r + 1 : r], 0);
      if (lane == 31) next = first_next;
      const bool head = e < L && (e == 0 || x[r] != prev);
      const bool tail = e < L && (e == L - 1 || x[r] != next);
      const unsigned hb = __ballot_sync(PR_FULL, head);
      const int run = runs + __popc(hb & lt) + (head ? 1 : 0) - 1;  // run index of element e
      if (tail) {
        oc[run] = x[r];
        on[run] = e - hrow[run] + 1;
      }
      runs += __popc(hb);
    }
    if (lane == 0) nnz[gp] = base;
    __syncwarp();
  }
}

// Copy each row's unique pairs from the stage to its CSR position (warp per row).
__global__ void k_compact_rows(const int32_t* __restrict__ st_col, const int32_t* __restrict__ st_cnt,
                               const int32_t* __restrict__ nnz, const int64_t* __restrict__ off, int64_t np,
                               int L, int64_t out_base, int32_t* __restrict__ col, int32_t* __restrict__ cnt) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t p = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); p < np; p += warps) {
    const int m = nnz[p];
    const int64_t dst = out_base + off[p];
    for (int e = lane; e < m; e += 32) {
      col[dst + e] = st_col[p * L + e];
      cnt[dst + e] = st_cnt[p * L + e];
    }
  }
}

// One chunk's rows in the layout first_hit_counts hands back (view_factors.py:273-287): the
// origin patch id of every pair, its receiver and its count widened to int64, at the chunk's
// exclusive row offsets (one warp per row).
__global__ void k_compact_host(const int32_t* __restrict__ st_col, const int32_t* __restrict__ st_cnt,
                               const int32_t* __restrict__ nnz, const int64_t* __restrict__ off, int64_t np,
                               int L, int64_t first_id, int32_t* __restrict__ origin, int32_t* __restrict__ col,
                               int64_t* __restrict__ cnt) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t p = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); p < np; p += warps) {
    const int m = nnz[p];
    const int64_t dst = off[p];
    for (int e = lane; e < m; e += 32) {
      origin[dst + e] = (int32_t)(first_id + p);
      col[dst + e] = st_col[p * L + e];
      cnt[dst + e] = st_cnt[p * L + e];
    }
  }
}

__global__ void k_i32_to_i64(const int32_t* __restrict__ in, int64_t* __restrict__ out, int64_t n) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
    out[t] = in[t];
}

__global__ void k_fill_i64(int64_t* __restrict__ out, int64_t n, int64_t v) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
    out[t] = v;
}

// ---------------------------------------------------------------------------- host

static void host_u128_mul(const pr_u128& a, const pr_u128& b, pr_u128& r) {
  unsigned __int128 x = ((unsigned __int128)a.hi << 64) | a.lo;
  unsigned __int128 y = ((unsigned __int128)b.hi << 64) | b.lo;
  unsigned __int128 z = x * y;
  r.lo = (uint64_t)z;
  r.hi = (uint64_t)(z >> 64);
}
static pr_u128 host_u128_add(const pr_u128& a, const pr_u128& b) {
  unsigned __int128 x = ((unsigned __int128)a.hi << 64) | a.lo;
  unsigned __int128 y = ((unsigned __int128)b.hi << 64) | b.lo;
  unsigned __int128 z = x + y;
  return pr_u128{(uint64_t)z, (uint64_t)(z >> 64)};
}

static pr_u128 host_affine(const pr_u128& A, const pr_u128& C, const pr_u128& x) {
  pr_u128 m;
  host_u128_mul(A, x, m);
  return host_u128_add(m, C);
}

// Seed tables on the device: kMapStride maps per seed, states (S), increments (S).
struct SeedTables {
  DevBuf<pr_u128> maps, state, inc;
  int build(const pr_pcg64* seeds, int S, cudaStream_t s) {
    std::vector<pr_u128> h_maps((size_t)S * kMapStride), h_state(S), h_inc(S);
    for (int q = 0; q < S; ++q) {
      pr_pcg64 sd;
      memcpy(&sd, seeds + q, sizeof(sd));  // seeds may be host memory only
      h_state[q] = pr_u128{sd.state_lo, sd.state_hi};
      h_inc[q] = pr_u128{sd.inc_lo, sd.inc_hi};
      pr_u128* m = h_maps.data() + (size_t)q * kMapStride;
      const pr_u128 A1{PR_PCG_MULT_LO, PR_PCG_MULT_HI}, C1 = h_inc[q];
      pr_u128 A = A1, C = C1;
      for (int i = 0; i < 64; ++i) {
        m[2 * i] = A;
        m[2 * i + 1] = C;
        // (A, C) o (A, C) = (A A, A C + C)
        pr_u128 AA, AC;
        host_u128_mul(A, A, AA);
        host_u128_mul(A, C, AC);
        C = host_u128_add(AC, C);
        A = AA;
      }
      // maps of n = 4 l steps by repeated composition with the one-step map
      pr_u128 An{1, 0}, Cn{0, 0};
      for (int n = 0; n <= 128; ++n) {
        if (n % 4 == 0 && n / 4 < 32) {
          m[kMapSmall + 2 * (n / 4)] = An;
          m[kMapSmall + 2 * (n / 4) + 1] = Cn;
        }
        if (n == 128) {
          m[kMapBatch] = An;
          m[kMapBatch + 1] = Cn;
        }
        // (A1, C1) o (An, Cn) = (A1 An, A1 Cn + C1)
        pr_u128 t;
        host_u128_mul(A1, An, t);
        Cn = host_affine(A1, C1, Cn);
        An = t;
      }
    }
    PR_TRY(maps.alloc(h_maps.size(), s));
    PR_TRY(state.alloc(S, s));
    PR_TRY(inc.alloc(S, s));
    PR_CUDA(cudaMemcpyAsync(maps.ptr, h_maps.data(), h_maps.size() * sizeof(pr_u128), cudaMemcpyHostToDevice, s));
    PR_CUDA(cudaMemcpyAsync(state.ptr, h_state.data(), S * sizeof(pr_u128), cudaMemcpyHostToDevice, s));
    PR_CUDA(cudaMemcpyAsync(inc.ptr, h_inc.data(), S * sizeof(pr_u128), cudaMemcpyHostToDevice, s));
    // the host vectors die at return: make the copies complete first
    PR_CUDA(cudaStreamSynchronize(s));
    return PR_OK;
  }
};

static Geom geom_of(const pr_case* c) {
  Geom g;
  g.occ = c->occ.ptr;
  g.cfp = c->cfp();
  g.hot = c->hot();
  g.cold = c->cold();
  g.nx = (int32_t)c->nx;
  g.ny = (int32_t)c->ny;
  g.nz = (int32_t)c->nz;
  g.n_cells = c->n_cells;
  return g;
}

static RaySrc src_of(const pr_case* c, const SeedTables& t) {
  RaySrc r;
  r.origin = c->origin.ptr;
  r.code = c->code.ptr;
  r.maps = t.maps.ptr;
  r.state = t.state.ptr;
  r.inc = t.inc.ptr;
  r.ny_d = (double)c->ny;
  r.nz_d = (double)c->nz;
  return r;
}

static int trace_grid() { return sm_count() * 8; }

// Variants of the pooled traversal: minimum resident blocks per SM (the register budget),
// rounds between lane refills, and cells of occupancy lookahead per round (lookN: N
// occupancy loads in flight per lane; burst: one cell per round).  Every variant writes the
// same receivers; the autotuner below picks the fastest per problem class by timing them
// on the first wave of the first call.
using TraceKernel = void (*)(const WaveChunk*, int, int64_t, int32_t*, unsigned long long*, unsigned long long*);
struct TraceVariant {
  TraceKernel kernel;
  const char* name;
};
static const TraceVariant kVariants[] = {
    {k_trace_pool<6, 4, 2>, "6blk-look2x4"},
    {k_trace_pool<6, 2, 3>, "6blk-look3x2"},
    {k_trace_pool<6, 2, 4>, "6blk-look4x2"},
    {k_trace_pool<6, 6, 2>, "6blk-look2x6"},
    {k_trace_pool<5, 4, 3>, "5blk-look3x4"},
    {k_trace_pool<7, 4, 2>, "7blk-look2x4"},
    {k_trace_pool<4, 4, 2>, "4blk-look2x4"},
    {k_trace_pool<5, 8, 0>, "5blk-burst8"},
    {k_trace_pool<6, 4, 0>, "6blk-burst4"},
    {k_trace_pool<7, 2, 3>, "7blk-look3x2"},
    {k_trace_pool<6, 2, 5>, "6blk-look5x2"},
    {k_trace_pool<7, 2, 4>, "7blk-look4x2"},
};
static constexpr int kNumVariants = (int)(sizeof(kVariants) / sizeof(kVariants[0]));

// Persistent grid of a variant: as many blocks as fit on every SM.
static int variant_grid(int v) {
  static int blocks[kNumVariants] = {0};
  if (blocks[v] == 0) {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kVariants[v].kernel, kWarps * 32, 0);
    blocks[v] = sm_count() * (per_sm > 0 ? per_sm : 1);
  }
  return blocks[v];
}

struct TuneKey {
  int64_t nx, ny, nz, L, cases;
  bool operator<(const TuneKey& o) const {
    return std::tie(nx, ny, nz, L, cases) < std::tie(o.nx, o.ny, o.nz, o.L, o.cases);
  }
};
static std::mutex g_tune_mu;
static std::map<TuneKey, int> g_tuned;
static int g_forced_variant = -1;
static int g_last_variant = 0;

}  // namespace pr

extern "C" {
// Force one traversal variant (0 .. count - 1), or -1 for the autotuner (default).
PR_API int pr_trace_set_variant(int v) {
  if (v < -1 || v >= pr::kNumVariants) {
    pr::set_error("traversal variant %d outside [-1, %d)", v, pr::kNumVariants);
    return PR_ERR_ARG;
  }
  std::lock_guard<std::mutex> lk(pr::g_tune_mu);
  pr::g_forced_variant = v;
  return PR_OK;
}
// Number of variants, the variant used by the last count pass, and its name (may be NULL).
PR_API int pr_trace_variant_info(int* count, int* last, const char** name) {
  std::lock_guard<std::mutex> lk(pr::g_tune_mu);
  if (count) *count = pr::kNumVariants;
  if (last) *last = pr::g_last_variant;
  if (name) *name = pr::kVariants[pr::g_last_variant].name;
  return PR_OK;
}
}

namespace pr {

struct WaveLaunch {
  const WaveChunk* chunks;  // device table
  int n_chunks;
  int64_t total;            // global ray indices [0, total)
  int32_t* recv;            // hit codes, by global ray index
  unsigned long long* work; // work-unit counter
  unsigned long long* ctr;  // 2 per chunk: DDA steps, failed rays
};

static int launch_variant(int v, const WaveLaunch& w, cudaStream_t s) {
  PR_CUDA(cudaMemsetAsync(w.work, 0, sizeof(unsigned long long), s));
  ::pr::launch_mark(), kVariants[v].kernel<<<variant_grid(v), kWarps * 32, 0, s>>>(w.chunks, w.n_chunks, w.total,
                                                                                  w.recv, w.work, w.ctr);
  PR_CUDA(cudaGetLastError());
  return PR_OK;
}

// Variant for this problem class: forced, cached, or measured now on the given wave (each
// variant traces it once, timed with events; the per-chunk counters are cleared after).
static int choose_variant(const TuneKey& key, const WaveLaunch& w, cudaStream_t s, int* out) {
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    if (g_forced_variant >= 0) {
      *out = g_forced_variant;
      return PR_OK;
    }
    auto it = g_tuned.find(key);
    if (it != g_tuned.end()) {
      *out = it->second;
      return PR_OK;
    }
  }
  cudaEvent_t e0, e1;
  PR_CUDA(cudaEventCreate(&e0));
  PR_CUDA(cudaEventCreate(&e1));
  float best = 1e30f;
  int best_v = 0;
  for (int v = 0; v < kNumVariants; ++v) {
    PR_CUDA(cudaEventRecord(e0, s));
    PR_TRY(launch_variant(v, w, s));
    PR_CUDA(cudaEventRecord(e1, s));
    PR_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    PR_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    if (ms < best) {
      best = ms;
      best_v = v;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  PR_CUDA(cudaMemsetAsync(w.ctr, 0, 2 * sizeof(unsigned long long) * w.n_chunks, s));
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tuned[key] = best_v;
  }
  *out = best_v;
  return PR_OK;
}

int generate_rays(const pr_case* c, int64_t p0, int64_t p1, int64_t R, const pr_pcg64* seed, double* origins,
                  double* dirs, cudaStream_t s) {
  PR_ARG(p0 >= 0 && p1 >= p0 && p1 <= c->n_patches, "patch range [%lld, %lld) outside [0, %lld)",
         (long long)p0, (long long)p1, (long long)c->n_patches);
  PR_ARG(R >= 0, "rays_per_patch must be non-negative");
  const int64_t n = (p1 - p0) * R;
  if (n == 0) return PR_OK;
  SeedTables t;
  PR_TRY(t.build(seed, 1, s));
  DevBuf<double> o, d;
  PR_TRY(o.alloc(3 * n, s));
  PR_TRY(d.alloc(3 * n, s));
  ::pr::launch_mark(), k_generate<<<grid_for(n, 256, trace_grid()), 256, 0, s>>>(src_of(c, t), p0, p1 - p0, R, o.ptr, d.ptr);
  PR_CUDA(cudaGetLastError());
  PR_CUDA(cudaMemcpyAsync(origins, o.ptr, o.bytes(), cudaMemcpyDefault, s));
  PR_CUDA(cudaMemcpyAsync(dirs, d.ptr, d.bytes(), cudaMemcpyDefault, s));
  PR_CUDA(cudaStreamSynchronize(s));
  return PR_OK;
}

int trace_given(const pr_case* c, const double* origins, const double* dirs, int64_t n, int32_t* receiver,
                int64_t* n_failed, cudaStream_t s) {
  if (n_failed) *n_failed = 0;
  if (n == 0) return PR_OK;
  DevBuf<double> o, d;
  DevBuf<int32_t> rv;
  DevBuf<unsigned long long> ctr;
  PR_TRY(o.alloc(3 * n, s));
  PR_TRY(d.alloc(3 * n, s));
  PR_TRY(rv.alloc(n, s));
  PR_TRY(ctr.alloc(2, s));
  PR_CUDA(cudaMemcpyAsync(o.ptr, origins, o.bytes(), cudaMemcpyDefault, s));
  PR_CUDA(cudaMemcpyAsync(d.ptr, dirs, d.bytes(), cudaMemcpyDefault, s));
  PR_CUDA(cudaMemsetAsync(ctr.ptr, 0, ctr.bytes(), s));
  ::pr::launch_mark(), k_trace_given<<<grid_for(n, 256, trace_grid()), 256, 0, s>>>(geom_of(c), o.ptr, d.ptr, n, rv.ptr, ctr.ptr);
  PR_CUDA(cudaGetLastError());
  unsigned long long h[2];
  PR_CUDA(cudaMemcpyAsync(receiver, rv.ptr, rv.bytes(), cudaMemcpyDefault, s));
  PR_CUDA(cudaMemcpyAsync(h, ctr.ptr, sizeof(h), cudaMemcpyDeviceToHost, s));
  PR_CUDA(cudaStreamSynchronize(s));
  if (n_failed) *n_failed = (int64_t)h[1];
  if (h[1]) {
    set_error("%lld rays did not resolve a receiving patch", (long long)h[1]);
    return PR_ERR_UNRESOLVED;
  }
  return PR_OK;
}

// Largest rays-per-origin segment the shared-memory sort handles (128 KiB of keys + heads).
static const int kMaxSegment = 16384;

// The per-patch sort's dynamic shared-memory limit is a per-device function attribute shared
// by every host thread: raise it once per device to the largest segment and never lower it.
static int enable_rle_smem() {
  static std::mutex mu;
  static bool done[64] = {false};
  int dev = 0;
  PR_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  if (dev >= 0 && dev < 64 && done[dev]) return PR_OK;
  PR_CUDA(cudaFuncSetAttribute(k_patch_rle, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)(2 * kMaxSegment * sizeof(int32_t))));
  if (dev >= 0 && dev < 64) done[dev] = true;
  return PR_OK;
}

// Rays of one launch (a wave): chunks of one or more cases are packed until this bound.
static const int64_t kWaveRays = (int64_t)1 << 27;
// Patches per chunk: a chunk holds at most 2^26 rays.
static const int64_t kChunkRays = (int64_t)1 << 26;

// Per-case accumulation of a batched count pass.
struct CaseCounts {
  std::unique_ptr<pr_counts> k;
  DevBuf<int64_t> nnz_all;  // row lengths
  struct Piece {
    DevBuf<int32_t> col, cnt;
    int64_t n = 0;
  };
  std::vector<Piece> pieces;  // compacted chunks in patch order
};

// A count pass of one case that hands its edge list to host memory while it runs: each
// chunk's rows, once compacted, are laid out as first_hit_counts returns them and copied on a
// stream of their own into origin / receiver / count at their place in the sorted list, while
// the next chunks trace; no device table is kept.
struct HostSink {
  int32_t* origin;
  int32_t* receiver;
  int64_t* count;
  int64_t capacity;  // pairs the arrays hold
  int64_t written = 0;
};

namespace {
// The copy stream of a host pass and what its copies read, released in this order: the stream
// is drained before the device buffers go back to the cache.
struct HostPass {
  struct Piece {
    DevBuf<int32_t> o, r;
    DevBuf<int64_t> c;
  };
  std::vector<Piece> pieces;
  std::vector<cudaEvent_t> events;
  cudaStream_t copy = nullptr;
  ~HostPass() {
    if (copy) {
      cudaStreamSynchronize(copy);
      cudaStreamDestroy(copy);
    }
    for (cudaEvent_t e : events) cudaEventDestroy(e);
    pieces.clear();
  }
};
}  // namespace

// first_hit_counts for n_cases geometries at once (view_factors.py:273-300 per case): every
// case traces rays_per_patch rays per patch for each of its S seeds (seeds[c * S + s]);
// chunks of all cases share persistent launches of the pooled traversal.  With `sink` (one
// case), the edge list goes to host memory as the chunks finish and `out` is not used.
int counts_batch(const pr_case* const* cases, int nc, int64_t R, const pr_pcg64* seeds, int S, cudaStream_t s,
                 pr_counts** out, HostSink* sink) {
  PR_ARG(nc > 0, "no cases");
  PR_ARG(!sink || nc == 1, "a host pass takes one case");
  PR_ARG(R > 0 && S > 0, "rays_per_patch and the number of seeds must be positive");
  const int64_t L64 = R * S;
  if (L64 > kMaxSegment) {
    set_error("%lld rays per origin patch exceed the %d supported in one call", (long long)L64, kMaxSegment);
    return PR_ERR_LIMIT;
  }
  const int L = (int)L64;
  int Lpad = 1;
  while (Lpad < L) Lpad <<= 1;
  if (Lpad < 64) Lpad = 64;
  int dev0 = 0;
  cudaGetDevice(&dev0);

  // seed tables and per-case outputs
  std::vector<SeedTables> tables(nc);
  std::vector<CaseCounts> cc(nc);
  for (int c = 0; c < nc; ++c) {
    PR_ARG(cases[c] != nullptr, "case %d is NULL", c);
    PR_ARG(cases[c]->device == dev0, "case %d lives on another device", c);
    // int32 hit codes (and cell indices)
    if (6 * cases[c]->n_cells + 2 * cases[c]->ny * cases[c]->nz > (int64_t)INT32_MAX) {
      set_error("case %d: %lld cells exceed the int32 hit codes of the traversal", c, (long long)cases[c]->n_cells);
      return PR_ERR_LIMIT;
    }
    PR_TRY(tables[c].build(seeds + (size_t)c * S, S, s));
    const int64_t P = cases[c]->n_patches;
    cc[c].k.reset(new pr_counts());
    cc[c].k->device = dev0;
    cc[c].k->csr = std::make_shared<CountCsr>();
    cc[c].k->csr->n_rows = P;
    PR_TRY(cc[c].k->csr->row_ptr.alloc(P + 1, s));
    PR_TRY(cc[c].k->rays.alloc(P > 0 ? P : 1, s));
    PR_TRY(cc[c].nnz_all.alloc(P > 0 ? P : 1, s));
    if (P > 0) {
      ::pr::launch_mark(), k_fill_i64<<<grid_for(P, 256), 256, 0, s>>>(cc[c].k->rays.ptr, P, L64);
      PR_CUDA(cudaGetLastError());
    }
  }

  // chunks: (case, first patch, patches)
  struct Chunk {
    int c;
    int64_t p0, np;
  };
  std::vector<Chunk> chunks;
  const int64_t chunk_patches = std::max<int64_t>(1, kChunkRays / L64);
  for (int c = 0; c < nc; ++c)
    for (int64_t p0 = 0; p0 < cases[c]->n_patches; p0 += chunk_patches)
      chunks.push_back({c, p0, std::min(chunk_patches, cases[c]->n_patches - p0)});

  // wave buffers
  int64_t wave_cap = 0;
  for (const Chunk& ch : chunks) wave_cap = std::max(wave_cap, ch.np * L64);
  wave_cap = std::max(wave_cap, std::min<int64_t>(kWaveRays, [&] {
                        int64_t t = 0;
                        for (const Chunk& ch : chunks) t += ch.np * L64;
                        return t;
                      }()));
  if (sink) {
    // one chunk per wave, so that every chunk's copy overlaps the next chunk's traversal
    wave_cap = 0;
    for (const Chunk& ch : chunks) wave_cap = std::max(wave_cap, ch.np * L64);
  }
  HostPass hp;
  if (sink) PR_CUDA(cudaStreamCreateWithFlags(&hp.copy, cudaStreamNonBlocking));
  DevBuf<int32_t> recv, st_col, st_cnt, nnz;
  DevBuf<int64_t> off;
  DevBuf<unsigned long long> work, ctr;
  DevBuf<WaveChunk> dchunks;
  DevBuf<RleChunk> drle;
  const int64_t max_wave_patches = wave_cap / L64 + (int64_t)chunks.size();
  // hit codes by wave-wide ray index: chunk starts are rounded up to whole work units
  PR_TRY(recv.alloc(wave_cap + (int64_t)chunks.size() * kUnit, s));
  PR_TRY(st_col.alloc(wave_cap, s));
  PR_TRY(st_cnt.alloc(wave_cap, s));
  PR_TRY(nnz.alloc(max_wave_patches, s));
  PR_TRY(off.alloc(max_wave_patches + 1, s));
  PR_TRY(work.alloc(1, s));
  PR_TRY(ctr.alloc(2 * chunks.size(), s));
  PR_TRY(dchunks.alloc(chunks.size(), s));
  PR_TRY(drle.alloc(chunks.size(), s));
  PR_CUDA(cudaMemsetAsync(ctr.ptr, 0, ctr.bytes(), s));
  PR_TRY(enable_rle_smem());
  const size_t smem = (size_t)2 * Lpad * sizeof(int32_t);
  const int rle_threads = Lpad >= 1024 ? 512 : (Lpad >= 256 ? 256 : 64);
  size_t scan_bytes = 0;
  PR_CUDA(cub::DeviceScan::InclusiveSum(nullptr, scan_bytes, off.ptr, off.ptr + 1, max_wave_patches, s));
  DevBuf<uint8_t> scan_tmp;
  PR_TRY(scan_tmp.alloc(scan_bytes + 16, s));

  int variant = 0;
  bool tuned = false;
  std::vector<WaveChunk> hw;
  std::vector<RleChunk> hr;
  std::vector<int64_t> totals;
  for (size_t w0 = 0; w0 < chunks.size();) {
    // pack a wave
    size_t w1 = w0;
    int64_t rays = 0;
    while (w1 < chunks.size() && (w1 == w0 || rays + chunks[w1].np * L64 <= wave_cap)) rays += chunks[w1++].np * L64;
    const int nw = (int)(w1 - w0);
    hw.assign(nw, WaveChunk{});
    hr.assign(nw, RleChunk{});
    int64_t start = 0, ray0 = 0, patch0 = 0;
    for (int k = 0; k < nw; ++k) {
      const Chunk& ch = chunks[w0 + k];
      const pr_case* c = cases[ch.c];
      WaveChunk& W = hw[k];
      W.occ = c->occ.ptr;
      W.origin = c->origin.ptr;
      W.code = c->code.ptr;
      W.maps = tables[ch.c].maps.ptr;
      W.state = tables[ch.c].state.ptr;
      W.inc = tables[ch.c].inc.ptr;
      W.n = ch.np * L64;
      W.np = ch.np;
      W.p0 = ch.p0;
      W.R = R;
      W.start = start;
      W.n_cells = c->n_cells;
      W.nx = (int32_t)c->nx;
      W.ny = (int32_t)c->ny;
      W.nz = (int32_t)c->nz;
      W.ny_d = (double)c->ny;
      W.nz_d = (double)c->nz;
      hr[k] = RleChunk{recv.ptr + start, c->ftab.ptr, ctr.ptr + 2 * (w0 + k) + 1, ch.np, patch0, ray0};
      start += (W.n + kUnit - 1) / kUnit * kUnit;
      ray0 += W.n;
      patch0 += ch.np;
    }
    const int64_t total = hw[nw - 1].start + hw[nw - 1].n;
    PR_CUDA(cudaMemcpyAsync(dchunks.ptr, hw.data(), nw * sizeof(WaveChunk), cudaMemcpyHostToDevice, s));
    PR_CUDA(cudaMemcpyAsync(drle.ptr, hr.data(), nw * sizeof(RleChunk), cudaMemcpyHostToDevice, s));
    unsigned long long* wave_ctr = ctr.ptr + 2 * w0;
    WaveLaunch wl{dchunks.ptr, nw, total, recv.ptr, work.ptr, wave_ctr};
    if (!tuned) {
      const pr_case* c0 = cases[chunks[w0].c];
      PR_TRY(choose_variant(TuneKey{c0->nx, c0->ny, c0->nz, L64, nc}, wl, s, &variant));
      tuned = true;
    }
    ::pr::timer_begin(kTimerTrace, s);
    PR_TRY(launch_variant(variant, wl, s));
    ::pr::timer_end(kTimerTrace, s);
    const int rle_grid = (int)std::min<int64_t>(patch0, (int64_t)sm_count() * 16);
    ::pr::timer_begin(kTimerRle, s);
    if (Lpad <= 1024) {
      const int wg = (int)std::min<int64_t>((patch0 + 3) / 4, (int64_t)sm_count() * 32);
      auto kern = Lpad <= 64 ? k_patch_rle_warp<2> : Lpad <= 128 ? k_patch_rle_warp<4>
                : Lpad <= 256 ? k_patch_rle_warp<8> : Lpad <= 512 ? k_patch_rle_warp<16> : k_patch_rle_warp<32>;
      ::pr::launch_mark(), kern<<<wg, 128, 0, s>>>(drle.ptr, nw, patch0, L, (int)R, st_col.ptr, st_cnt.ptr, nnz.ptr);
    } else
    ::pr::launch_mark(), k_patch_rle<<<rle_grid, rle_threads, smem, s>>>(drle.ptr, nw, patch0, L, (int)R, Lpad,
                                                                     st_col.ptr, st_cnt.ptr, nnz.ptr);
    ::pr::timer_end(kTimerRle, s);
    PR_CUDA(cudaGetLastError());
    // per chunk: row lengths into the case, exclusive offsets for the compaction
    totals.assign(nw, 0);
    for (int k = 0; k < nw; ++k) {
      const Chunk& ch = chunks[w0 + k];
      const RleChunk& rc = hr[k];
      ::pr::launch_mark(), k_i32_to_i64<<<grid_for(ch.np, 256), 256, 0, s>>>(nnz.ptr + rc.patch0,
                                                                            cc[ch.c].nnz_all.ptr + ch.p0, ch.np);
      PR_CUDA(cudaGetLastError());
      int64_t* o = off.ptr + rc.patch0 + k;  // np + 1 slots per chunk
      PR_CUDA(cudaMemsetAsync(o, 0, sizeof(int64_t), s));
      PR_CUDA(cub::DeviceScan::InclusiveSum(scan_tmp.ptr, scan_bytes, cc[ch.c].nnz_all.ptr + ch.p0, o + 1, ch.np, s));
      PR_CUDA(cudaMemcpyAsync(&totals[k], o + ch.np, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    }
    PR_CUDA(cudaStreamSynchronize(s));
    for (int k = 0; k < nw && sink; ++k) {
      const Chunk& ch = chunks[w0 + k];
      const RleChunk& rc = hr[k];
      const int64_t n = totals[k];
      if (sink->written + n > sink->capacity) {
        set_error("the edge list exceeds the %lld pairs the host arrays hold", (long long)sink->capacity);
        return PR_ERR_LIMIT;
      }
      HostPass::Piece pc;
      PR_TRY(pc.o.alloc(n > 0 ? n : 1, s));
      PR_TRY(pc.r.alloc(n > 0 ? n : 1, s));
      PR_TRY(pc.c.alloc(n > 0 ? n : 1, s));
      ::pr::launch_mark(), k_compact_host<<<grid_for(ch.np * 32, 256), 256, 0, s>>>(
          st_col.ptr + rc.ray0, st_cnt.ptr + rc.ray0, nnz.ptr + rc.patch0, off.ptr + rc.patch0 + k, ch.np, L, ch.p0,
          pc.o.ptr, pc.r.ptr, pc.c.ptr);
      PR_CUDA(cudaGetLastError());
      cudaEvent_t ev = nullptr;
      PR_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
      hp.events.push_back(ev);
      PR_CUDA(cudaEventRecord(ev, s));
      PR_CUDA(cudaStreamWaitEvent(hp.copy, ev, 0));
      if (n > 0) {
        const int64_t at = sink->written;
        PR_CUDA(cudaMemcpyAsync(sink->origin + at, pc.o.ptr, (size_t)n * 4, cudaMemcpyDeviceToHost, hp.copy));
        PR_CUDA(cudaMemcpyAsync(sink->receiver + at, pc.r.ptr, (size_t)n * 4, cudaMemcpyDeviceToHost, hp.copy));
        PR_CUDA(cudaMemcpyAsync(sink->count + at, pc.c.ptr, (size_t)n * 8, cudaMemcpyDeviceToHost, hp.copy));
      }
      sink->written += n;
      hp.pieces.push_back(std::move(pc));
    }
    for (int k = 0; k < nw && !sink; ++k) {
      const Chunk& ch = chunks[w0 + k];
      const RleChunk& rc = hr[k];
      CaseCounts::Piece pc;
      pc.n = totals[k];
      PR_TRY(pc.col.alloc(pc.n > 0 ? pc.n : 1, s));
      PR_TRY(pc.cnt.alloc(pc.n > 0 ? pc.n : 1, s));
      ::pr::launch_mark(), k_compact_rows<<<grid_for(ch.np * 32, 256), 256, 0, s>>>(
          st_col.ptr + rc.ray0, st_cnt.ptr + rc.ray0, nnz.ptr + rc.patch0, off.ptr + rc.patch0 + k, ch.np, L, 0,
          pc.col.ptr, pc.cnt.ptr);
      PR_CUDA(cudaGetLastError());
      cc[ch.c].pieces.push_back(std::move(pc));
    }
    // the next wave's kernels reuse the stage buffers after these compactions in stream order
    w0 = w1;
  }

  // per case: concatenate the pieces, row offsets, counters
  std::vector<unsigned long long> hctr(2 * chunks.size());
  PR_CUDA(cudaMemcpyAsync(hctr.data(), ctr.ptr, ctr.bytes(), cudaMemcpyDeviceToHost, s));
  PR_CUDA(cudaStreamSynchronize(s));
  int64_t failed = 0;
  std::vector<int64_t> steps(nc, 0), fails(nc, 0);
  for (size_t k = 0; k < chunks.size(); ++k) {
    steps[chunks[k].c] += (int64_t)hctr[2 * k];
    fails[chunks[k].c] += (int64_t)hctr[2 * k + 1];
  }
  if (sink) {
    PR_CUDA(cudaStreamSynchronize(hp.copy));
    {
      std::lock_guard<std::mutex> lk(g_tune_mu);
      g_last_variant = variant;
    }
    if (fails[0]) {
      set_error("%lld rays did not resolve a receiving patch", (long long)fails[0]);
      return PR_ERR_UNRESOLVED;
    }
    return PR_OK;
  }
  for (int c = 0; c < nc; ++c) {
    CountCsr& csr = *cc[c].k->csr;
    const int64_t P = csr.n_rows;
    int64_t total = 0;
    for (auto& pc : cc[c].pieces) total += pc.n;
    csr.nnz = total;
    PR_TRY(csr.col.alloc(total > 0 ? total : 1, s));
    PR_TRY(csr.cnt.alloc(total > 0 ? total : 1, s));
    int64_t at = 0;
    for (auto& pc : cc[c].pieces) {
      if (pc.n) {
        PR_CUDA(cudaMemcpyAsync(csr.col.ptr + at, pc.col.ptr, pc.n * 4, cudaMemcpyDeviceToDevice, s));
        PR_CUDA(cudaMemcpyAsync(csr.cnt.ptr + at, pc.cnt.ptr, pc.n * 4, cudaMemcpyDeviceToDevice, s));
      }
      at += pc.n;
    }
    cc[c].pieces.clear();
    PR_CUDA(cudaMemsetAsync(csr.row_ptr.ptr, 0, sizeof(int64_t), s));
    if (P > 0) {
      size_t b = 0;
      PR_CUDA(cub::DeviceScan::InclusiveSum(nullptr, b, cc[c].nnz_all.ptr, csr.row_ptr.ptr + 1, P, s));
      DevBuf<uint8_t> tmp;
      PR_TRY(tmp.alloc(b + 16, s));
      PR_CUDA(cub::DeviceScan::InclusiveSum(tmp.ptr, b, cc[c].nnz_all.ptr, csr.row_ptr.ptr + 1, P, s));
    }
    cc[c].k->rays_traced = P * L64;
    cc[c].k->dda_steps = steps[c];
    cc[c].k->last_stream = s;
    failed += fails[c];
  }
  PR_CUDA(cudaStreamSynchronize(s));
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_last_variant = variant;
  }
  if (failed) {
    set_error("%lld rays did not resolve a receiving patch", (long long)failed);
    return PR_ERR_UNRESOLVED;
  }
  for (int c = 0; c < nc; ++c) out[c] = cc[c].k.release();
  return PR_OK;
}

int first_hit_counts(const pr_case* c, int64_t R, const pr_pcg64* seeds, int S, cudaStream_t s, pr_counts** out) {
  return counts_batch(&c, 1, R, seeds, S, s, out, nullptr);
}

int first_hit_counts_host(const pr_case* c, int64_t R, const pr_pcg64* seeds, int S, cudaStream_t s,
                          int32_t* origin, int32_t* receiver, int64_t* count, int64_t capacity, int64_t* n_pairs) {
  HostSink sink{origin, receiver, count, capacity, 0};
  *n_pairs = 0;
  PR_TRY(counts_batch(&c, 1, R, seeds, S, s, nullptr, &sink));
  *n_pairs = sink.written;
  return PR_OK;
}

}  // namespace pr
