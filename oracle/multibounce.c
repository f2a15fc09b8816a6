/* ORACLE — test infrastructure only.
 *
 * CPU restatement of porerad's multi-bounce ray kernels (porerad/properties.py and
 * porerad/penetration.py, written there for Taichi), the CPU leg of bench.py's properties
 * workload and a statistical checker of the device kernels.  One ray per loop iteration
 * under OpenMP, like the reference's parallel Taichi loop:
 *   - the 32-bit hash generator: state = h(seed + (ray + 1) * 747796405), then
 *     state = h(state + 0x9E3779B9) per draw, uniform = (state & 0xFFFFFF) / 2^24
 *     (properties.py:83-96);
 *   - the cell traversal: start cell floor(o), stepped back on an axis where the direction
 *     is negative and o lies within 1e-12 of a face (floor(o + 0.5)); periodic y and z; exits
 *     through x = 0 and x = N; ties within 1e-12 advance every crossed axis; the normal is the
 *     last face crossed, x over y over z; step cap 10 N^3 + 10 (properties.py:98-197);
 *   - Lambertian reflection about the normal with a helper axis, radius sqrt(xi1), azimuth
 *     2 pi xi2 (glibc sin and cos here), elevation sqrt(1 - xi1) (properties.py:200-226);
 *   - restart rules "article" (from the segment start advanced by the incoming distance) and
 *     "hit_point" (from the hit point), both offset 1e-9 along the normal (properties.py:14-22).
 * Tallies: properties (events, sum of event lengths, censored, sum of censored lengths,
 * interactions, scattered, sum of mu, sum of mu^2); penetration (reflected, transmitted,
 * absorbed, stopped at a cap).  Built with -ffp-contract=off. */
#include <math.h>
#include <stdint.h>

static uint32_t mb_hash(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7FEB352Du;
  x ^= x >> 15;
  x *= 0x846CA68Bu;
  x ^= x >> 16;
  return x;
}

static double mb_rand(uint32_t* s) {
  *s = mb_hash(*s + 0x9E3779B9u);
  return (double)(*s & 0x00FFFFFFu) / (double)0x01000000u;
}

static int pymod(int a, int m) {
  const int r = a % m;
  return r < 0 ? r + m : r;
}

typedef struct {
  int fate; /* 0 solid, 1 exit x = 0, 2 exit x = N, 3 step cap */
  double t, nx, ny, nz;
} hit_t;

static hit_t trace(const uint8_t* solid, int sx, int sy, int sz, double ox, double oy, double oz, double dx0,
                   double dy0, double dz0) {
  const double norm = sqrt(dx0 * dx0 + dy0 * dy0 + dz0 * dz0);
  const double dx = dx0 / norm, dy = dy0 / norm, dz = dz0 / norm;
  int i = (int)floor(ox), j = (int)floor(oy), k = (int)floor(oz);
  if (dx < 0.0 && fabs(ox - floor(ox + 0.5)) <= 1.0e-12) i -= 1;
  if (dy < 0.0 && fabs(oy - floor(oy + 0.5)) <= 1.0e-12) j -= 1;
  if (dz < 0.0 && fabs(oz - floor(oz + 0.5)) <= 1.0e-12) k -= 1;
  int st[3] = {0, 0, 0};
  double tm[3] = {1e300, 1e300, 1e300}, td[3] = {1e300, 1e300, 1e300};
  const double d[3] = {dx, dy, dz}, o[3] = {ox, oy, oz};
  const int c[3] = {i, j, k};
  for (int a = 0; a < 3; ++a) {
    if (d[a] > 0.0) {
      st[a] = 1;
      tm[a] = ((double)(c[a] + 1) - o[a]) / d[a];
      td[a] = 1.0 / d[a];
    } else if (d[a] < 0.0) {
      st[a] = -1;
      tm[a] = ((double)c[a] - o[a]) / d[a];
      td[a] = -1.0 / d[a];
    }
  }
  hit_t h = {-1, 0.0, 0.0, 0.0, 0.0};
  const long long cap = 10LL * sx * sy * sz + 10;
  for (long long steps = 0; h.fate == -1 && steps < cap;) {
    ++steps;
    if (i < 0) {
      h.fate = 1;
    } else if (i >= sx) {
      h.fate = 2;
    } else if (solid[((long long)i * sy + pymod(j, sy)) * sz + pymod(k, sz)]) {
      h.fate = 0;
    } else {
      const double tn = fmin(tm[0], fmin(tm[1], tm[2]));
      const int cx = fabs(tm[0] - tn) <= 1e-12, cy = fabs(tm[1] - tn) <= 1e-12, cz = fabs(tm[2] - tn) <= 1e-12;
      if (cx) {
        i += st[0];
        tm[0] += td[0];
        h.nx = -(double)st[0];
        h.ny = 0.0;
        h.nz = 0.0;
      }
      if (cy) {
        j += st[1];
        tm[1] += td[1];
        if (!cx) {
          h.nx = 0.0;
          h.ny = -(double)st[1];
          h.nz = 0.0;
        }
      }
      if (cz) {
        k += st[2];
        tm[2] += td[2];
        if (!cx && !cy) {
          h.nx = 0.0;
          h.ny = 0.0;
          h.nz = -(double)st[2];
        }
      }
      h.t = tn;
    }
  }
  if (h.fate == -1) h.fate = 3;
  return h;
}

static void lambertian(uint32_t* s, double nx, double ny, double nz, double* dx, double* dy, double* dz) {
  const double xi1 = mb_rand(s), xi2 = mb_rand(s);
  double hx = 1.0, hy = 0.0, hz = 0.0;
  if (fabs(nx) > 0.9) {
    hx = 0.0;
    hy = 1.0;
  }
  double ux = hy * nz - hz * ny, uy = hz * nx - hx * nz, uz = hx * ny - hy * nx;
  const double un = sqrt(ux * ux + uy * uy + uz * uz);
  ux /= un;
  uy /= un;
  uz /= un;
  const double vx = ny * uz - nz * uy, vy = nz * ux - nx * uz, vz = nx * uy - ny * ux;
  const double r = sqrt(xi1), phi = (2.0 * M_PI) * xi2;
  const double cx = r * cos(phi), cy = r * sin(phi), cz = sqrt(fmax(0.0, 1.0 - xi1));
  *dx = (cx * ux + cy * vx) + cz * nx;
  *dy = (cx * uy + cy * vy) + cz * ny;
  *dz = (cx * uz + cy * vz) + cz * nz;
}

/* out: 8 tallies (properties) or 4 counts in out[0..3] (penetration) */
void oracle_multibounce(const uint8_t* solid, int sx, int sy, int sz, long long n, uint32_t seed, double eps,
                        int max_bounces, int hit_point, int penetration, double* out) {
  double a0 = 0, a1 = 0, a2 = 0, a3 = 0, a4 = 0, a5 = 0, a6 = 0, a7 = 0;
#pragma omp parallel for schedule(dynamic, 1024) reduction(+ : a0, a1, a2, a3, a4, a5, a6, a7)
  for (long long ray = 0; ray < n; ++ray) {
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    uint32_t s = mb_hash(seed + (uint32_t)(ray + 1) * 747796405u);
    const double ry = mb_rand(&s), rz = mb_rand(&s);
    double ox = 0.0, oy = ry * (double)sy, oz = rz * (double)sz;
    double dx = 1.0, dy = 0.0, dz = 0.0;
    if (penetration) lambertian(&s, 1.0, 0.0, 0.0, &dx, &dy, &dz);
    hit_t h = trace(solid, sx, sy, sz, ox, oy, oz, dx, dy, dz);
    if (h.fate != 0) {
      if (penetration) acc[h.fate == 1 ? 0 : (h.fate == 2 ? 1 : 3)] += 1.0;
      else {
        acc[2] += 1.0;
        acc[3] += h.t;
      }
    } else {
      double nx = h.nx, ny = h.ny, nz = h.nz, dist = h.t;
      if (nx * nx + ny * ny + nz * nz <= 1e-24) {
        nx = -dx;
        ny = -dy;
        nz = -dz;
      }
      if (!penetration) {
        acc[0] += 1.0;
        acc[1] += dist;
      }
      if (hit_point) {
        ox += dx * dist;
        oy += dy * dist;
        oz += dz * dist;
      }
      for (int bounces = 0;;) {
        if (!penetration) acc[4] += 1.0;
        if (mb_rand(&s) < eps) {
          if (penetration) acc[2] += 1.0;
          break;
        }
        const double px = dx, py = dy, pz = dz;
        lambertian(&s, nx, ny, nz, &dx, &dy, &dz);
        if (!penetration) {
          const double mu = (px * dx + py * dy) + pz * dz;
          acc[5] += 1.0;
          acc[6] += mu;
          acc[7] += mu * mu;
        }
        if (++bounces >= max_bounces) {
          if (penetration) acc[3] += 1.0;
          break;
        }
        if (hit_point) {
          ox += nx * 1e-9;
          oy += ny * 1e-9;
          oz += nz * 1e-9;
        } else {
          ox = (ox + px * dist) + nx * 1e-9;
          oy = (oy + py * dist) + ny * 1e-9;
          oz = (oz + pz * dist) + nz * 1e-9;
        }
        h = trace(solid, sx, sy, sz, ox, oy, oz, dx, dy, dz);
        if (h.fate != 0) {
          if (penetration) acc[h.fate == 1 ? 0 : (h.fate == 2 ? 1 : 3)] += 1.0;
          break;
        }
        nx = h.nx;
        ny = h.ny;
        nz = h.nz;
        dist = h.t;
        if (nx * nx + ny * ny + nz * nz <= 1e-24) {
          nx = -dx;
          ny = -dy;
          nz = -dz;
        }
        ox += dx * dist;
        oy += dy * dist;
        oz += dz * dist;
      }
    }
    a0 += acc[0];
    a1 += acc[1];
    a2 += acc[2];
    a3 += acc[3];
    a4 += acc[4];
    a5 += acc[5];
    a6 += acc[6];
    a7 += acc[7];
  }
  out[0] = a0;
  out[1] = a1;
  out[2] = a2;
  out[3] = a3;
  out[4] = a4;
  out[5] = a5;
  out[6] = a6;
  out[7] = a7;
}
