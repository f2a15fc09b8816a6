/* ORACLE — test infrastructure only. CPU restatement of the reference's
 * first-hit voxel traversal, used by the tests, by __graft_entry__.smoke() and by
 * bench.py's CPU-baseline leg as the checker. The product path never calls it.
 *
 * Follows porerad/view_factors.py:185-258 (_initial_cell, _axis_state,
 * _trace_kernel): Amanatides-Woo cell walk in binary64 with a 1e-12 tie
 * tolerance, periodic y/z, walls at x < 0 (hot) and x >= nx (cold), and the
 * step cap max(10*N^3 + 10, min(8 nx (1 + (|dy|+|dz|)/|dx|) + 100, 1e8)).
 * Compiled with -ffp-contract=off so every operation rounds once, as the
 * Numba-compiled reference does.
 */
#include <math.h>
#include <stdint.h>

#define ORC_TIE 1.0e-12
#define ORC_INF 1.0e300

static long orc_initial_cell(double pos, double dir) {
  long idx = (long)floor(pos);
  if (dir < 0.0 && fabs(pos - rint(pos)) <= ORC_TIE) idx -= 1;
  return idx;
}

static void orc_axis(double pos, double dir, long idx, long* step, double* tmax, double* tdelta) {
  if (dir > 0.0) {
    *step = 1;
    *tmax = (((double)idx + 1.0) - pos) / dir;
    *tdelta = 1.0 / dir;
  } else if (dir < 0.0) {
    *step = -1;
    *tmax = ((double)idx - pos) / dir;
    *tdelta = -1.0 / dir;
  } else {
    *step = 0;
    *tmax = ORC_INF;
    *tdelta = ORC_INF;
  }
}

static long orc_mod(long a, long n) {
  long m = a % n;
  return m < 0 ? m + n : m;
}

/* receiver[r] = first patch hit, failed[r] = 1 when unresolved; steps[r] (optional)
 * = number of cells visited. Arrays are C-contiguous: origins/dirs (n_rays, 3),
 * solid (nx, ny, nz) uint8, hot/cold (ny, nz) int32, cell_face (nx*ny*nz, 6) int32. */
void oracle_trace(const uint8_t* solid, long nx, long ny, long nz, const double* origins,
                  const double* dirs, long n_rays, const int32_t* hot, const int32_t* cold,
                  const int32_t* cell_face, int32_t* receiver, uint8_t* failed, int64_t* steps) {
  const long n_cells = nx * ny * nz;
#pragma omp parallel for schedule(dynamic, 1024)
  for (long r = 0; r < n_rays; ++r) {
    const double ox = origins[3 * r], oy = origins[3 * r + 1], oz = origins[3 * r + 2];
    const double dx = dirs[3 * r], dy = dirs[3 * r + 1], dz = dirs[3 * r + 2];
    int32_t hit = -1;
    int done = 0;
    long visited = 0;
    receiver[r] = -1;
    failed[r] = 0;
    if (dx == 0.0) {
      failed[r] = 1;
      if (steps) steps[r] = 0;
      continue;
    }
    long i = orc_initial_cell(ox, dx), j = orc_initial_cell(oy, dy), k = orc_initial_cell(oz, dz);
    long sx, sy, sz;
    double tx, ty, tz, ddx, ddy, ddz;
    orc_axis(ox, dx, i, &sx, &tx, &ddx);
    orc_axis(oy, dy, j, &sy, &ty, &ddy);
    orc_axis(oz, dz, k, &sz, &tz, &ddz);
    double t = 0.0;
    int face = -1;
    double scale = 8.0 * (double)nx * (1.0 + (fabs(dy) + fabs(dz)) / fabs(dx)) + 100.0;
    if (scale > 100000000.0) scale = 100000000.0;
    long cap = 10 * n_cells + 10;
    if ((long)scale > cap) cap = (long)scale;
    for (long it = 0; it < cap; ++it) {
      visited++;
      if (i < 0 || i >= nx) {
        long jj = orc_mod((long)floor(oy + dy * t), ny);
        long kk = orc_mod((long)floor(oz + dz * t), nz);
        hit = (i < 0) ? hot[jj * nz + kk] : cold[jj * nz + kk];
        done = 1;
        break;
      }
      long jj = orc_mod(j, ny), kk = orc_mod(k, nz);
      long cell = (i * ny + jj) * nz + kk;
      if (solid[cell] != 0) {
        hit = (face >= 0) ? cell_face[cell * 6 + face] : -1;
        done = 1;
        break;
      }
      double tn = tx;
      if (ty < tn) tn = ty;
      if (tz < tn) tn = tz;
      const int cx = fabs(tx - tn) <= ORC_TIE;
      const int cy = fabs(ty - tn) <= ORC_TIE;
      const int cz = fabs(tz - tn) <= ORC_TIE;
      if (cx) {
        i += sx;
        tx += ddx;
        face = sx > 0 ? 1 : 0;
      }
      if (cy) {
        j += sy;
        ty += ddy;
        if (!cx) face = sy > 0 ? 3 : 2;
      }
      if (cz) {
        k += sz;
        tz += ddz;
        if (!cx && !cy) face = sz > 0 ? 5 : 4;
      }
      t = tn;
    }
    receiver[r] = hit;
    if (!done || hit < 0) failed[r] = 1;
    if (steps) steps[r] = visited;
  }
}
