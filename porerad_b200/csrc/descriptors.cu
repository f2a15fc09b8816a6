// Morphology descriptors of a two-phase voxel microstructure (porerad/descriptors.py) on the
// device: the integer counts from which the reference's scalar and directional descriptors
// follow exactly.  Phase values: 1 solid, 0 pore (a cell of any other value is neither, as
// the reference's masks p == 1 and p == 0 treat it); the array is x-major, (i ny + j) nz + k.
//
//  * k_morph_counts (grid-stride over cells): solid and pore cells; faces between solid and
//    non-solid cells inside the box per normal axis (interface_area, descriptors.py:38-43);
//    faces between pore and non-pore cells of the periodic cell (interface_face_counts,
//    descriptors.py:120-123, whose solid is the complement of the pore); pore runs per axis
//    ending at the box faces, counted by their first cells (mean_pore_chords,
//    descriptors.py:46-48: the mean chord is pore cells over runs).
//  * k_periodic_chords (one thread per axis-parallel line): the chords of the periodic cell
//    (periodic_chords, descriptors.py:82-109: the first and last runs of a line touching both
//    ends merged into one, an all-pore line one chord of length N) as a histogram of chord
//    lengths, plus the all-pore lines.
//  * 26-connected pore clusters (pore_connectivity, descriptors.py:51-60) by a lock-free
//    union-find: each pore cell unites with its 13 neighbours that follow it in the 3x3x3
//    block, a root always hooked under the smaller root by compare-and-swap (so every parent
//    index is below its child's and each find ends within n steps); then cluster sizes, the
//    box faces each cluster touches, the largest cluster and percolation along each axis.
#include <new>

#include "pr_internal.cuh"

namespace pr {

namespace {

struct MorphGrid {
  const uint8_t* __restrict__ ph;
  int nx, ny, nz;
};

// cells number fewer than 2^31 (checked on the host): 32-bit index arithmetic throughout
__device__ __forceinline__ uint8_t phase_at(const MorphGrid& g, int i, int j, int k) {
  return g.ph[(i * g.ny + j) * g.nz + k];
}

constexpr int kMorphCounters = 11;  // solid, pore, inner faces x/y/z, periodic faces x/y/z, runs x/y/z
constexpr int kMorphThreads = 256;

// Adds K per-thread counters over the block (warp shuffles, then one warp over the warps'
// partials) and issues one atomic per counter and block.
template <int K>
__device__ __forceinline__ void block_add(unsigned long long (&v)[K], unsigned long long* __restrict__ out) {
  __shared__ unsigned long long part[kMorphThreads / 32][K];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < K; ++q) {
    unsigned long long x = v[q];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if (lane == 0) part[w][q] = x;
  }
  __syncthreads();
  if (w == 0) {
#pragma unroll
    for (int q = 0; q < K; ++q) {
      unsigned long long x = lane < kMorphThreads / 32 ? part[lane][q] : 0ull;
      for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
      if (lane == 0 && x) atomicAdd(out + q, x);
    }
  }
}

__global__ void __launch_bounds__(kMorphThreads) k_morph_counts(MorphGrid g, unsigned long long* __restrict__ counters) {
  const int64_t n = (int64_t)g.nx * g.ny * g.nz;
  unsigned long long c[kMorphCounters];
#pragma unroll
  for (int q = 0; q < kMorphCounters; ++q) c[q] = 0;
  const int plane = g.ny * g.nz;
  for (int64_t tt = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; tt < n; tt += (int64_t)gridDim.x * blockDim.x) {
    const int t = (int)tt;
    const int i = t / plane, r = t - i * plane, j = r / g.nz, k = r - j * g.nz;
    const uint8_t v = g.ph[t];
    const int ip = i + 1 < g.nx ? i + 1 : 0, jp = j + 1 < g.ny ? j + 1 : 0, kp = k + 1 < g.nz ? k + 1 : 0;
    const uint8_t vx = phase_at(g, ip, j, k), vy = phase_at(g, i, jp, k), vz = phase_at(g, i, j, kp);
    const uint8_t bx = i ? phase_at(g, i - 1, j, k) : 1, by = j ? phase_at(g, i, j - 1, k) : 1,
                  bz = k ? phase_at(g, i, j, k - 1) : 1;
    const bool s = v == 1, p = v == 0;
    c[0] += s;
    c[1] += p;
    if (i + 1 < g.nx) c[2] += s != (vx == 1);
    if (j + 1 < g.ny) c[3] += s != (vy == 1);
    if (k + 1 < g.nz) c[4] += s != (vz == 1);
    c[5] += p != (vx == 0);
    c[6] += p != (vy == 0);
    c[7] += p != (vz == 0);
    c[8] += p && bx != 0;  // a pore run starts here (the box face counts as a non-pore cell)
    c[9] += p && by != 0;
    c[10] += p && bz != 0;
  }
  block_add<kMorphCounters>(c, counters);
}

// Chords of the lines along `axis` (0 x, 1 y, 2 z) of the periodic cell: hist[len] counts
// the chords of each length (len <= N), *all_pore the lines lying entirely in the pore.  One
// thread per line reads it 32 cells at a time (independent loads) into a pore bit mask and
// walks the solid cells of the mask.  The histogram is kept in shared memory when
// shared_len (= N + 1) is non-zero.
__global__ void __launch_bounds__(kMorphThreads) k_periodic_chords(MorphGrid g, int axis, int shared_len,
                                                                   unsigned long long* __restrict__ hist,
                                                                   unsigned long long* __restrict__ all_pore) {
  extern __shared__ unsigned long long sh_hist[];
  for (int q = threadIdx.x; q < shared_len; q += blockDim.x) sh_hist[q] = 0;
  __syncthreads();
  unsigned long long* h = shared_len ? sh_hist : hist;
  const int N = axis == 0 ? g.nx : axis == 1 ? g.ny : g.nz;
  // the line's other two coordinates (a, b) in index order; cell stride along the line
  const int d2 = axis == 2 ? g.ny : g.nz;
  const int lines = (axis == 0 ? g.ny : g.nx) * d2;
  const int step = axis == 0 ? g.ny * g.nz : axis == 1 ? g.nz : 1;
  unsigned long long n_all[1] = {0};
  for (int64_t LL = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; LL < lines; LL += (int64_t)gridDim.x * blockDim.x) {
    const int L = (int)LL;
    const int a = L / d2, b = L - a * d2;
    const int base = axis == 0 ? a * g.nz + b : axis == 1 ? a * g.ny * g.nz + b : (a * g.ny + b) * g.nz;
    const uint8_t* line = g.ph + base;
    int head = -1;  // length of the run starting at 0, held back for a wrap merge; 0: none
    int run = 0;
    for (int s0 = 0; s0 < N; s0 += 32) {
      const int cnt = N - s0 < 32 ? N - s0 : 32;
      unsigned int m = 0;
#pragma unroll
      for (int q = 0; q < 32; ++q)
        if (q < cnt) m |= (unsigned int)(line[(s0 + q) * step] == 0) << q;
      unsigned int sol = ~m & (cnt == 32 ? 0xffffffffu : (1u << cnt) - 1u);
      int pos = 0;
      while (sol) {
        const int p = __ffs(sol) - 1;
        run += p - pos;
        if (head < 0) head = run;  // the first solid cell closes the run at 0 (possibly empty)
        else if (run) atomicAdd(h + run, 1ull);
        run = 0;
        pos = p + 1;
        sol &= sol - 1;
      }
      run += cnt - pos;
    }
    if (head < 0) {  // no solid cell: an all-pore line, one chord of length N
      atomicAdd(h + N, 1ull);
      ++n_all[0];
    } else if (run + head) {  // the runs touching both ends (either may be empty) form one chord
      atomicAdd(h + (run + head), 1ull);
    }
  }
  block_add<1>(n_all, all_pore);
  if (shared_len) {
    __syncthreads();
    for (int q = threadIdx.x; q < shared_len; q += blockDim.x)
      if (sh_hist[q]) atomicAdd(hist + q, sh_hist[q]);
  }
}

// The same chords with the lines cut into segments of `seg` <= 32 cells, one thread per
// segment and `lpl` (a power of two, at most 32) lanes per line, so that short lines still
// fill the GPU.  A segment thread emits the runs between its own solid cells; the first lane
// of the line then walks the segments' (leading pore, trailing pore, all pore) summaries in
// order, which closes the runs that cross segment boundaries and the wrap-around chord.
__global__ void __launch_bounds__(kMorphThreads) k_chords_seg(MorphGrid g, int axis, int lpl, int seg, int shared_len,
                                                              unsigned long long* __restrict__ hist,
                                                              unsigned long long* __restrict__ all_pore) {
  extern __shared__ unsigned long long sh_hist[];
  for (int q = threadIdx.x; q < shared_len; q += blockDim.x) sh_hist[q] = 0;
  __syncthreads();
  unsigned long long* h = shared_len ? sh_hist : hist;
  const int N = axis == 0 ? g.nx : axis == 1 ? g.ny : g.nz;
  const int d2 = axis == 2 ? g.ny : g.nz;
  const int lines = (axis == 0 ? g.ny : g.nx) * d2;
  const int step = axis == 0 ? g.ny * g.nz : axis == 1 ? g.nz : 1;
  const int lane = threadIdx.x & 31, first = lane & ~(lpl - 1), part = lane - first;
  const int64_t slots = ((int64_t)lines * lpl + 31) & ~(int64_t)31;  // whole warps: uniform shuffles
  unsigned long long n_all[1] = {0};
  for (int64_t gt = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; gt < slots; gt += (int64_t)gridDim.x * blockDim.x) {
    const int L = (int)(gt / lpl);
    const bool live = L < lines;
    const int s0 = part * seg;
    const int cnt = !live || s0 >= N ? 0 : (N - s0 < seg ? N - s0 : seg);
    int pre = cnt, suf = cnt;
    if (cnt) {
      const int a = L / d2, b = L - a * d2;
      const int base = axis == 0 ? a * g.nz + b : axis == 1 ? a * g.ny * g.nz + b : (a * g.ny + b) * g.nz;
      const uint8_t* line = g.ph + base;
      unsigned int m = 0;
#pragma unroll
      for (int q = 0; q < 32; ++q)
        if (q < cnt) m |= (unsigned int)(line[(s0 + q) * step] == 0) << q;
      unsigned int sol = ~m & (cnt == 32 ? 0xffffffffu : (1u << cnt) - 1u);
      if (sol) {
        pre = __ffs(sol) - 1;
        suf = cnt - 1 - (31 - __clz(sol));
        int prev = pre;
        sol &= sol - 1;
        while (sol) {  // runs between consecutive solid cells of this segment
          const int p = __ffs(sol) - 1;
          if (p - prev - 1 > 0) atomicAdd(h + (p - prev - 1), 1ull);
          prev = p;
          sol &= sol - 1;
        }
      }
    }
    const bool full = pre == cnt;  // no solid cell in the segment (an empty segment included)
    int run = 0, head = -1;
    for (int q = 0; q < lpl; ++q) {
      const int c_q = __shfl_sync(0xffffffffu, cnt, first + q);
      const int p_q = __shfl_sync(0xffffffffu, pre, first + q);
      const int s_q = __shfl_sync(0xffffffffu, suf, first + q);
      const bool f_q = __shfl_sync(0xffffffffu, (int)full, first + q) != 0;
      if (f_q) {
        run += c_q;
      } else {
        run += p_q;
        if (head < 0) head = run;
        else if (run && part == 0 && live) atomicAdd(h + run, 1ull);
        run = s_q;
      }
    }
    if (part == 0 && live) {
      if (head < 0) {
        atomicAdd(h + N, 1ull);
        ++n_all[0];
      } else if (run + head) {
        atomicAdd(h + (run + head), 1ull);
      }
    }
  }
  block_add<1>(n_all, all_pore);
  if (shared_len) {
    __syncthreads();
    for (int q = threadIdx.x; q < shared_len; q += blockDim.x)
      if (sh_hist[q]) atomicAdd(hist + q, sh_hist[q]);
  }
}

// ---- 26-connected pore clusters
//
// Tiles of 8 x 8 x 16 cells first label their own cells in shared memory; only the unions
// that cross a tile face then go through global memory, where every cell already points at
// the root of its tile-local component.  Within a tile, local indices run in the same order
// as global ones, so a component's local root is its smallest global index and the rule
// "hook the larger root under the smaller" holds across both phases.

constexpr int kTX = 8, kTY = 8, kTZ = 16, kTile = kTX * kTY * kTZ;

// forward neighbour q = 14..26 of the 3 x 3 x 3 block: offsets (di, dj, dk)
__device__ __forceinline__ void fwd_offset(int q, int& di, int& dj, int& dk) {
  di = q / 9 - 1;
  dj = (q / 3) % 3 - 1;
  dk = q % 3 - 1;
}

__device__ __forceinline__ unsigned int box_faces(const MorphGrid& g, int i, int j, int k) {
  return (i == 0 ? 1u : 0u) | (i == g.nx - 1 ? 2u : 0u) | (j == 0 ? 4u : 0u) | (j == g.ny - 1 ? 8u : 0u) |
         (k == 0 ? 16u : 0u) | (k == g.nz - 1 ? 32u : 0u);
}

__device__ __forceinline__ int s_find(volatile int* p, int x) {
  for (int guard = 0; guard < kTile; ++guard) {
    const int q = p[x];
    if (q == x) return x;
    const int gq = p[q];
    if (gq != q) p[x] = gq;  // path halving: any ancestor is a valid parent
    x = q;
  }
  return -1;
}

__device__ __forceinline__ int uf_find(int* __restrict__ parent, int x, int limit) {
  for (int guard = 0; guard < limit; ++guard) {
    const int p = __ldcg(parent + x);
    if (p == x) return x;
    const int gp = __ldcg(parent + p);
    if (gp != p) parent[x] = gp;
    x = p;
  }
  return -1;
}

// union of the components of x and y; false when a find ran past its bound
__device__ __forceinline__ bool uf_union(int* __restrict__ parent, int x, int y, int n) {
  for (int guard = 0; guard < n; ++guard) {
    x = uf_find(parent, x, n);
    y = uf_find(parent, y, n);
    if (x < 0 || y < 0) return false;
    if (x == y) return true;
    if (x < y) {
      const int s = x;
      x = y;
      y = s;
    }
    if (atomicCAS(parent + x, x, y) == x) return true;
  }
  return false;
}

// One tile per block: local labels in shared memory; parent[cell] = global index of its local
// root (-1 for other cells); size/faces of each local component stored at its root.
__global__ void __launch_bounds__(256) k_label_tiles(MorphGrid g, int tiles_y, int tiles_z, int* __restrict__ parent,
                                                     unsigned int* __restrict__ size,
                                                     unsigned int* __restrict__ faces,
                                                     unsigned int* __restrict__ bad) {
  __shared__ int par_s[kTile];
  __shared__ unsigned int cnt_s[kTile];
  __shared__ unsigned int face_s[kTile];
  const int tile = blockIdx.x;
  const int i0 = tile / (tiles_y * tiles_z) * kTX, j0 = (tile / tiles_z) % tiles_y * kTY, k0 = tile % tiles_z * kTZ;
  volatile int* vp = par_s;
  const int lane = threadIdx.x & 31;
  // Runs along z first, without atomics: a warp holds two rows of kTZ = 16 cells, and every
  // pore cell points at the first cell of its run (the nearest solid lane below it, +1).
  static_assert(kTZ == 16 && kTile % 256 == 0, "two tile rows per warp; uniform loops");
  for (int l = threadIdx.x; l < kTile; l += blockDim.x) {
    const int i = i0 + l / (kTY * kTZ), j = j0 + (l / kTZ) % kTY, k = k0 + l % kTZ;
    const bool in = i < g.nx && j < g.ny && k < g.nz;
    const bool pore = in && g.ph[(i * g.ny + j) * g.nz + k] == 0;
    const unsigned int pm = __ballot_sync(0xffffffffu, pore);
    const int row0 = lane & ~(kTZ - 1);
    const unsigned int below = lane ? 0xffffffffu >> (32 - lane) : 0u;
    const unsigned int solid_below = ~pm & below & (0xFFFFu << row0);
    const int start = solid_below ? 32 - __clz(solid_below) : row0;
    par_s[l] = pore ? l - (lane - start) : -1;
    cnt_s[l] = 0;
    face_s[l] = 0;
  }
  __syncthreads();
  // The other 12 forward neighbours.  Lanes of a run ask for the same union (same current
  // parents on both sides), so one lane per distinct pair of a warp performs it.
  for (int l = threadIdx.x; l < kTile; l += blockDim.x) {
    const bool pore = vp[l] >= 0;
    const int li = l / (kTY * kTZ), lj = (l / kTZ) % kTY, lk = l % kTZ;
    for (int q = 15; q < 27; ++q) {
      int di, dj, dk;
      fwd_offset(q, di, dj, dk);
      const int a = li + di, b = lj + dj, c = lk + dk;
      const bool inside = pore && a < kTX && b >= 0 && b < kTY && c >= 0 && c < kTZ;
      const int u = inside ? (a * kTY + b) * kTZ + c : 0;
      const int pu = inside ? vp[u] : -1;
      const bool ok = pu >= 0;
      const int pl = ok ? vp[l] : 0;
      const unsigned int key = ok ? ((unsigned int)pl << 16) | (unsigned int)pu : 0xFFFFFFFFu;
      const unsigned int grp = __match_any_sync(0xffffffffu, key);
      if (!ok || lane != __ffs(grp) - 1) continue;
      int x = pl, y = pu, guard = 0;
      for (; guard < kTile; ++guard) {
        x = s_find(vp, x);
        y = s_find(vp, y);
        if (x < 0 || y < 0) {
          guard = kTile;
          break;
        }
        if (x == y) break;
        if (x < y) {
          const int t = x;
          x = y;
          y = t;
        }
        if (atomicCAS(par_s + x, x, y) == x) break;
      }
      if (guard >= kTile) atomicOr(bad, 1u);
    }
  }
  __syncthreads();
  for (int l = threadIdx.x; l < kTile; l += blockDim.x)
    if (vp[l] >= 0) {
      const int r = s_find(vp, l);
      if (r < 0) atomicOr(bad, 1u);
      else vp[l] = r;
    }
  __syncthreads();
  for (int l = threadIdx.x; l < kTile; l += blockDim.x) {  // kTile is a multiple of blockDim.x: uniform loop
    const int i = i0 + l / (kTY * kTZ), j = j0 + (l / kTZ) % kTY, k = k0 + l % kTZ;
    const bool in = i < g.nx && j < g.ny && k < g.nz;
    const int r = vp[l];
    if (in) {
      const int cell = (i * g.ny + j) * g.nz + k;
      const int ri = i0 + r / (kTY * kTZ), rj = j0 + (r / kTZ) % kTY, rk = k0 + r % kTZ;
      parent[cell] = r >= 0 ? (ri * g.ny + rj) * g.nz + rk : -1;
    }
    const unsigned int same = __match_any_sync(0xffffffffu, r);
    if (r >= 0 && lane == __ffs(same) - 1) atomicAdd(cnt_s + r, (unsigned int)__popc(same));
    const unsigned int f = r >= 0 ? box_faces(g, i, j, k) : 0u;
    if (f) atomicOr(face_s + r, f);
  }
  __syncthreads();
  for (int l = threadIdx.x; l < kTile; l += blockDim.x)
    if (vp[l] == l) {
      const int i = i0 + l / (kTY * kTZ), j = j0 + (l / kTZ) % kTY, k = k0 + l % kTZ;
      const int cell = (i * g.ny + j) * g.nz + k;
      size[cell] = cnt_s[l];
      faces[cell] = face_s[l];
    }
}

// Unions across tile faces, one block per tile: each pore cell on a face of its tile pairs
// the parents of itself and of every pore forward neighbour in another tile (tile-local roots,
// or roots they were hooked under since); a shared-memory hash set keeps the distinct pairs,
// and one thread unites each (a few dozen per tile instead of one per cell pair).
constexpr int kPairSlots = 2048;

__global__ void __launch_bounds__(256) k_label_merge(MorphGrid g, int tiles_y, int tiles_z, int* __restrict__ parent,
                                                     unsigned int* __restrict__ bad) {
  __shared__ unsigned long long pairs[kPairSlots];
  const int n = g.nx * g.ny * g.nz;
  for (int q = threadIdx.x; q < kPairSlots; q += blockDim.x) pairs[q] = ~0ull;
  __syncthreads();
  const int tile = blockIdx.x;
  const int i0 = tile / (tiles_y * tiles_z) * kTX, j0 = (tile / tiles_z) % tiles_y * kTY, k0 = tile % tiles_z * kTZ;
  const int lane = threadIdx.x & 31;
  // uniform loops (kTile is a multiple of the block; 13 offsets for every lane) so that the lanes of
  // a warp asking for the same pair of parents meet in one __match_any_sync: one of them goes on
  for (int l = threadIdx.x; l < kTile; l += blockDim.x) {
    const int li = l / (kTY * kTZ), lj = (l / kTZ) % kTY, lk = l % kTZ;
    const int i = i0 + li, j = j0 + lj, k = k0 + lk;
    const bool face = li == kTX - 1 || lj == 0 || lj == kTY - 1 || lk == 0 || lk == kTZ - 1;
    const bool in = i < g.nx && j < g.ny && k < g.nz;
    const int t = in ? (i * g.ny + j) * g.nz + k : 0;
    const bool cand = face && in && g.ph[t] == 0;
    const int pt = cand ? __ldcg(parent + t) : 0;
    for (int q = 14; q < 27; ++q) {
      int di, dj, dk;
      fwd_offset(q, di, dj, dk);
      const bool other_tile = li + di >= kTX || lj + dj < 0 || lj + dj >= kTY || lk + dk < 0 || lk + dk >= kTZ;
      const int a = i + di, b = j + dj, c = k + dk;
      bool ok = cand && other_tile && a < g.nx && b >= 0 && b < g.ny && c >= 0 && c < g.nz;
      const int u = ok ? (a * g.ny + b) * g.nz + c : 0;
      ok = ok && g.ph[u] == 0;
      const int pu = ok ? __ldcg(parent + u) : 0;
      const unsigned long long key = ok ? ((unsigned long long)(unsigned int)pt << 32) | (unsigned int)pu : ~0ull;
      const unsigned int grp = __match_any_sync(0xffffffffu, key);
      if (!ok || lane != __ffs(grp) - 1) continue;
      unsigned int h = (unsigned int)((key * 0x9E3779B97F4A7C15ull) >> 53) & (kPairSlots - 1);
      bool fresh = true;  // a full probe sequence unites without the check (correct, only slower)
      for (int probe = 0; probe < 64; ++probe) {
        const unsigned long long old = atomicCAS(pairs + h, ~0ull, key);
        if (old == ~0ull) break;
        if (old == key) {
          fresh = false;
          break;
        }
        h = (h + 1) & (kPairSlots - 1);
      }
      if (fresh && !uf_union(parent, pt, pu, n)) atomicOr(bad, 1u);
    }
  }
}

// Local components hooked under another root pass their size and faces to it.
__global__ void __launch_bounds__(256) k_label_roots(MorphGrid g, int* __restrict__ parent,
                                                     unsigned int* __restrict__ size,
                                                     unsigned int* __restrict__ faces,
                                                     unsigned int* __restrict__ bad) {
  const int n = g.nx * g.ny * g.nz;
  for (int64_t tt = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; tt < n; tt += (int64_t)gridDim.x * blockDim.x) {
    const int t = (int)tt;
    const unsigned int s = size[t];
    if (!s) continue;  // not the root of a tile-local component
    const int r = uf_find(parent, t, n);
    if (r < 0) {
      atomicOr(bad, 1u);
      continue;
    }
    if (r == t) continue;
    atomicAdd(size + r, s);
    const unsigned int f = faces[t];
    if (f) atomicOr(faces + r, f);
  }
}

// out[0] largest cluster, out[1] number of clusters, out[2] percolation bits (axis a: bit a)
__global__ void __launch_bounds__(256) k_label_summary(const int* __restrict__ parent,
                                                       const unsigned int* __restrict__ size,
                                                       const unsigned int* __restrict__ faces, int n,
                                                       unsigned long long* __restrict__ out) {
  unsigned long long mx = 0, clusters = 0, perc = 0;
  for (int64_t tt = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; tt < n; tt += (int64_t)gridDim.x * blockDim.x) {
    const int t = (int)tt;
    if (parent[t] != t) continue;  // only the roots of whole clusters
    const unsigned int s = size[t];
    mx = s > mx ? s : mx;
    ++clusters;
    const unsigned int f = faces[t];
    for (int a = 0; a < 3; ++a)
      if ((f >> (2 * a) & 3u) == 3u) perc |= 1ull << a;
  }
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long m2 = __shfl_xor_sync(0xffffffffu, mx, o);
    mx = m2 > mx ? m2 : mx;
    clusters += __shfl_xor_sync(0xffffffffu, clusters, o);
    perc |= __shfl_xor_sync(0xffffffffu, perc, o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (mx) atomicMax(out, mx);
    if (clusters) atomicAdd(out + 1, clusters);
    if (perc) atomicOr(out + 2, perc);
  }
}

constexpr int kChordSharedMax = 6144;  // histogram entries kept in shared memory (48 KB)

}  // namespace

}  // namespace pr

using namespace pr;

extern "C" {

PR_API int pr_morphology_counts(const uint8_t* phases, int64_t nx, int64_t ny, int64_t nz, int what,
                                pr_morphology* out, int64_t* chord_counts_x, int64_t* chord_counts_y,
                                int64_t* chord_counts_z, void* stream) {
  PR_ARG(phases && out, "phases and out must not be NULL");
  PR_ARG(nx > 0 && ny > 0 && nz > 0, "phase array must not be empty");
  PR_ARG((what & ~(PR_MORPH_CONNECTIVITY | PR_MORPH_CHORDS)) == 0, "unknown descriptor flags %d", what);
  if ((double)nx * (double)ny * (double)nz >= (double)INT32_MAX) {
    set_error("phase array of %.0f cells exceeds the 2^31 - 2 cells of this build", (double)nx * ny * nz);
    return PR_ERR_LIMIT;
  }
  const int64_t n = nx * ny * nz;
  int64_t* chord_out[3] = {chord_counts_x, chord_counts_y, chord_counts_z};
  const cudaStream_t s = (cudaStream_t)stream;
  const int64_t dims[3] = {nx, ny, nz};

  DevBuf<uint8_t> staged;
  const uint8_t* ph = phases;
  if (!is_device_pointer(phases)) {
    PR_TRY(staged.alloc((size_t)n, s));
    PR_CUDA(cudaMemcpyAsync(staged.ptr, phases, (size_t)n, cudaMemcpyHostToDevice, s));
    ph = staged.ptr;
  }
  // results: counters, all-pore lines x/y/z, cluster summary (3), status, then the histograms
  const int64_t head = kMorphCounters + 3 + 3 + 1;
  const int64_t words = head + (nx + 1) + (ny + 1) + (nz + 1);
  DevBuf<unsigned long long> res;
  PR_TRY(res.alloc((size_t)words, s));
  PR_CUDA(cudaMemsetAsync(res.ptr, 0, (size_t)words * 8, s));
  const MorphGrid g{ph, (int)nx, (int)ny, (int)nz};
  const int cap = sm_count() * 8;

  timer_begin(kTimerMorph, s);
  k_morph_counts<<<grid_for(n, 256, cap), 256, 0, s>>>(g, res.ptr);
  timer_end(kTimerMorph, s);
  launch_mark();
  PR_CUDA(cudaGetLastError());

  if (what & PR_MORPH_CHORDS) {
    unsigned long long* hist = res.ptr + head;
    for (int a = 0; a < 3; ++a) {
      const int64_t lines = n / dims[a];
      const int sh_len = dims[a] + 1 <= kChordSharedMax ? (int)(dims[a] + 1) : 0;
      if (dims[a] <= 1024) {  // segments of at most 32 cells, a power-of-two number of lanes per line
        int lpl = 1;
        while (lpl < 32 && (dims[a] + lpl - 1) / lpl > 16) lpl *= 2;
        const int seg = (int)((dims[a] + lpl - 1) / lpl);
        k_chords_seg<<<grid_for(lines * lpl, 256, cap), 256, (size_t)sh_len * 8, s>>>(
            g, a, lpl, seg, sh_len, hist, res.ptr + kMorphCounters + a);
      } else {
        k_periodic_chords<<<grid_for(lines, 256, cap), 256, (size_t)sh_len * 8, s>>>(g, a, sh_len, hist,
                                                                                   res.ptr + kMorphCounters + a);
      }
      launch_mark();
      PR_CUDA(cudaGetLastError());
      hist += dims[a] + 1;
    }
  }

  DevBuf<int> parent;
  DevBuf<unsigned int> cl;  // sizes (n), faces (n), status (1)
  if (what & PR_MORPH_CONNECTIVITY) {
    PR_TRY(parent.alloc((size_t)n, s));
    PR_TRY(cl.alloc((size_t)(2 * n + 1), s));
    PR_CUDA(cudaMemsetAsync(cl.ptr, 0, (size_t)(2 * n + 1) * 4, s));
    unsigned int* bad = cl.ptr + 2 * n;
    timer_begin(kTimerLabel, s);
    const int ty = (int)((ny + kTY - 1) / kTY), tz = (int)((nz + kTZ - 1) / kTZ);
    const int tiles = (int)((nx + kTX - 1) / kTX) * ty * tz;
    const int grid = grid_for(n, 256, cap);
    k_label_tiles<<<tiles, 256, 0, s>>>(g, ty, tz, parent.ptr, cl.ptr, cl.ptr + n, bad);
    k_label_merge<<<tiles, 256, 0, s>>>(g, ty, tz, parent.ptr, bad);
    k_label_roots<<<grid, 256, 0, s>>>(g, parent.ptr, cl.ptr, cl.ptr + n, bad);
    k_label_summary<<<grid, 256, 0, s>>>(parent.ptr, cl.ptr, cl.ptr + n, (int)n, res.ptr + kMorphCounters + 3);
    timer_end(kTimerLabel, s);
    for (int q = 0; q < 4; ++q) launch_mark();
    PR_CUDA(cudaGetLastError());
    PR_CUDA(cudaMemcpyAsync(res.ptr + kMorphCounters + 6, bad, 4, cudaMemcpyDeviceToDevice, s));
  }

  unsigned long long* host = new (std::nothrow) unsigned long long[words];
  if (!host) {
    set_error("host allocation of %lld words failed", (long long)words);
    return PR_ERR_OOM;
  }
  cudaError_t e = cudaMemcpyAsync(host, res.ptr, (size_t)words * 8, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    delete[] host;
    set_error("CUDA error %s (%s) reading the morphology counts", cudaGetErrorName(e), cudaGetErrorString(e));
    return PR_ERR_CUDA;
  }
  const unsigned long long* c = host;
  out->cells = n;
  out->solid_cells = (int64_t)c[0];
  out->pore_cells = (int64_t)c[1];
  for (int a = 0; a < 3; ++a) {
    out->interface_faces[a] = (int64_t)c[2 + a];
    out->periodic_faces[a] = (int64_t)c[5 + a];
    out->pore_runs[a] = (int64_t)c[8 + a];
    out->all_pore_lines[a] = (what & PR_MORPH_CHORDS) ? (int64_t)c[kMorphCounters + a] : -1;
  }
  const bool conn = (what & PR_MORPH_CONNECTIVITY) != 0;
  out->largest_pore_cluster = conn ? (int64_t)c[kMorphCounters + 3] : -1;
  out->pore_clusters = conn ? (int64_t)c[kMorphCounters + 4] : -1;
  for (int a = 0; a < 3; ++a) out->pore_percolates[a] = conn ? (int32_t)((c[kMorphCounters + 5] >> a) & 1u) : -1;
  const unsigned int status = (unsigned int)(c[kMorphCounters + 6] & 0xFFFFFFFFu);
  if (what & PR_MORPH_CHORDS) {
    const unsigned long long* h = host + head;
    for (int a = 0; a < 3; ++a) {
      if (chord_out[a])
        for (int64_t l = 0; l <= dims[a]; ++l) chord_out[a][l] = (int64_t)h[l];
      h += dims[a] + 1;
    }
  }
  delete[] host;
  if (status) {
    set_error("pore cluster labelling did not settle within its step bound");
    return PR_ERR_LIMIT;
  }
  return PR_OK;
}

}  // extern "C"
