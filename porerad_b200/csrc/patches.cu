// Surface patches of an x-oriented voxel geometry on the device.
//
// Follows build_surface_patches, porerad/view_factors.py:70-132:
//  - wall patches first, one per boundary cell that is pore, in (j, k) order with
//    the hot (x = 0) patch before the cold (x = nx) patch (view_factors.py:85-92);
//  - then one internal patch per solid cell face whose neighbour is pore, in
//    (i, j, k, face) order, faces 0..5 = +x, -x, +y, -y, +z, -z; y and z neighbours
//    periodic, faces on the x boundaries excluded (view_factors.py:94-109);
//  - cell_face_patch / hot_wall_patch / cold_wall_patch map a hit face back to its
//    patch (view_factors.py:112-119).
// Patch ids come from exclusive prefix sums over the per-cell face counts, so the
// order is the reference's by construction.  The same pass writes the bit-packed
// occupancy grid the traversal reads.
#include <cub/device/device_scan.cuh>

#include "pr_math.cuh"
#include "pr_objects.cuh"

namespace pr {

// Offset of a patch origin from its cell centre along the face normal: the binary64
// value of the Python expression 0.5 + 1.0e-9 (view_factors.py:106-107).
__device__ __constant__ double kFaceOffset = 0.5 + 1.0e-9;

__global__ void k_cell_faces(const uint8_t* __restrict__ phases, int64_t nx, int64_t ny, int64_t nz,
                             uint8_t* __restrict__ solid, uint8_t* __restrict__ mask,
                             int32_t* __restrict__ nfaces) {
  const int64_t n = nx * ny * nz;
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = c % nz;
    const int64_t j = (c / nz) % ny;
    const int64_t i = c / (ny * nz);
    const bool s = phases[c] == 1;
    solid[c] = s ? 1 : 0;
    unsigned m = 0;
    if (s) {
      auto pore = [&](int64_t ii, int64_t jj, int64_t kk) { return phases[(ii * ny + jj) * nz + kk] != 1; };
      if (i + 1 < nx && pore(i + 1, j, k)) m |= 1u << 0;
      if (i >= 1 && pore(i - 1, j, k)) m |= 1u << 1;
      if (pore(i, j + 1 == ny ? 0 : j + 1, k)) m |= 1u << 2;
      if (pore(i, j == 0 ? ny - 1 : j - 1, k)) m |= 1u << 3;
      if (pore(i, j, k + 1 == nz ? 0 : k + 1)) m |= 1u << 4;
      if (pore(i, j, k == 0 ? nz - 1 : k - 1)) m |= 1u << 5;
    }
    mask[c] = (uint8_t)m;
    nfaces[c] = __popc(m);
  }
}

// Bit c of the flat occupancy array = solid flag of cell c = (i ny + j) nz + k: word w holds
// cells 32 w .. 32 w + 31, so a cell's occupancy bit and its cell_face_patch rows share the
// one index.
__global__ void k_pack_occupancy(const uint8_t* __restrict__ solid, int64_t n_cells, uint32_t* __restrict__ occ) {
  const int64_t n = (n_cells + 31) / 32;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    uint32_t word = 0;
    for (int b = 0; b < 32; ++b) {
      const int64_t c = t * 32 + b;
      if (c < n_cells && solid[c]) word |= 1u << b;
    }
    occ[t] = word;
  }
}

__global__ void k_wall_counts(const uint8_t* __restrict__ solid, int64_t nx, int64_t ny, int64_t nz,
                              int32_t* __restrict__ nwall) {
  const int64_t n = ny * nz;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    const int hot = solid[t] == 0;                            // cell (0, j, k)
    const int cold = solid[(nx - 1) * ny * nz + t] == 0;      // cell (nx-1, j, k)
    nwall[t] = hot + cold;
  }
}

__global__ void k_write_walls(const uint8_t* __restrict__ solid, int64_t nx, int64_t ny, int64_t nz,
                              const int32_t* __restrict__ woff, int8_t* __restrict__ cls,
                              int8_t* __restrict__ face, int8_t* __restrict__ code, int32_t* __restrict__ cell,
                              double* __restrict__ origin, int32_t* __restrict__ hot_map,
                              int32_t* __restrict__ cold_map) {
  const int64_t n = ny * nz;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t j = t / nz, k = t % nz;
    int32_t id = woff[t];
    const bool hot = solid[t] == 0;
    const bool cold = solid[(nx - 1) * ny * nz + t] == 0;
    const double y = (double)j + 0.5, z = (double)k + 0.5;
    hot_map[t] = hot ? id : -1;
    if (hot) {
      cls[id] = 0; face[id] = -1; code[id] = 0; cell[id] = -1;
      origin[3 * (int64_t)id] = 1.0e-9;
      origin[3 * (int64_t)id + 1] = y;
      origin[3 * (int64_t)id + 2] = z;
      ++id;
    }
    cold_map[t] = cold ? id : -1;
    if (cold) {
      cls[id] = 1; face[id] = -1; code[id] = 1; cell[id] = -1;
      origin[3 * (int64_t)id] = pr_sub((double)nx, 1.0e-9);
      origin[3 * (int64_t)id + 1] = y;
      origin[3 * (int64_t)id + 2] = z;
    }
  }
}

__global__ void k_write_internal(const uint8_t* __restrict__ mask, const int32_t* __restrict__ off,
                                 int64_t nx, int64_t ny, int64_t nz, int32_t n_wall, int8_t* __restrict__ cls,
                                 int8_t* __restrict__ face, int8_t* __restrict__ code, int32_t* __restrict__ cell,
                                 double* __restrict__ origin, int32_t* __restrict__ cfp) {
  const int64_t n = nx * ny * nz;
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
    const unsigned m = mask[c];
    int32_t id = n_wall + off[c];
    const int64_t k = c % nz;
    const int64_t j = (c / nz) % ny;
    const int64_t i = c / (ny * nz);
    for (int f = 0; f < 6; ++f) {
      if (!(m & (1u << f))) {
        cfp[c * 6 + f] = -1;
        continue;
      }
      cfp[c * 6 + f] = id;
      cls[id] = 2; face[id] = (int8_t)f; code[id] = (int8_t)f; cell[id] = (int32_t)c;
      double o[3] = {(double)i + 0.5, (double)j + 0.5, (double)k + 0.5};
      const int ax = f >> 1;
      o[ax] = (f & 1) ? pr_sub(o[ax], kFaceOffset) : pr_add(o[ax], kFaceOffset);
      o[1] = pr_pymod_pos(o[1], (double)ny);
      o[2] = pr_pymod_pos(o[2], (double)nz);
      origin[3 * (int64_t)id] = o[0];
      origin[3 * (int64_t)id + 1] = o[1];
      origin[3 * (int64_t)id + 2] = o[2];
      ++id;
    }
  }
}

// Exclusive prefix sum of n int32 values (sum must fit int32), total returned on the host.
int exclusive_scan_i32(const int32_t* in, int32_t* out, int64_t n, int64_t* total, cudaStream_t s) {
  size_t tmp_bytes = 0;
  PR_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, in, out, n, s));
  DevBuf<uint8_t> tmp;
  PR_TRY(tmp.alloc(tmp_bytes + 16, s));
  PR_CUDA(cub::DeviceScan::ExclusiveSum(tmp.ptr, tmp_bytes, in, out, n, s));
  if (total) {
    int32_t last_in = 0, last_out = 0;
    PR_CUDA(cudaMemcpyAsync(&last_in, in + n - 1, 4, cudaMemcpyDeviceToHost, s));
    PR_CUDA(cudaMemcpyAsync(&last_out, out + n - 1, 4, cudaMemcpyDeviceToHost, s));
    PR_CUDA(cudaStreamSynchronize(s));
    *total = (int64_t)last_in + (int64_t)last_out;
  }
  return PR_OK;
}

int case_build(pr_case* c, const uint8_t* phases, cudaStream_t s) {
  const int64_t n = c->n_cells;
  const int64_t lat = c->ny * c->nz;
  DevBuf<uint8_t> ph, mask;
  DevBuf<int32_t> nf, off, nw, woff;
  PR_TRY(ph.alloc(n, s));
  PR_CUDA(cudaMemcpyAsync(ph.ptr, phases, n, cudaMemcpyDefault, s));
  PR_TRY(c->solid.alloc(n, s));
  PR_TRY(mask.alloc(n, s));
  PR_TRY(nf.alloc(n, s));
  PR_TRY(off.alloc(n, s));
  ::pr::launch_mark(), k_cell_faces<<<grid_for(n, 256, 148 * 16), 256, 0, s>>>(ph.ptr, c->nx, c->ny, c->nz, c->solid.ptr, mask.ptr, nf.ptr);
  PR_CUDA(cudaGetLastError());
  PR_TRY(c->occ.alloc((n + 31) / 32, s));
  ::pr::launch_mark(), k_pack_occupancy<<<grid_for((n + 31) / 32, 256, 148 * 16), 256, 0, s>>>(c->solid.ptr, n, c->occ.ptr);
  PR_CUDA(cudaGetLastError());

  PR_TRY(nw.alloc(lat, s));
  PR_TRY(woff.alloc(lat, s));
  ::pr::launch_mark(), k_wall_counts<<<grid_for(lat, 256), 256, 0, s>>>(c->solid.ptr, c->nx, c->ny, c->nz, nw.ptr);
  PR_CUDA(cudaGetLastError());
  int64_t n_wall = 0, n_int = 0;
  PR_TRY(exclusive_scan_i32(nw.ptr, woff.ptr, lat, &n_wall, s));
  PR_TRY(exclusive_scan_i32(nf.ptr, off.ptr, n, &n_int, s));
  const int64_t P = n_wall + n_int;
  if (P >= (int64_t)INT32_MAX) {
    set_error("%lld surface patches exceed the int32 patch ids", (long long)P);
    return PR_ERR_LIMIT;
  }
  c->n_wall = n_wall;
  c->n_patches = P;
  PR_TRY(c->cls.alloc(P, s));
  PR_TRY(c->face.alloc(P, s));
  PR_TRY(c->code.alloc(P, s));
  PR_TRY(c->cell.alloc(P, s));
  PR_TRY(c->origin.alloc(3 * P, s));
  PR_TRY(c->ftab.alloc(6 * n + 2 * lat, s));
  ::pr::launch_mark(), k_write_walls<<<grid_for(lat, 256), 256, 0, s>>>(c->solid.ptr, c->nx, c->ny, c->nz, woff.ptr, c->cls.ptr,
                                                  c->face.ptr, c->code.ptr, c->cell.ptr, c->origin.ptr,
                                                  c->hot(), c->cold());
  PR_CUDA(cudaGetLastError());
  ::pr::launch_mark(), k_write_internal<<<grid_for(n, 256, 148 * 16), 256, 0, s>>>(mask.ptr, off.ptr, c->nx, c->ny, c->nz,
                                                             (int32_t)n_wall, c->cls.ptr, c->face.ptr,
                                                             c->code.ptr, c->cell.ptr, c->origin.ptr, c->cfp());
  PR_CUDA(cudaGetLastError());
  return PR_OK;
}

}  // namespace pr
