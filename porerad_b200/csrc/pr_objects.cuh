// Device-resident objects behind the opaque handles of porerad.h.
#pragma once
#include <memory>
#include <vector>

#include "pr_internal.cuh"

namespace pr {

// Switches to the object's device for the duration of a call.
struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

// Sorted CSR of integer first-hit counts: row = origin patch, col = receiver patch.
struct CountCsr {
  int64_t n_rows = 0, nnz = 0;
  DevBuf<int64_t> row_ptr;  // n_rows + 1
  DevBuf<int32_t> col;      // nnz, ascending within a row
  DevBuf<int32_t> cnt;      // nnz, > 0
};

// Symmetric exchange matrix S' = 0.5 (A F + F^T A) without the support diagonal
// (delta A, applied separately).  Entry storage, by mode:
//   kPacked:  one 32-bit word (col << bits) | n per entry, value factor * n, n = n_ij + n_ji
//             on the union of the patterns of F and F^T, columns ascending (every patch
//             with the same area and ray count, and column/count bits fit in 32);
//   kCounts:  col (int32) + n (int32) on the same union (same uniform case, wide ids);
//   kValues:  col (int32) + binary64 value 0.5 A n / R of the entry's origin patch; row i
//             holds row i of F followed by row i of F^T (two ascending runs).
enum SymMode { kPacked = 0, kCounts = 1, kValues = 2 };

// Column blocks of a union-stored S' for products that stage x in shared memory: block b
// holds columns [b W, (b + 1) W); seg[(b - 1) n + i] (b = 1 .. nb - 1) is the offset of
// block b's first entry in row i from row_ptr[i].  CTA c of a blocked product owns rows
// [cta_row[c], cta_row[c + 1]), at most rows_cap of them, split so that every CTA has
// about the same number of entries plus rows.
struct ColBlocks {
  bool ready = false;
  int W = 0, nb = 0, ctas = 0, rows_cap = 0;
  DevBuf<int32_t> seg;
  DevBuf<int64_t> cta_row;
};

struct SymCsr {
  int64_t n_rows = 0, nnz = 0;
  DevBuf<int64_t> row_ptr;
  DevBuf<uint32_t> words;  // packed words, or the column of every entry
  DevBuf<int32_t> cnt;     // kCounts
  DevBuf<double> val;      // kValues
  int mode = kPacked;
  int bits = 0;            // count bits of a packed word
  double factor = 0.0;     // 0.5 A / R in the uniform modes
  ColBlocks blk;           // union modes
};

}  // namespace pr

struct pr_case {
  int device = 0;
  int64_t nx = 0, ny = 0, nz = 0, n_cells = 0;
  int64_t n_patches = 0, n_wall = 0;
  double H = 0.0, area = 0.0;
  pr::DevBuf<uint8_t> solid;      // n_cells, 0/1
  pr::DevBuf<uint32_t> occ;       // bit-packed solid flags, bit c = cell c (flat)
  pr::DevBuf<int8_t> cls;         // patch class 0 hot, 1 cold, 2 internal
  pr::DevBuf<int8_t> face;        // patch face 0..5, -1 for walls
  pr::DevBuf<int8_t> code;        // emission normal: 0..5 as +x,-x,+y,-y,+z,-z
  pr::DevBuf<int32_t> cell;       // owning cell, -1 for walls
  pr::DevBuf<double> origin;      // (P, 3)
  // Face table: cell_face_patch (n_cells, 6), then the hot and the cold wall patch of each
  // (j, k) lattice site.  A first hit is recorded as an index into this table (its hit code).
  pr::DevBuf<int32_t> ftab;
  cudaStream_t last_stream = nullptr;
  int32_t* cfp() const { return ftab.ptr; }
  int32_t* hot() const { return ftab.ptr + 6 * n_cells; }
  int32_t* cold() const { return ftab.ptr + 6 * n_cells + ny * nz; }
  void rebind(cudaStream_t s) {
    solid.stream = occ.stream = s;
    cls.stream = face.stream = code.stream = s;
    cell.stream = origin.stream = ftab.stream = s;
  }
  size_t device_bytes() const {
    return solid.bytes() + occ.bytes() + cls.bytes() + face.bytes() + code.bytes() + cell.bytes() +
           origin.bytes() + ftab.bytes();
  }
};

struct pr_counts {
  int device = 0;
  std::shared_ptr<pr::CountCsr> csr;
  pr::DevBuf<int64_t> rays;  // rays per origin
  int64_t rays_traced = 0, dda_steps = 0;
  cudaStream_t last_stream = nullptr;
};

struct pr_operator {
  int device = 0;
  int64_t n = 0;
  std::shared_ptr<pr::CountCsr> F;
  pr::DevBuf<int64_t> rays;   // R_i
  pr::DevBuf<double> area;    // A_i
  pr::SymCsr S;
  pr::DevBuf<double> scale;   // d
  double delta = 0.0;
  int method = 0, iterations = 0;
  double row_sum_error = 0.0;
  mutable int64_t spmv_calls = 0;
  // transposed count CSR (kept from the assembly for raw_rmatvec)
  mutable std::shared_ptr<pr::CountCsr> FT;
  mutable cudaStream_t last_stream = nullptr;
};

// Cell-centred finite-volume conduction on an x-oriented grid (porerad/conduction.py): the
// conductance of each cell's +x, +y and +z face (harmonic mean times dx, 0 on the +x face of
// the last layer; y and z periodic), the diagonal of A, and the wall responses.
struct pr_conduction {
  int device = 0;
  int64_t nx = 0, ny = 0, nz = 0, n = 0;
  double H = 0.0, dx = 0.0;
  pr::DevBuf<double> k, gx, gy, gz, diag, hot, cold;
  cudaStream_t last_stream = nullptr;
};
