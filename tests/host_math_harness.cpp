// Host build of porerad_b200/csrc/pr_math.cuh for the CPU tests (g++ -ffp-contract=off).
#include "../porerad_b200/csrc/pr_math.cuh"

extern "C" {

// count draws of one PCG64 stream after jumping n steps, mapped to [0, 1).
void hm_pcg_doubles(uint64_t state_hi, uint64_t state_lo, uint64_t inc_hi, uint64_t inc_lo, uint64_t jump,
                    const uint64_t* maps /* 64 x (A_lo, A_hi, C_lo, C_hi) */, int count, double* out) {
  pr_u128 table[128];
  for (int i = 0; i < 64; ++i) {
    table[2 * i] = pr_u128{maps[4 * i], maps[4 * i + 1]};
    table[2 * i + 1] = pr_u128{maps[4 * i + 2], maps[4 * i + 3]};
  }
  pr_u128 s = pr_pcg_jump(pr_u128{state_lo, state_hi}, jump, table);
  const pr_u128 inc{inc_lo, inc_hi};
  for (int k = 0; k < count; ++k) out[k] = pr_pcg_next_double(&s, inc);
}

void hm_sincos(const double* x, long n, double* s, double* c) {
  for (long i = 0; i < n; ++i) pr_sincos(x[i], s + i, c + i);
}

void hm_pymod(const double* a, long n, double b, double* out) {
  for (long i = 0; i < n; ++i) out[i] = pr_pymod_pos(a[i], b);
}
}
