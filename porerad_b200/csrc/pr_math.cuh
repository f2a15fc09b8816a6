// Exact-arithmetic helpers shared by the sm_100a kernels and the host-side
// self-tests: IEEE-754 binary64 operations with no contraction, double-double
// arithmetic, a near-correctly-rounded sin/cos for the ray-direction angle, and
// the 128-bit PCG64 (XSL-RR 128/64) generator that NumPy's PCG64 implements.
//
// Every function here compiles both as CUDA device code and as plain C++ on the
// host (g++ -ffp-contract=off), so the host tests exercise the very same code the
// kernels run.
#pragma once
#include <stdint.h>
#include <math.h>

#if defined(__CUDACC__)
#define PR_HD __host__ __device__ __forceinline__
#else
#define PR_HD static inline
#endif

// ---------------------------------------------------------------------------
// Binary64 primitives. On the device these are the round-to-nearest intrinsics,
// which the compiler never fuses into FMAs; on the host the file is compiled with
// -ffp-contract=off so the plain operators mean the same thing.
// ---------------------------------------------------------------------------
PR_HD double pr_add(double a, double b) {
#if defined(__CUDA_ARCH__)
  return __dadd_rn(a, b);
#else
  return a + b;
#endif
}
PR_HD double pr_sub(double a, double b) {
#if defined(__CUDA_ARCH__)
  return __dsub_rn(a, b);
#else
  return a - b;
#endif
}
PR_HD double pr_mul(double a, double b) {
#if defined(__CUDA_ARCH__)
  return __dmul_rn(a, b);
#else
  return a * b;
#endif
}
PR_HD double pr_div(double a, double b) {
#if defined(__CUDA_ARCH__)
  return __ddiv_rn(a, b);
#else
  return a / b;
#endif
}
PR_HD double pr_sqrt(double a) {
#if defined(__CUDA_ARCH__)
  return __dsqrt_rn(a);
#else
  return sqrt(a);
#endif
}
PR_HD double pr_fma(double a, double b, double c) {
#if defined(__CUDA_ARCH__)
  return __fma_rn(a, b, c);
#else
  return fma(a, b, c);
#endif
}

// NumPy's float64 remainder for a positive divisor: the sign of the result follows
// the divisor (Python semantics); fmod is exact, the correction is one rounded add.
PR_HD double pr_pymod_pos(double a, double b) {
  double m = fmod(a, b);
  if (m != 0.0) {
    if (m < 0.0) m = pr_add(m, b);
  } else {
    m = 0.0;  // +0.0, the sign of the divisor
  }
  return m;
}

// ---------------------------------------------------------------------------
// Double-double arithmetic (Dekker / Knuth error-free transforms, FMA products).
// ---------------------------------------------------------------------------
struct pr_dd {
  double hi, lo;
};

PR_HD pr_dd pr_two_sum(double a, double b) {
  double s = pr_add(a, b);
  double bb = pr_sub(s, a);
  double e = pr_add(pr_sub(a, pr_sub(s, bb)), pr_sub(b, bb));
  return {s, e};
}
PR_HD pr_dd pr_fast_two_sum(double a, double b) {  // requires |a| >= |b| or a == 0
  double s = pr_add(a, b);
  double e = pr_sub(b, pr_sub(s, a));
  return {s, e};
}
PR_HD pr_dd pr_two_prod(double a, double b) {
  double p = pr_mul(a, b);
  double e = pr_fma(a, b, -p);
  return {p, e};
}
PR_HD pr_dd pr_dd_mul(pr_dd a, pr_dd b) {
  pr_dd p = pr_two_prod(a.hi, b.hi);
  double e = pr_add(p.lo, pr_add(pr_mul(a.hi, b.lo), pr_mul(a.lo, b.hi)));
  return pr_fast_two_sum(p.hi, e);
}
PR_HD pr_dd pr_dd_mul_d(pr_dd a, double b) {
  pr_dd p = pr_two_prod(a.hi, b);
  double e = pr_fma(a.lo, b, p.lo);
  return pr_fast_two_sum(p.hi, e);
}
PR_HD pr_dd pr_dd_add(pr_dd a, pr_dd b) {
  pr_dd s = pr_two_sum(a.hi, b.hi);
  pr_dd t = pr_two_sum(a.lo, b.lo);
  double e = pr_add(s.lo, t.hi);
  s = pr_fast_two_sum(s.hi, e);
  e = pr_add(s.lo, t.lo);
  return pr_fast_two_sum(s.hi, e);
}

// ---------------------------------------------------------------------------
// sin and cos of x in [0, 2*pi] (the Lambertian azimuth 2*pi*u).
//
// Method: Cody-Waite reduction r = x - k*pi/2 with pi/2 split into a 33-bit, a
// 33-bit and a 53-bit part (k <= 4, so k*P1 and k*P2 are exact and x - k*P1 is
// exact by Sterbenz' lemma), carried as a double-double; then the Taylor series
// of sin and cos about 0 for |r| <= pi/4, with the low-order coefficients in
// double-double and the tail (relative size < 1e-6) in binary64 Horner form.
// The double-double result carries a relative error below about 2^-70, so its
// rounding to binary64 is the correctly rounded value except when the exact value
// lies within that distance of a rounding midpoint.
//
// The constants are the binary64 (or double-double) roundings of pi/2 pieces and
// of (-1)^n / n!, computed exactly with rational arithmetic.
// ---------------------------------------------------------------------------
#define PR_PIO2_1 0x1.921fb54400000p+0    // pi/2 truncated to 33 bits
#define PR_PIO2_2 0x1.0b4611a600000p-34   // next 33 bits
#define PR_PIO2_3 0x1.3198a2e037073p-69   // remainder rounded to 53 bits
#define PR_TWO_OVER_PI 0x1.45f306dc9c883p-1

PR_HD void pr_sincos_reduced(pr_dd r, double* s_out, double* c_out) {
  const pr_dd z = pr_dd_mul(r, r);
  const double zh = z.hi;
  // sin(r) = r + r*z*(s3 + z*(s5 + z*(s7 + z*T(z)))),  T(z) = s9 + s11 z + ... + s21 z^6
  double ts = 0x1.71b8ef6dcf572p-66;              // 1/21!
  ts = pr_fma(ts, zh, -0x1.2f49b46814157p-57);   // -1/19!
  ts = pr_fma(ts, zh, 0x1.952c77030ad4ap-49);    // 1/17!
  ts = pr_fma(ts, zh, -0x1.ae7f3e733b81fp-41);   // -1/15!
  ts = pr_fma(ts, zh, 0x1.6124613a86d09p-33);    // 1/13!
  ts = pr_fma(ts, zh, -0x1.ae64567f544e4p-26);   // -1/11!
  ts = pr_fma(ts, zh, 0x1.71de3a556c734p-19);    // 1/9!
  pr_dd qs = pr_dd_add(pr_dd{-0x1.a01a01a01a01ap-13, -0x1.a01a01a01a01ap-73}, pr_dd_mul_d(z, ts));  // s7
  qs = pr_dd_add(pr_dd{0x1.1111111111111p-7, 0x1.1111111111111p-63}, pr_dd_mul(z, qs));           // s5
  qs = pr_dd_add(pr_dd{-0x1.5555555555555p-3, -0x1.5555555555555p-57}, pr_dd_mul(z, qs));         // s3
  pr_dd sn = pr_dd_add(r, pr_dd_mul(pr_dd_mul(r, z), qs));
  // cos(r) = 1 + z*(-1/2 + z*(c4 + z*(c6 + z*(c8 + z*U(z))))),  U(z) = c10 + ... + c22 z^6
  double tc = -0x1.0ce396db7f853p-70;             // -1/22!
  tc = pr_fma(tc, zh, 0x1.e542ba4020225p-62);    // 1/20!
  tc = pr_fma(tc, zh, -0x1.6827863b97d97p-53);   // -1/18!
  tc = pr_fma(tc, zh, 0x1.ae7f3e733b81fp-45);    // 1/16!
  tc = pr_fma(tc, zh, -0x1.93974a8c07c9dp-37);   // -1/14!
  tc = pr_fma(tc, zh, 0x1.1eed8eff8d898p-29);    // 1/12!
  tc = pr_fma(tc, zh, -0x1.27e4fb7789f5cp-22);   // -1/10!
  pr_dd qc = pr_dd_add(pr_dd{0x1.a01a01a01a01ap-16, 0x1.a01a01a01a01ap-76}, pr_dd_mul_d(z, tc));  // c8
  qc = pr_dd_add(pr_dd{-0x1.6c16c16c16c17p-10, 0x1.f49f49f49f49fp-65}, pr_dd_mul(z, qc));         // c6
  qc = pr_dd_add(pr_dd{0x1.5555555555555p-5, 0x1.5555555555555p-59}, pr_dd_mul(z, qc));           // c4
  qc = pr_dd_add(pr_dd{-0.5, 0.0}, pr_dd_mul(z, qc));
  pr_dd cs = pr_dd_add(pr_dd{1.0, 0.0}, pr_dd_mul(z, qc));
  *s_out = sn.hi;
  *c_out = cs.hi;
}

PR_HD void pr_sincos(double x, double* s_out, double* c_out) {
  const double kd = rint(pr_mul(x, PR_TWO_OVER_PI));
  const int k = (int)kd;
  // r = x - k*(P1 + P2 + P3) as a double-double
  const double r1 = pr_sub(x, pr_mul(kd, PR_PIO2_1));  // exact
  pr_dd r = pr_two_sum(r1, -pr_mul(kd, PR_PIO2_2));     // k*P2 exact
  r = pr_fast_two_sum(r.hi, pr_sub(r.lo, pr_mul(kd, PR_PIO2_3)));
  double s, c;
  pr_sincos_reduced(r, &s, &c);
  switch (k & 3) {
    case 0: *s_out = s; *c_out = c; break;
    case 1: *s_out = c; *c_out = -s; break;
    case 2: *s_out = -s; *c_out = -c; break;
    default: *s_out = -c; *c_out = s; break;
  }
}

// ---------------------------------------------------------------------------
// PCG64 (PCG XSL-RR 128/64, the generator behind numpy.random.PCG64):
//   state <- state * M + inc (mod 2^128), then output = rotr64(hi ^ lo, hi >> 58).
// A jump of n steps is the affine map state <- A_n state + C_n; the host supplies
// the maps for n = 2^0 .. 2^63 of a given stream.
// ---------------------------------------------------------------------------
struct pr_u128 {
  uint64_t lo, hi;
};

PR_HD uint64_t pr_umulhi64(uint64_t a, uint64_t b) {
#if defined(__CUDA_ARCH__)
  return __umul64hi(a, b);
#else
  return (uint64_t)(((unsigned __int128)a * (unsigned __int128)b) >> 64);
#endif
}
PR_HD pr_u128 pr_u128_mul(pr_u128 a, pr_u128 b) {  // low 128 bits of a*b
  pr_u128 r;
  r.lo = a.lo * b.lo;
  r.hi = pr_umulhi64(a.lo, b.lo) + a.hi * b.lo + a.lo * b.hi;
  return r;
}
PR_HD pr_u128 pr_u128_add(pr_u128 a, pr_u128 b) {
  pr_u128 r;
  r.lo = a.lo + b.lo;
  r.hi = a.hi + b.hi + (r.lo < a.lo ? 1u : 0u);
  return r;
}
PR_HD pr_u128 pr_u128_affine(pr_u128 mul, pr_u128 add, pr_u128 s) {
  return pr_u128_add(pr_u128_mul(mul, s), add);
}

#define PR_PCG_MULT_HI 0x2360ED051FC65DA4ull
#define PR_PCG_MULT_LO 0x4385DF649FCCF645ull

PR_HD uint64_t pr_pcg_output(pr_u128 s) {
  const uint64_t v = s.hi ^ s.lo;
  const unsigned rot = (unsigned)(s.hi >> 58);
  return (v >> rot) | (v << ((64u - rot) & 63u));
}

// One PCG64 draw mapped to [0, 1) the way numpy.random.Generator.random does:
// the top 53 bits times 2^-53.
PR_HD double pr_pcg_next_double(pr_u128* s, pr_u128 inc) {
  const pr_u128 m = {PR_PCG_MULT_LO, PR_PCG_MULT_HI};
  *s = pr_u128_affine(m, inc, *s);
  return (double)(pr_pcg_output(*s) >> 11) * 0x1.0p-53;
}

// Jump a stream ahead by n steps using the power-of-two maps table[2*i] = A_{2^i},
// table[2*i + 1] = C_{2^i}.
PR_HD pr_u128 pr_pcg_jump(pr_u128 s, uint64_t n, const pr_u128* table) {
  int i = 0;
  while (n) {
    if (n & 1u) s = pr_u128_affine(table[2 * i], table[2 * i + 1], s);
    n >>= 1;
    ++i;
  }
  return s;
}
