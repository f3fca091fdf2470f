// expf_exact.h -- an expf that returns, for every float argument, the same bits
// as glibc 2.39's expf, on the host and on the device.
//
// Why: the reference computes Metropolis and replica-exchange acceptance as
// `x < f32::exp(a)` (tamc-core/src/metropolis.rs:50-52, tamc-core/src/pt.rs:136,
// tamc-core/src/parallel/pt.rs:54), and Rust's f32::exp is libm's expf.  A
// bit-exact replay of the reference's Markov chain must therefore reproduce
// glibc's rounding, including the ~1e-4 fraction of arguments where glibc's
// expf is not correctly rounded.
//
// How: `expf_core` evaluates e^x in double precision from the mathematics
// alone -- x = k ln2 + r with a two-part ln2 (hi has 39 significant bits so
// k*hi is exact), then the degree-13 Taylor polynomial of e^r (|r| <= ln2/2,
// truncation < 5e-18) in Horner form, then the exact 2^k scaling -- and rounds
// the result to float once.  Every operation is an explicitly rounded IEEE
// double add/mul (no contraction), so host and device produce identical bits.
// Where the result differs from glibc, an exception table (generated at build
// time by exhaustively comparing expf_core with the host's glibc expf over all
// float arguments in [-110, 89]; see gen_expf_table.c) supplies glibc's value.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define TAMC_HD __host__ __device__ __forceinline__
#else
#define TAMC_HD static inline
#endif

#if defined(__CUDA_ARCH__)
#define TAMC_DADD(a, b) __dadd_rn((a), (b))
#define TAMC_DMUL(a, b) __dmul_rn((a), (b))
#define TAMC_RINT(a) rint(a)
#else
#include <math.h>
#include <string.h>
// Host callers compile with -ffp-contract=off, so these are separately rounded.
#define TAMC_DADD(a, b) ((a) + (b))
#define TAMC_DMUL(a, b) ((a) * (b))
#define TAMC_RINT(a) rint(a)
#endif

TAMC_HD uint32_t tamc_f2u(float f) {
#if defined(__CUDA_ARCH__)
  return __float_as_uint(f);
#else
  uint32_t u;
  memcpy(&u, &f, 4);
  return u;
#endif
}
TAMC_HD float tamc_u2f(uint32_t u) {
#if defined(__CUDA_ARCH__)
  return __uint_as_float(u);
#else
  float f;
  memcpy(&f, &u, 4);
  return f;
#endif
}
TAMC_HD double tamc_pow2(int k) {  // exact 2^k for -1022 <= k <= 1023
  const uint64_t b = (uint64_t)(k + 1023) << 52;
#if defined(__CUDA_ARCH__)
  return __longlong_as_double((long long)b);
#else
  double d;
  memcpy(&d, &b, 8);
  return d;
#endif
}

// e^x rounded once to float.  Valid for every float; NaN propagates.
TAMC_HD float tamc_expf_core(float xf) {
  if (xf != xf) return xf;
  if (xf > 89.0f) return tamc_u2f(0x7f800000u);
  if (xf < -110.0f) return 0.0f;
  const double x = (double)xf;
  const double LOG2E = 0x1.71547652b82fep+0;
  const double LN2_HI = 0x1.62e42fefa0000p-1;   // ln2 with 39 significant bits
  const double LN2_LO = 0x1.cf79abc9e3b3ap-40;   // ln2 - LN2_HI
  const double kd = TAMC_RINT(TAMC_DMUL(x, LOG2E));
  const int k = (int)kd;
  const double r = TAMC_DADD(TAMC_DADD(x, TAMC_DMUL(-kd, LN2_HI)), TAMC_DMUL(-kd, LN2_LO));
  // Horner evaluation of sum_{n=0}^{13} r^n / n!
  double p = 0x1.6124613a86d09p-33;
  p = TAMC_DADD(TAMC_DMUL(p, r), 0x1.1eed8eff8d898p-29);
  p = TAMC_DADD(TAMC_DMUL(p, r), 0x1.ae64567f544e4p-26);
  p = TAMC_DADD(TAMC_DMUL(p, r), 0x1.27e4fb7789f5cp-22);
  p = TAMC_DADD(TAMC_DMUL(p, r), 0x1.71de3a556c734p-19);
  p = TAMC_DADD(TAMC_DMUL(p, r), 0x1.a01a01a01a01ap-16);
  p = TAMC_DADD(TAMC_DMUL(p, r), 0x1.a01a01a01a01ap-13);
  p = TAMC_DADD(TAMC_DMUL(p, r), 0x1.6c16c16c16c17p-10);
  p = TAMC_DADD(TAMC_DMUL(p, r), 0x1.1111111111111p-7);
  p = TAMC_DADD(TAMC_DMUL(p, r), 0x1.5555555555555p-5);
  p = TAMC_DADD(TAMC_DMUL(p, r), 0x1.5555555555555p-3);
  p = TAMC_DADD(TAMC_DMUL(p, r), 0x1.0000000000000p-1);
  p = TAMC_DADD(TAMC_DMUL(p, r), 1.0);
  p = TAMC_DADD(TAMC_DMUL(p, r), 1.0);
  return (float)TAMC_DMUL(p, tamc_pow2(k));
}

// Exception table layout (device or host arrays):
//   bucket b covers argument bit patterns [b << 12, (b+1) << 12) after
//   mapping: idx = bits >> 12 for non-negative floats, (bits - 0x80000000) >> 12
//   + TAMC_EXPF_NEG_BUCKET0 for negative floats.  off[b]..off[b+1] index the
//   sorted (key, value) pairs of that bucket.
#define TAMC_EXPF_POS_MAX_BITS 0x42B20000u   /* 89.0f */
#define TAMC_EXPF_NEG_MAX_BITS 0xC2DC0000u   /* -110.0f */
#define TAMC_EXPF_POS_BUCKETS ((TAMC_EXPF_POS_MAX_BITS >> 12) + 1u)
#define TAMC_EXPF_NEG_BUCKET0 TAMC_EXPF_POS_BUCKETS
#define TAMC_EXPF_NUM_BUCKETS (TAMC_EXPF_POS_BUCKETS + (((TAMC_EXPF_NEG_MAX_BITS - 0x80000000u) >> 12) + 1u))

TAMC_HD int tamc_expf_bucket(uint32_t bits, uint32_t* b) {
  if (bits <= TAMC_EXPF_POS_MAX_BITS) { *b = bits >> 12; return 1; }
  if (bits >= 0x80000000u && bits <= TAMC_EXPF_NEG_MAX_BITS) {
    *b = TAMC_EXPF_NEG_BUCKET0 + ((bits - 0x80000000u) >> 12);
    return 1;
  }
  return 0;
}

// glibc-identical expf given the exception table (off: TAMC_EXPF_NUM_BUCKETS+1
// offsets; keys/vals: argument and glibc result bit patterns).
TAMC_HD float tamc_expf_exact(float x, const uint32_t* off, const uint32_t* keys, const uint32_t* vals) {
  const float r = tamc_expf_core(x);
  const uint32_t bits = tamc_f2u(x);
  uint32_t b;
  if (tamc_expf_bucket(bits, &b)) {
    const uint32_t e1 = off[b + 1];
    for (uint32_t i = off[b]; i < e1; ++i)
      if (keys[i] == bits) return tamc_u2f(vals[i]);
  }
  return r;
}
