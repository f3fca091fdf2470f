// fast_common.cuh -- building blocks of the colour-ordered (TAMC_MODE_FAST) kernels.
//
// Spin storage is bit-sliced across replicas: for every site a 32-bit word
// whose bit b is the spin of replica b of the word's group (1 = spin -1, the
// reference's packing convention, src/ising.rs:102-115).  A "quad" is 4
// adjacent bits; one task updates one site for the 4 replicas of a quad, with
// the 4 uniforms of one Philox-4x32-10 call keyed by (seed) and countered by
// (site, sweep, quad id, tag), so results do not depend on how tasks are
// spread over threads or CTAs.
#pragma once
#include "device.cuh"

namespace tamc {

struct FastInst {  // colour-ordered instance (device pointers)
  uint32_t n, nnz, ncolors;
  float offset;
  const uint32_t* color_off;  // ncolors + 1
  const uint32_t* perm;       // new -> original
  const uint32_t* iperm;      // original -> new
  const uint32_t* rp;         // n + 1
  const uint2* ent;           // nnz (new column, J bits)
  const uint16_t* col16;      // nnz new column as 16 bits, padded to 8 entries; null if n > 65536
  uint32_t udeg;              // entries per row if uniform (row s = [s*udeg, (s+1)*udeg)), else 0
  const float* bias;          // n
  const float* kd;            // n self-loop coefficient
  const double* sus;          // [nchi][n], colour order
  uint32_t nchi;
};

FastInst make_fast_inst(const tamc_inst* d);

// Local field of site s for the 4 replicas held in bits [shift, shift+4) of
// the words W[j * ws + wo]:  f_r = h_s + Σ_j J_sj s_j^r, summed in the
// reference's row order (src/ising.rs:471-475).
__device__ __forceinline__ float4 local_field4(uint32_t s, uint32_t shift, const uint32_t* __restrict__ rp,
                                               const uint2* __restrict__ ent, const float* __restrict__ bias,
                                               const uint32_t* W, uint32_t ws, uint32_t wo) {
  const uint32_t e0 = rp[s], e1 = rp[s + 1];
  const float h = bias[s];
  float4 f = make_float4(h, h, h, h);
  for (uint32_t e = e0; e < e1; ++e) {
    const uint2 c = ent[e];
    const uint32_t w = W[c.x * ws + wo] >> shift;
    f.x += __uint_as_float(c.y ^ (w << 31));
    f.y += __uint_as_float(c.y ^ ((w << 30) & 0x80000000u));
    f.z += __uint_as_float(c.y ^ ((w << 29) & 0x80000000u));
    f.w += __uint_as_float(c.y ^ ((w << 28) & 0x80000000u));
  }
  return f;
}

// The same with every row holding exactly DEG entries (row s starts at
// s*DEG): no row-pointer loads, and the loop unrolls.  Same sums, same order.
template <uint32_t DEG>
__device__ __forceinline__ float4 local_field4_deg(uint32_t s, uint32_t shift, const uint2* __restrict__ ent,
                                                   const float* __restrict__ bias, const uint32_t* W, uint32_t ws,
                                                   uint32_t wo) {
  const float h = bias[s];
  float4 f = make_float4(h, h, h, h);
#pragma unroll
  for (uint32_t k = 0; k < DEG; ++k) {
    const uint2 c = ent[s * DEG + k];
    const uint32_t w = W[c.x * ws + wo] >> shift;
    f.x += __uint_as_float(c.y ^ (w << 31));
    f.y += __uint_as_float(c.y ^ ((w << 30) & 0x80000000u));
    f.z += __uint_as_float(c.y ^ ((w << 29) & 0x80000000u));
    f.w += __uint_as_float(c.y ^ ((w << 28) & 0x80000000u));
  }
  return f;
}

// g_r = s_r f_r for the quad; the flip costs ΔE_r = -2 g_r (src/ising.rs:476-477).
__device__ __forceinline__ float4 spin_field4(float4 f, uint32_t own) {
  float4 g;
  g.x = __uint_as_float(__float_as_uint(f.x) ^ (own << 31));
  g.y = __uint_as_float(__float_as_uint(f.y) ^ ((own << 30) & 0x80000000u));
  g.z = __uint_as_float(__float_as_uint(f.z) ^ ((own << 29) & 0x80000000u));
  g.w = __uint_as_float(__float_as_uint(f.w) ^ ((own << 28) & 0x80000000u));
  return g;
}

// Metropolis rule: accept iff u < min(1, e^(-beta ΔE)) = min(1, 2^(b2 g)) with
// b2 = 2 beta log2(e) (TAMC_2LOG2E) and g = -ΔE/2.  u is a 23-bit uniform
// built by placing the random mantissa under the exponent of 1.0 (u + 1 in
// [1, 2)) and compared with p + 1.  ΔE <= 0 gives p + 1 >= 2 > u + 1, so it
// always accepts, as the reference's rule does, with no clamp.  b2 g is the
// same float as -(beta log2 e) ΔE: both are one rounding of the same product.
#define TAMC_2LOG2E 2.8853900817779268f
__device__ __forceinline__ float ex2_approx(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ bool accept_g(float g, float b2, uint32_t r) {
  const float p1 = ex2_approx(b2 * g) + 1.0f;
  return __uint_as_float(0x3f800000u | (r >> 9)) < p1;
}

// Energies are accumulated in 64-bit fixed point with 2^-32 resolution:
// integer addition is associative, so sums do not depend on how sites are
// spread over threads (CTA size, batching) and results are bit-reproducible.
#define TAMC_FX_SCALE 4294967296.0f
#define TAMC_FX_INV 2.3283064365386963e-10
__device__ __forceinline__ long long to_fx(float x) { return __float2ll_rn(x * TAMC_FX_SCALE); }
struct Fx4 {
  long long x, y, z, w;
};

// One quad update with inverse temperatures pre-scaled by 2 log2(e)
// (TAMC_2LOG2E).  Returns the 4-bit flip mask; with ACC, adds accepted ΔE to
// acc in fixed point.
template <bool ACC, uint32_t DEG = 0>
__device__ __forceinline__ uint32_t quad_update(uint32_t s, uint32_t shift, const FastInst& F, const uint32_t* W,
                                                uint32_t ws, uint32_t wo, float4 b2, uint4 rnd, Fx4& acc) {
  const float4 f = DEG ? local_field4_deg<DEG>(s, shift, F.ent, F.bias, W, ws, wo)
                       : local_field4(s, shift, F.rp, F.ent, F.bias, W, ws, wo);
  const uint32_t own = W[s * ws + wo] >> shift;
  const float4 g = spin_field4(f, own);
  const bool a0 = accept_g(g.x, b2.x, rnd.x);
  const bool a1 = accept_g(g.y, b2.y, rnd.y);
  const bool a2 = accept_g(g.z, b2.z, rnd.z);
  const bool a3 = accept_g(g.w, b2.w, rnd.w);
  if (ACC) {
    acc.x += to_fx(a0 ? -2.0f * g.x : 0.0f);
    acc.y += to_fx(a1 ? -2.0f * g.y : 0.0f);
    acc.z += to_fx(a2 ? -2.0f * g.z : 0.0f);
    acc.w += to_fx(a3 ? -2.0f * g.w : 0.0f);
  }
  return (uint32_t)a0 | ((uint32_t)a1 << 1) | ((uint32_t)a2 << 2) | ((uint32_t)a3 << 3);
}

// Per-replica energy contribution of site s for a quad:
//   e_r = s_r (h_s + Σ_j J_sj s_j^r / 2)   (energy_ref row term, src/ising.rs:441-449)
__device__ __forceinline__ float4 energy_terms4(uint32_t s, uint32_t shift, const FastInst& F, const uint32_t* W,
                                                uint32_t ws, uint32_t wo) {
  const uint32_t e0 = F.rp[s], e1 = F.rp[s + 1];
  const float h = F.bias[s];
  float4 f = make_float4(h, h, h, h);
  for (uint32_t e = e0; e < e1; ++e) {
    const uint2 c = F.ent[e];
    const uint32_t w = W[c.x * ws + wo] >> shift;
    const uint32_t hj = __float_as_uint(0.5f * __uint_as_float(c.y));
    f.x += __uint_as_float(hj ^ (w << 31));
    f.y += __uint_as_float(hj ^ ((w << 30) & 0x80000000u));
    f.z += __uint_as_float(hj ^ ((w << 29) & 0x80000000u));
    f.w += __uint_as_float(hj ^ ((w << 28) & 0x80000000u));
  }
  const uint32_t own = W[s * ws + wo] >> shift;
  float4 e;
  e.x = __uint_as_float(__float_as_uint(f.x) ^ (own << 31));
  e.y = __uint_as_float(__float_as_uint(f.y) ^ ((own << 30) & 0x80000000u));
  e.z = __uint_as_float(__float_as_uint(f.z) ^ ((own << 29) & 0x80000000u));
  e.w = __uint_as_float(__float_as_uint(f.w) ^ ((own << 28) & 0x80000000u));
  return e;
}

// 4 initial spins from one Philox call: spin = +1 iff the top bit is set
// (the same rule as rand_ising_state's Uniform(0,1), src/ising.rs:172).
__device__ __forceinline__ uint32_t init_nibble(uint4 r) {
  return (r.x >> 31 ^ 1u) | ((r.y >> 31 ^ 1u) << 1) | ((r.z >> 31 ^ 1u) << 2) | ((r.w >> 31 ^ 1u) << 3);
}

}  // namespace tamc
