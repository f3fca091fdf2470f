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
  int pmj;                    // +-1 couplings, zero field, no self-loop, udeg 4 or 6 (multi-spin coding)
  uint32_t lat_L;             // side of a periodic square / cubic lattice in file order (16 or 32), else 0
  const float* fJt;           // lattice instances: couplings [udeg][n] (entry m of colour row s at m n + s)
  const uint16_t* fcolt;      // lattice instances: columns [udeg][n], same layout
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
// The decision of quad_update from the local field f and the quad's own spins.
template <bool ACC>
__device__ __forceinline__ uint32_t quad_accept(float4 f, uint32_t own, float4 b2, uint4 rnd, Fx4& acc) {
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

template <uint32_t DEG>
__device__ __forceinline__ float4 quad_field(uint32_t s, uint32_t shift, const FastInst& F, const uint32_t* W,
                                             uint32_t ws, uint32_t wo) {
  return DEG ? local_field4_deg<DEG>(s, shift, F.ent, F.bias, W, ws, wo)
             : local_field4(s, shift, F.rp, F.ent, F.bias, W, ws, wo);
}

template <bool ACC, uint32_t DEG = 0>
__device__ __forceinline__ uint32_t quad_update(uint32_t s, uint32_t shift, const FastInst& F, const uint32_t* W,
                                                uint32_t ws, uint32_t wo, float4 b2, uint4 rnd, Fx4& acc) {
  const float4 f = quad_field<DEG>(s, shift, F, W, ws, wo);
  return quad_accept<ACC>(f, W[s * ws + wo] >> shift, b2, rnd, acc);
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

// 32x32 bit transpose across a warp: lane L passes row L (bit c = column c)
// and gets column L (bit r = row r's bit L).  Five butterfly steps; at step j
// the lanes L and L^j swap the off-diagonal j x j blocks of their 2j x 2j tile.
__device__ __forceinline__ uint32_t transpose32(uint32_t x, uint32_t lane) {
  uint32_t m = 0x0000ffffu;
#pragma unroll
  for (uint32_t j = 16; j != 0; j >>= 1, m ^= m << j) {
    const uint32_t y = __shfl_xor_sync(0xffffffffu, x, j);
    x = (lane & j) ? ((x & ~m) | ((y & ~m) >> j)) : ((x & m) | ((y & m) << j));
  }
  return x;
}

// ------------------------------------------------- multi-spin coding ----
// For +-J instances (every J = +-1, no field, rows of DEG = 4 or 6 entries) a
// site update acts on the 32 replicas of one word at once.  Bond (s, j) is
// unsatisfied in replica r (it adds +1 to the energy) when J s_s s_j = +1;
// with the bit convention (1 = spin -1) that is bit r of
// ~(W_s ^ W_j ^ neg_J).  With x unsatisfied bonds the flip costs
// dE = 2 (DEG - 2 x): x >= DEG / 2 always flips, x < DEG / 2 flips with
// probability exp(-beta dE).  That probability, for the replica's beta and
// level x, is held as a 32-bit threshold T = floor(p 2^32), stored bit-plane
// by bit-plane (plane k: bit r = bit k of replica r's T); a uniform 32-bit
// u < T decides, compared from the top bit down against random words, one
// bit of u per word for all undecided replicas at once, so a word costs a few
// random words instead of 32 uniforms.  u is uniform, so each replica flips
// with probability T / 2^32 (within 2^-32 of p).
//   planes: MscPlanes of the word (levels 0 .. DEG/2 - 1)
struct MscLevels {
  uint32_t lv[3];  // replicas at level x = 0, 1, 2 (x < DEG/2 only)
  uint32_t p0, p1, p2;  // bit planes of x
};

template <uint32_t DEG>
__device__ __forceinline__ MscLevels msc_levels(uint32_t S0, const uint32_t* Wj, uint32_t negmask) {
  uint32_t p0 = 0, p1 = 0, p2 = 0;
#pragma unroll
  for (uint32_t m = 0; m < DEG; ++m) {
    const uint32_t u = ~(S0 ^ Wj[m] ^ (0u - ((negmask >> m) & 1u)));
    const uint32_t c0 = p0 & u;
    p0 ^= u;
    const uint32_t c1 = p1 & c0;
    p1 ^= c0;
    p2 ^= c1;
  }
  MscLevels L;
  L.p0 = p0;
  L.p1 = p1;
  L.p2 = p2;
  const uint32_t z = ~(p0 | p1 | p2);
  L.lv[0] = z;                      // x = 0
  L.lv[1] = p0 & ~p1 & ~p2;         // x = 1
  L.lv[2] = DEG == 6 ? (~p0 & p1 & ~p2) : 0u;  // x = 2 (uphill only for DEG 6)
  return L;
}

// Four comparison levels k = 4 kk .. 4 kk + 3 of one word: level k compares
// random word k (component k % 4 of Philox call kk) with threshold plane
// 31 - k.  The four planes of a level group are one aligned 16-byte load
// (planes 28 - 4 kk .. 31 - 4 kk; `pl` 16-byte aligned).
template <uint32_t DEG>
__device__ __forceinline__ void msc_step4(uint4 r, const uint32_t* pl, const MscLevels& L, uint32_t kk, uint32_t& und,
                                          uint32_t& lt) {
  constexpr uint32_t LV = DEG / 2;
  uint32_t t0 = 0, t1 = 0, t2 = 0, t3 = 0;
#pragma unroll
  for (uint32_t l = 0; l < LV; ++l) {
    const uint4 P = *reinterpret_cast<const uint4*>(pl + l * 32 + 28 - 4 * kk);
    t0 |= P.w & L.lv[l];
    t1 |= P.z & L.lv[l];
    t2 |= P.y & L.lv[l];
    t3 |= P.x & L.lv[l];
  }
  lt |= und & ~r.x & t0;
  und &= ~(r.x ^ t0);
  lt |= und & ~r.y & t1;
  und &= ~(r.y ^ t1);
  lt |= und & ~r.z & t2;
  und &= ~(r.z ^ t2);
  lt |= und & ~r.w & t3;
  und &= ~(r.w ^ t3);
}

// The flip mask of one word: `pl` = threshold planes [DEG/2][32] of the word,
// `al` / `nv` = replicas whose level always / never flips ([DEG/2]); random
// words from Philox keyed by `key` and counted by (s, i, (wo << 8) | call).
// Levels run in groups of four (one Philox call each) until no replica is
// undecided; a replica decided within a group is untouched by its remaining
// levels, so the result is the one of a level-by-level loop.
template <uint32_t DEG>
__device__ __forceinline__ uint32_t msc_flip(const MscLevels& L, const uint32_t* pl, const uint32_t* al,
                                             const uint32_t* nv, uint32_t s, uint32_t i, uint32_t wo, uint2 key) {
  constexpr uint32_t LV = DEG / 2;
  uint32_t uphill = 0, always = 0, und = 0;
#pragma unroll
  for (uint32_t l = 0; l < LV; ++l) {
    uphill |= L.lv[l];
    always |= L.lv[l] & al[l];
    und |= L.lv[l] & ~al[l] & ~nv[l];
  }
  uint32_t lt = 0;
  for (uint32_t kk = 0; kk < 8 && und; ++kk)
    msc_step4<DEG>(philox4x32_10w(make_uint4(s, i, (wo << 8) | kk, PTAG_MSC), key), pl, L, kk, und, lt);
  return ~uphill | always | lt;
}

// msc_flip for two words of the same site at once (words wo and wo + 1, each
// with its own planes and random words): the same decisions, with both Philox
// calls of a level group issued together so that their rounds overlap.
template <uint32_t DEG>
__device__ __forceinline__ void msc_flip2(const MscLevels& L0, const MscLevels& L1, const uint32_t* pl0,
                                          const uint32_t* pl1, uint32_t s, uint32_t i, uint32_t wo, uint2 key,
                                          uint32_t& f0, uint32_t& f1) {
  constexpr uint32_t LV = DEG / 2;
  const uint32_t *al0 = pl0 + 96, *nv0 = pl0 + 99, *al1 = pl1 + 96, *nv1 = pl1 + 99;
  uint32_t up0 = 0, alw0 = 0, und0 = 0, up1 = 0, alw1 = 0, und1 = 0;
#pragma unroll
  for (uint32_t l = 0; l < LV; ++l) {
    up0 |= L0.lv[l];
    alw0 |= L0.lv[l] & al0[l];
    und0 |= L0.lv[l] & ~al0[l] & ~nv0[l];
    up1 |= L1.lv[l];
    alw1 |= L1.lv[l] & al1[l];
    und1 |= L1.lv[l] & ~al1[l] & ~nv1[l];
  }
  uint32_t lt0 = 0, lt1 = 0;
  for (uint32_t kk = 0; kk < 8 && (und0 | und1); ++kk) {
    const uint4 r0 = philox4x32_10w(make_uint4(s, i, (wo << 8) | kk, PTAG_MSC), key);
    const uint4 r1 = philox4x32_10w(make_uint4(s, i, ((wo + 1) << 8) | kk, PTAG_MSC), key);
    msc_step4<DEG>(r0, pl0, L0, kk, und0, lt0);
    msc_step4<DEG>(r1, pl1, L1, kk, und1, lt1);
  }
  f0 = ~up0 | alw0 | lt0;
  f1 = ~up1 | alw1 | lt1;
}

// Threshold planes of replica word `wo` for inverse temperatures beta[r]:
// called by the 32 lanes of one warp, lane r for replica r of the word.
template <uint32_t DEG>
__device__ __forceinline__ void msc_planes(float beta, uint32_t lane, uint32_t* pl, uint32_t* al, uint32_t* nv) {
  constexpr uint32_t LV = DEG / 2;
#pragma unroll
  for (uint32_t l = 0; l < LV; ++l) {
    const double p = exp(-(double)beta * (double)(2 * ((int)DEG - 2 * (int)l)));
    const bool a = !(p < 1.0);
    const uint32_t T = a ? 0xffffffffu : (uint32_t)(p * 4294967296.0);
    const uint32_t ab = __ballot_sync(0xffffffffu, a), zb = __ballot_sync(0xffffffffu, !a && T == 0);
    for (uint32_t k = 0; k < 32; ++k) {
      const uint32_t b = __ballot_sync(0xffffffffu, (T >> k) & 1u);
      if (lane == 0) pl[l * 32 + k] = b;
    }
    if (lane == 0) {
      al[l] = ab;
      nv[l] = zb;
    }
  }
}

// Per-replica energy change of one word's flips, summed over the 32 lanes (32
// sites of the same word): lane r receives the fixed-point sum for replica r.
// dE = 2 (DEG - 2 x) per flip, so the sum is 2 DEG n_flip - 4 (n0 + 2 n1 + 4 n2)
// with n_k the flips with bit k of x set.
template <uint32_t DEG>
__device__ __forceinline__ long long msc_energy(uint32_t flip, const MscLevels& L, uint32_t lane) {
  const int nf = __popc(transpose32(flip, lane));
  const int n0 = __popc(transpose32(flip & L.p0, lane));
  const int n1 = __popc(transpose32(flip & L.p1, lane));
  const int n2 = __popc(transpose32(flip & L.p2, lane));
  const long long units = 2ll * DEG * nf - 4ll * (n0 + 2 * n1 + 4 * n2);
  return units * 4294967296ll;  // to_fx of the integer energy change
}

}  // namespace tamc
