// fast_pt.cu -- the fused PT-ICM round kernel (TAMC_MODE_FAST).
//
// One CTA runs whole PT rounds of one job (an instance with its replica
// ladder) with the replica state resident in shared memory; CTAs pull jobs
// from a device work queue (longest first), so one launch serves a single
// instance or a batch of uneven instances alike.  Per round, in the reference's
// order (parallel_pt_loop, src/pt.rs:446-450):
//
//  1. Houdayer ICM (src/pt.rs:31-77) for every chain pair and every slot >= lo
//     at once: with the slot-major layout, D = W[c0] ^ W[c1] has bit t set
//     where the two replicas at slot t disagree.  Per slot a warp counts the
//     q<0 sites, draws the seed index from Philox and finds the seed site;
//     the clusters of all 32 slots of a word then grow together by
//     bit-parallel label propagation  Cl[s] |= D[s] & OR_{j~s} Cl[j]  to a
//     fixed point (the connected q<0 component of each seed), and the move
//     flips Cl in both chains.  Energies change by the cluster boundary terms.
//  2. Replica exchange along each chain (warp per chain): decisions with
//     threaded (stale ΔE, tamc-core/src/parallel/pt.rs:41-59) or serial
//     (propagated ΔE, tamc-core/src/pt.rs:120-150) semantics; the composed
//     adjacent swaps are one bit permutation per chain word, applied to every
//     site with a carry trick:
//        new = ((v>>1)&D) | (((v&S)+D)&E) | (v&~(D|D<<1)),
//     S = run starts, E = run ends + 1 of the accepted-swap mask D.
//  3. One Metropolis sweep of all replicas in colour order (see fast_common.cuh).
//  4. Ground-state tracking and, on the reference's schedule, e/q/suscept
//     measurements and bit-packed state snapshots (src/pt.rs:167-226, 542-583).
#include "fast_pt.cuh"

namespace tamc {
namespace {

__device__ __forceinline__ uint64_t bitperm(uint64_t v, uint64_t D) {
  const uint64_t S = D & ~(D << 1);
  const uint64_t E = (D << 1) & ~D;
  return ((v >> 1) & D) | (((v & S) + D) & E) | (v & ~(D | (D << 1)));
}

__device__ __forceinline__ float u24(uint32_t r) { return (float)(r >> 8) * (1.0f / 16777216.0f); }

struct Smem {
  uint32_t* W;
  uint32_t* D;
  uint32_t* Cl;
  double* Ec;
  double* Er;
  float4* beta4;
  float4* red;
  float4* redq;
  uint32_t* nneg;
  double* dE0;
  double* dE1;
  unsigned long long* Dm;
  uint32_t* rp;
  float* bias;
  uint2* ent;
};

__host__ __device__ inline size_t al16(size_t x) { return (x + 15) & ~(size_t)15; }

__host__ __device__ inline size_t carve_all(Smem* S, char* base, uint32_t n, uint32_t nw, uint32_t C, uint32_t ntp,
                                            uint32_t qps, uint32_t T, uint32_t nnz, bool csr) {
  size_t o = 0;
  auto take = [&](size_t bytes) {
    char* p = base + o;
    o = al16(o + bytes);
    return p;
  };
  char* W = take((size_t)n * nw * 4);
  char* D = take((size_t)n * 4);
  char* Cl = take((size_t)n * 4);
  char* Ec = take((size_t)C * ntp * 8);
  char* Er = take((size_t)C * ntp * 8);
  char* b4 = take((size_t)qps * 16);
  char* red = take((size_t)T * 16);
  char* redq = take((size_t)T * 16);
  char* nneg = take(32 * 4);
  char* dE0 = take(32 * 8);
  char* dE1 = take(32 * 8);
  char* Dm = take((size_t)C * 8);
  char* rp = nullptr;
  char* bias = nullptr;
  char* ent = nullptr;
  if (csr) {
    rp = take((size_t)(n + 1) * 4);
    bias = take((size_t)n * 4);
    ent = take((size_t)nnz * 8);
  }
  if (S) {
    S->W = (uint32_t*)W;
    S->D = (uint32_t*)D;
    S->Cl = (uint32_t*)Cl;
    S->Ec = (double*)Ec;
    S->Er = (double*)Er;
    S->beta4 = (float4*)b4;
    S->red = (float4*)red;
    S->redq = (float4*)redq;
    S->nneg = (uint32_t*)nneg;
    S->dE0 = (double*)dE0;
    S->dE1 = (double*)dE1;
    S->Dm = (unsigned long long*)Dm;
    S->rp = (uint32_t*)rp;
    S->bias = (float*)bias;
    S->ent = (uint2*)ent;
  }
  return o;
}

// Energies of all slots from scratch (energy_ref semantics, f32 row terms
// summed in f64): Ec = Er = offset + Σ_s e_s.
__device__ void full_energies(const PtJob& J, const FastInst& F, Smem& S, uint32_t Teff) {
  const uint32_t tid = threadIdx.x;
  const uint32_t k = tid % J.qps;
  const uint32_t ch = k / J.qpc, q = k % J.qpc;
  const uint32_t wo = ch * J.wpc + (q >> 3), shift = 4 * (q & 7u);
  long long a0 = 0, a1 = 0, a2 = 0, a3 = 0;
  if (tid < Teff) {
    for (uint32_t s = tid / J.qps; s < J.n; s += Teff / J.qps) {
      const float4 e = energy_terms4(s, shift, F, S.W, J.nw, wo);
      a0 += to_fx(e.x);
      a1 += to_fx(e.y);
      a2 += to_fx(e.z);
      a3 += to_fx(e.w);
    }
  }
  long long* redd = reinterpret_cast<long long*>(S.red);  // red and redq are contiguous: 2*T*16 bytes
  __syncthreads();
  if (tid < Teff) {
    redd[tid * 4 + 0] = a0;
    redd[tid * 4 + 1] = a1;
    redd[tid * 4 + 2] = a2;
    redd[tid * 4 + 3] = a3;
  }
  __syncthreads();
  for (uint32_t x = tid; x < J.C * J.ntp; x += blockDim.x) {
    const uint32_t c = x / J.ntp, t = x % J.ntp;
    const uint32_t kk = c * J.qpc + t / 4;
    long long sum = 0;
    for (uint32_t th = kk; th < Teff; th += J.qps) sum += redd[th * 4 + (t & 3u)];
    S.Ec[x] = (double)J.F.offset + (double)sum * TAMC_FX_INV;
    S.Er[x] = S.Ec[x];
  }
  __syncthreads();
}

__device__ void icm_phase(const PtJob& J, const FastInst& F, Smem& S, uint32_t i) {
  const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5, nwarp = blockDim.x >> 5;
  const uint32_t n = J.n;
  for (uint32_t p = 0; 2 * p + 1 < J.C; ++p) {
    const uint32_t c0 = 2 * p, c1 = 2 * p + 1;
    for (uint32_t w = 0; w < J.wpc; ++w) {
      const uint32_t tb = 32 * w;
      uint32_t lomask = 0;
      for (uint32_t b = 0; b < 32; ++b)
        if (tb + b >= J.lo && tb + b < J.nt) lomask |= 1u << b;
      if (!lomask) continue;
      const uint32_t o0 = c0 * J.wpc + w, o1 = c1 * J.wpc + w;
      for (uint32_t s = tid; s < n; s += blockDim.x) {
        S.D[s] = (S.W[s * J.nw + o0] ^ S.W[s * J.nw + o1]) & lomask;
        S.Cl[s] = 0;
      }
      if (tid < 32) S.nneg[tid] = 0;
      __syncthreads();
      // count the q<0 sites per slot, draw the seed index, locate the seed
      for (uint32_t b = warp; b < 32; b += nwarp) {
        if (!((lomask >> b) & 1u)) continue;
        uint32_t cnt = 0;
        for (uint32_t base = 0; base < n; base += 32) {
          const uint32_t s = base + lane;
          cnt += __popc(__ballot_sync(0xffffffffu, s < n && ((S.D[s] >> b) & 1u)));
        }
        if (cnt == 0) continue;
        const uint32_t u = philox4x32_10(make_uint4(tb + b, i, p, PTAG_ICM), J.key).x;
        uint32_t k = (uint32_t)(((uint64_t)u * cnt) >> 32);
        for (uint32_t base = 0; base < n; base += 32) {
          const uint32_t s = base + lane;
          const uint32_t bal = __ballot_sync(0xffffffffu, s < n && ((S.D[s] >> b) & 1u));
          const uint32_t c = __popc(bal);
          if (k < c) {
            const uint32_t pos = __fns(bal, 0, (int)k + 1);
            if (lane == 0) {
              atomicOr(&S.Cl[base + pos], 1u << b);
              S.nneg[b] = cnt;
            }
            break;
          }
          k -= c;
        }
      }
      __syncthreads();
      // grow all clusters of this word to their fixed point
      for (;;) {
        int changed = 0;
        for (uint32_t s = tid; s < n; s += blockDim.x) {
          const uint32_t d = S.D[s];
          if (!d) continue;
          const uint32_t c = S.Cl[s];
          const uint32_t rem = d & ~c;
          if (!rem) continue;
          uint32_t nb = 0;
          const uint32_t e1 = F.rp[s + 1];
          for (uint32_t e = F.rp[s]; e < e1; ++e) {
            const uint32_t j = F.ent[e].x;
            if (j != s) nb |= S.Cl[j];
          }
          const uint32_t add = rem & nb;
          if (add) {
            S.Cl[s] = c | add;
            changed = 1;
          }
        }
        if (!__syncthreads_or(changed)) break;
      }
      // energy change of flipping each cluster in both replicas (true Hamiltonian)
      for (uint32_t b = warp; b < 32; b += nwarp) {
        if (!S.nneg[b]) continue;
        double a0 = 0, a1 = 0;
        for (uint32_t s = lane; s < n; s += 32) {
          if (!((S.Cl[s] >> b) & 1u)) continue;
          const float h = F.bias[s];
          float f0 = h, f1 = h;
          const uint32_t e1 = F.rp[s + 1];
          for (uint32_t e = F.rp[s]; e < e1; ++e) {
            const uint2 ce = F.ent[e];
            if (ce.x == s || ((S.Cl[ce.x] >> b) & 1u)) continue;
            const float Jv = __uint_as_float(ce.y);
            f0 += ((S.W[ce.x * J.nw + o0] >> b) & 1u) ? -Jv : Jv;
            f1 += ((S.W[ce.x * J.nw + o1] >> b) & 1u) ? -Jv : Jv;
          }
          const float s0 = ((S.W[s * J.nw + o0] >> b) & 1u) ? -1.0f : 1.0f;
          const float s1 = ((S.W[s * J.nw + o1] >> b) & 1u) ? -1.0f : 1.0f;
          a0 += (double)(-2.0f * s0 * f0);
          a1 += (double)(-2.0f * s1 * f1);
        }
        for (int off = 16; off > 0; off >>= 1) {
          a0 += __shfl_xor_sync(0xffffffffu, a0, off);
          a1 += __shfl_xor_sync(0xffffffffu, a1, off);
        }
        if (lane == 0) {
          S.dE0[b] = a0;
          S.dE1[b] = a1;
        }
      }
      __syncthreads();
      for (uint32_t s = tid; s < n; s += blockDim.x) {
        const uint32_t c = S.Cl[s];
        if (c) {
          S.W[s * J.nw + o0] ^= c;
          S.W[s * J.nw + o1] ^= c;
        }
      }
      if (tid < 32 && S.nneg[tid]) {
        // the reference invalidates both caches; the next energy() is energy_ref
        const uint32_t x0 = c0 * J.ntp + tb + tid, x1 = c1 * J.ntp + tb + tid;
        S.Er[x0] += S.dE0[tid];
        S.Er[x1] += S.dE1[tid];
        S.Ec[x0] = S.Er[x0];
        S.Ec[x1] = S.Er[x1];
      }
      __syncthreads();
    }
  }
}

__device__ void exchange_phase(const PtJob& J, Smem& S, uint32_t i) {
  const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5, nwarp = blockDim.x >> 5;
  const uint32_t nt = J.nt;
  for (uint32_t c = warp; c < J.C; c += nwarp) {
    double* Ec = S.Ec + c * J.ntp;
    double* Er = S.Er + c * J.ntp;
    uint64_t D = 0;
    if (J.threaded) {
      bool d[2] = {false, false};
      for (int h = 0; h < 2; ++h) {
        const uint32_t j = lane + 32u * h;
        if (j + 1 < nt) {
          const float des = (float)Ec[j + 1] - (float)Ec[j];
          const float dlt = (J.betas[j + 1] - J.betas[j]) * des;
          d[h] = dlt >= 0.0f ||
                 u24(philox4x32_10(make_uint4(j, i, c, PTAG_EXCH), J.key).x) < __expf(dlt);
        }
      }
      D = (uint64_t)__ballot_sync(0xffffffffu, d[0]) | ((uint64_t)__ballot_sync(0xffffffffu, d[1]) << 32);
    } else {
      if (lane == 0) {
        float carry = 0.0f;
        bool prev = false;
        for (uint32_t j = 0; j + 1 < nt; ++j) {
          float des = (float)Ec[j + 1] - (float)Ec[j];
          if (prev) des += carry;  // ΔE propagation after a swap (tamc-core/src/pt.rs:138-141)
          const float dlt = (J.betas[j + 1] - J.betas[j]) * des;
          const bool dj = dlt >= 0.0f ||
                          u24(philox4x32_10(make_uint4(j, i, c, PTAG_EXCH), J.key).x) < __expf(dlt);
          if (dj) D |= 1ull << j;
          prev = dj;
          carry = des;
        }
      }
      D = __shfl_sync(0xffffffffu, D, 0);
    }
    // acceptance counts, slot permutation of energies and tags, round trips
    uint32_t* acc = J.acc + (size_t)c * nt;
    uint8_t* tg = J.tags + (size_t)c * nt;
    double e_new[2], r_new[2];
    uint8_t t_new[2];
    for (int h = 0; h < 2; ++h) {
      const uint32_t k = lane + 32u * h;
      if (k >= nt) continue;
      if ((D >> k) & 1ull) acc[k] += 1;
      uint32_t src = k;
      if ((D >> k) & 1ull) src = k + 1;
      else if (k > 0 && ((D >> (k - 1)) & 1ull)) {
        const uint64_t nd = ~D & ((1ull << k) - 1ull);
        src = nd ? (uint32_t)(64 - __clzll((long long)nd)) : 0u;
      }
      e_new[h] = Ec[src];
      r_new[h] = Er[src];
      t_new[h] = tg[src];
    }
    __syncwarp();
    for (int h = 0; h < 2; ++h) {
      const uint32_t k = lane + 32u * h;
      if (k >= nt) continue;
      Ec[k] = e_new[h];
      Er[k] = r_new[h];
      tg[k] = t_new[h];
    }
    __syncwarp();
    if (lane == 0) {  // PTState::update_round_trips (tamc-core/src/pt.rs:54-72)
      uint8_t lo = tg[0];
      if (lo == 0) lo = 1;
      else if (lo == 4) { J.rtrips[c] += 1; lo = 1; }
      else if (lo == 2) lo = 3;
      tg[0] = lo;
      uint8_t hi = tg[nt - 1];
      if (hi == 0) hi = 2;
      else if (hi == 3) { J.rtrips[c] += 1; hi = 2; }
      else if (hi == 1) hi = 4;
      tg[nt - 1] = hi;
    }
    __syncwarp();
    for (uint32_t k = lane; k < nt; k += 32) {
      const uint8_t v = tg[k];
      if (v == 1 || v == 3) J.dhist[((size_t)c * nt + k) * 2] += 1;
      else if (v == 2 || v == 4) J.dhist[((size_t)c * nt + k) * 2 + 1] += 1;
    }
    if (lane == 0) S.Dm[c] = D;
  }
  __syncthreads();
  // move the spins: one bit permutation per chain word
  for (uint32_t s = tid; s < J.n; s += blockDim.x) {
    for (uint32_t c = 0; c < J.C; ++c) {
      const uint64_t D = S.Dm[c];
      if (!D) continue;
      uint32_t* w = S.W + s * J.nw + c * J.wpc;
      uint64_t v = w[0];
      if (J.wpc > 1) v |= (uint64_t)w[1] << 32;
      v = bitperm(v, D);
      w[0] = (uint32_t)v;
      if (J.wpc > 1) w[1] = (uint32_t)(v >> 32);
    }
  }
  __syncthreads();
}

template <bool SELF>
__device__ void sweep_phase(const PtJob& J, const FastInst& F, Smem& S, uint32_t i, uint32_t Teff) {
  const uint32_t tid = threadIdx.x;
  const uint32_t k = tid % J.qps;
  const uint32_t ch = k / J.qpc, q = k % J.qpc;
  const uint32_t wo = ch * J.wpc + (q >> 3), shift = 4 * (q & 7u);
  const uint32_t qid = ch * 16u + q;
  const float4 beta = S.beta4[k];
  const uint32_t stride = Teff / J.qps;
  Fx4 acc{0, 0, 0, 0};
  Fx4 qacc{0, 0, 0, 0};
  for (uint32_t c = 0; c < F.ncolors; ++c) {
    if (tid < Teff) {
      const uint32_t c1 = J.F.color_off[c + 1];
      for (uint32_t s = J.F.color_off[c] + tid / J.qps; s < c1; s += stride) {
        const uint4 rnd = philox4x32_10(make_uint4(s, i, qid, PTAG_SWEEP), J.key);
        const uint32_t m = quad_update<true>(s, shift, F, S.W, J.nw, wo, beta, rnd, acc);
        if (m) {
          atomicXor(&S.W[s * J.nw + wo], m << shift);
          if (SELF) {
            const long long k2 = to_fx(2.0f * J.F.kd[s]);
            qacc.x += (m & 1u) ? k2 : 0;
            qacc.y += (m & 2u) ? k2 : 0;
            qacc.z += (m & 4u) ? k2 : 0;
            qacc.w += (m & 8u) ? k2 : 0;
          }
        }
      }
    }
    __syncthreads();
  }
  Fx4* red = reinterpret_cast<Fx4*>(S.red);   // T Fx4 = red + redq (2 * T * 16 bytes)
  red[tid] = acc;
  __syncthreads();
  long long sums[4] = {0, 0, 0, 0};
  for (uint32_t x = tid, r = 0; x < J.C * J.ntp && r < 4; x += blockDim.x, ++r) {
    const uint32_t c = x / J.ntp, t = x % J.ntp;
    const uint32_t kk = c * J.qpc + t / 4;
    long long sum = 0;
    for (uint32_t th = kk; th < Teff; th += J.qps) {
      const Fx4 v = red[th];
      sum += (t & 3u) == 0 ? v.x : (t & 3u) == 1 ? v.y : (t & 3u) == 2 ? v.z : v.w;
    }
    sums[r] = sum;
  }
  long long qsums[4] = {0, 0, 0, 0};
  if (SELF) {
    __syncthreads();
    red[tid] = qacc;
    __syncthreads();
    for (uint32_t x = tid, r = 0; x < J.C * J.ntp && r < 4; x += blockDim.x, ++r) {
      const uint32_t c = x / J.ntp, t = x % J.ntp;
      const uint32_t kk = c * J.qpc + t / 4;
      long long q = 0;
      for (uint32_t th = kk; th < Teff; th += J.qps) {
        const Fx4 v = red[th];
        q += (t & 3u) == 0 ? v.x : (t & 3u) == 1 ? v.y : (t & 3u) == 2 ? v.z : v.w;
      }
      qsums[r] = q;
    }
  }
  // IsingSampler::sweep: energy += Σ accepted ΔE (src/ising.rs:226-232)
  for (uint32_t x = tid, r = 0; x < J.C * J.ntp && r < 4; x += blockDim.x, ++r) {
    S.Ec[x] += (double)sums[r] * TAMC_FX_INV;
    S.Er[x] += (double)(sums[r] + qsums[r]) * TAMC_FX_INV;
  }
  __syncthreads();
}

__device__ __forceinline__ bool sched(int64_t period, uint32_t i, uint32_t meas_init, uint32_t num_sweeps) {
  return period >= 0 && i >= meas_init && ((i - meas_init) % (uint32_t)period == 0 || i == num_sweeps - 1);
}

__device__ void measure_phase(const PtJob& J, const FastInst& F, Smem& S, uint32_t i, uint32_t& m_cur,
                              uint32_t& s_cur) {
  __shared__ int s_new;
  __shared__ uint32_t s_k, s_c, s_t;
  const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5, nwarp = blockDim.x >> 5;
  const uint32_t n = J.n, nt = J.nt, C = J.C;
  // ground-state tracking (first minimum over slots, then chains; strict improvement)
  if (tid == 0) {
    float best = 0.0f;
    uint32_t bc = 0, bt = 0;
    for (uint32_t c = 0; c < C; ++c) {
      uint32_t i1 = 0;
      float e1 = (float)S.Ec[c * J.ntp];
      for (uint32_t t = 1; t < nt; ++t) {
        const float e = (float)S.Ec[c * J.ntp + t];
        if (e < e1) { e1 = e; i1 = t; }
      }
      if (c == 0 || e1 < best) { best = e1; bc = c; bt = i1; }
    }
    s_new = 0;
    if (!*J.log.have || best < *J.log.minE) {
      *J.log.have = 1;
      *J.log.minE = best;
      const uint32_t k = *J.log.count;
      if (k < J.log.cap) {
        J.log.steps[k] = i;
        J.log.E[k] = best;
        s_new = 1;
        s_k = k;
        s_c = bc;
        s_t = bt;
      }
      *J.log.count = k + 1;
    }
  }
  __syncthreads();
  if (s_new) {
    const uint32_t nw64 = (n + 63) / 64;
    const uint32_t o = s_c * J.wpc + (s_t >> 5), b = s_t & 31u;
    for (uint32_t wd = tid; wd < nw64; wd += blockDim.x) {
      uint64_t v = 0;
      for (uint32_t x = 0; x < 64 && wd * 64 + x < n; ++x)
        v |= (uint64_t)((S.W[F.iperm[wd * 64 + x] * J.nw + o] >> b) & 1u) << x;
      J.log.words[(size_t)s_k * nw64 + wd] = v;
    }
  }
  const uint32_t P = C / 2;
  if (sched(J.sample, i, J.meas_init, J.num_sweeps)) {
    const uint32_t m = m_cur++;
    for (uint32_t x = tid; x < C * nt; x += blockDim.x) {
      const uint32_t c = x / nt, t = x % nt;
      J.out.e[(size_t)t * J.out.M * C + (size_t)m * C + c] = (float)S.Ec[c * J.ntp + t];
    }
    for (uint32_t y = warp; y < P * nt; y += nwarp) {
      const uint32_t p = y / nt, t = y % nt;
      const uint32_t o0 = 2 * p * J.wpc + (t >> 5), o1 = (2 * p + 1) * J.wpc + (t >> 5), b = t & 31u;
      uint32_t neg = 0;
      for (uint32_t s = lane; s < n; s += 32) neg += (S.W[s * J.nw + o0] ^ S.W[s * J.nw + o1]) >> b & 1u;
      for (int off = 16; off > 0; off >>= 1) neg += __shfl_xor_sync(0xffffffffu, neg, off);
      if (lane == 0) J.out.q[(size_t)t * J.out.M * P + (size_t)m * P + p] = (int32_t)n - 2 * (int32_t)neg;
      for (uint32_t kx = 0; kx < J.out.nchi; ++kx) {
        const double* wv = F.sus + (size_t)kx * n;
        double chi = 0.0;
        for (uint32_t s = lane; s < n; s += 32) {
          const uint32_t x = (S.W[s * J.nw + o0] ^ S.W[s * J.nw + o1]) >> b & 1u;
          chi += x ? -wv[s] : wv[s];
        }
        for (int off = 16; off > 0; off >>= 1) chi += __shfl_xor_sync(0xffffffffu, chi, off);
        if (lane == 0)
          J.out.sus[((size_t)t * J.out.nchi + kx) * J.out.M * P + (size_t)m * P + p] = (float)chi;
      }
    }
  }
  if (sched(J.sample_states, i, J.meas_init, J.num_sweeps)) {
    const uint32_t smp = s_cur++;
    const uint32_t nb = (n + 7) / 8;
    const uint32_t Z = J.level == 0 ? nt : (J.level == 1 ? nt / 2 : 1);
    const uint32_t total = Z * C * nb;
    for (uint32_t x = tid; x < total; x += blockDim.x) {
      const uint32_t byte = x % nb, c = (x / nb) % C, z = x / (nb * C);
      const uint32_t t = J.level == 0 ? z : (J.level == 1 ? nt - 1 - z : nt - 1);
      const uint32_t o = c * J.wpc + (t >> 5), b = t & 31u;
      uint32_t v = 0;
      for (uint32_t bit = 0; bit < 8 && byte * 8 + bit < n; ++bit)
        v |= ((S.W[F.iperm[byte * 8 + bit] * J.nw + o] >> b) & 1u) << bit;
      J.out.samp[(((size_t)z * J.out.S + smp) * C + c) * nb + byte] = (uint8_t)v;
    }
  }
  __syncthreads();
}

template <bool SELF>
__device__ void run_job(const PtJob& J, char* smem_base) {
  Smem S;
  carve_all(&S, smem_base, J.n, J.nw, J.C, J.ntp, J.qps, blockDim.x, J.F.nnz, J.csr_smem != 0);
  const uint32_t tid = threadIdx.x, T = blockDim.x;
  const uint32_t n = J.n;
  FastInst F = J.F;
  if (J.csr_smem) {
    for (uint32_t x = tid; x <= n; x += T) S.rp[x] = J.F.rp[x];
    for (uint32_t x = tid; x < n; x += T) S.bias[x] = J.F.bias[x];
    for (uint32_t x = tid; x < J.F.nnz; x += T) S.ent[x] = J.F.ent[x];
    F.rp = S.rp;
    F.bias = S.bias;
    F.ent = S.ent;
  }
  for (uint32_t k = tid; k < J.qps; k += T) {
    const uint32_t q = k % J.qpc;
    const float L2E = 1.4426950408889634f;  // beta * log2(e) for ex2
    S.beta4[k] = make_float4(J.betas[4 * q] * L2E, J.betas[4 * q + 1] * L2E, J.betas[4 * q + 2] * L2E,
                             J.betas[4 * q + 3] * L2E);
  }
  const uint32_t Teff = (T / J.qps) * J.qps;
  if (J.init == 1) {
    // random initial replicas, then their energies
    for (uint32_t x = tid; x < n * J.nw; x += T) {
      const uint32_t s = x / J.nw, wo = x % J.nw;
      const uint32_t ch = wo / J.wpc, w = wo % J.wpc;
      uint32_t v = 0;
      for (uint32_t qq = 0; qq < 8; ++qq) {
        const uint32_t q = 8 * w + qq;
        if (q >= J.qpc) break;
        v |= init_nibble(philox4x32_10(make_uint4(s, 0xffffffffu, ch * 16u + q, PTAG_INIT), J.key)) << (4 * qq);
      }
      S.W[x] = v;
    }
    __syncthreads();
    full_energies(J, F, S, Teff);
  } else {
    for (uint32_t x = tid; x < n * J.nw; x += T) S.W[x] = J.W[x];
    for (uint32_t x = tid; x < J.C * J.ntp; x += T) {
      S.Ec[x] = J.Ec[x];
      S.Er[x] = J.Er[x];
    }
    __syncthreads();
    if (J.init == 2) full_energies(J, F, S, Teff);
  }
  uint32_t m_cur = J.m_base, s_cur = J.s_base;
  for (uint32_t i = J.sweep_begin; i < J.sweep_end; ++i) {
    if (J.icm) icm_phase(J, F, S, i);
    exchange_phase(J, S, i);
    sweep_phase<SELF>(J, F, S, i, Teff);
    if (i >= J.meas_init) measure_phase(J, F, S, i, m_cur, s_cur);
  }
  for (uint32_t x = tid; x < n * J.nw; x += T) J.W[x] = S.W[x];
  for (uint32_t x = tid; x < J.C * J.ntp; x += T) {
    J.Ec[x] = S.Ec[x];
    J.Er[x] = S.Er[x];
  }
  if (tid == 0 && J.count_out) *J.count_out = *J.log.count;
  __syncthreads();
}

__global__ void __launch_bounds__(512, 1) k_pt_fused(const PtJob* __restrict__ jobs, uint32_t njobs, uint32_t* ctr) {
  extern __shared__ uint4 smem_u4[];
  __shared__ uint32_t s_job;
  for (;;) {
    if (threadIdx.x == 0) s_job = atomicAdd(ctr, 1u);
    __syncthreads();
    const uint32_t jid = s_job;
    __syncthreads();
    if (jid >= njobs) break;
    const PtJob J = jobs[jid];
    if (J.self_loops) run_job<true>(J, reinterpret_cast<char*>(smem_u4));
    else run_job<false>(J, reinterpret_cast<char*>(smem_u4));
  }
}

// ============================================================ plain form ====
// One instance spread over the whole GPU, one launch per sweep phase:
//   k_plain_head  (1 CTA): close the previous round (add its sweep energy sums,
//                 measurements), then ICM and replica exchange of the next
//                 round, with the replica words in global memory;
//   k_plain_sweep (grid) : one launch per colour class, (site, quad) tasks
//                 spread over all SMs, flips by atomicXor on the global words,
//                 ΔE sums by 64-bit integer atomics (order-independent).
// The phase functions are the fused kernel's, so both forms produce the same
// Markov chain bit for bit; the round index and measurement counters live in
// device memory (PlainCtl) so a captured chunk of rounds replays unchanged.
__host__ __device__ inline size_t plain_head_smem(uint32_t n, uint32_t C, uint32_t ntp) {
  return al16((size_t)n * 4) * 2 + al16((size_t)C * ntp * 8) * 2 + al16(32 * 4) + al16(32 * 8) * 2 +
         al16((size_t)C * 8);
}

__global__ void __launch_bounds__(1024, 1) k_plain_head(const PtJob* __restrict__ jp, PlainCtl* ctl,
                                                       long long* acc, int mode) {
  extern __shared__ uint4 smem_u4[];
  const PtJob J = *jp;
  const uint32_t tid = threadIdx.x;
  char* base = reinterpret_cast<char*>(smem_u4);
  Smem S{};
  size_t o = 0;
  auto take = [&](size_t bytes) {
    char* p = base + o;
    o = al16(o + bytes);
    return p;
  };
  S.D = (uint32_t*)take((size_t)J.n * 4);
  S.Cl = (uint32_t*)take((size_t)J.n * 4);
  S.Ec = (double*)take((size_t)J.C * J.ntp * 8);
  S.Er = (double*)take((size_t)J.C * J.ntp * 8);
  S.nneg = (uint32_t*)take(32 * 4);
  S.dE0 = (double*)take(32 * 8);
  S.dE1 = (double*)take(32 * 8);
  S.Dm = (unsigned long long*)take((size_t)J.C * 8);
  S.W = J.W;
  const FastInst F = J.F;
  const uint32_t CN = J.C * J.ntp;
  long long* accq = acc + CN;
  for (uint32_t x = tid; x < CN; x += blockDim.x) {
    double ec = J.Ec[x], er = J.Er[x];
    if (mode == 2) {  // initial energies from the fixed-point sums of the energy kernel
      ec = (double)J.F.offset + (double)acc[x] * TAMC_FX_INV;
      er = ec;
      acc[x] = 0;
    } else if (ctl->pending) {  // IsingSampler::sweep: energy += Σ accepted ΔE
      ec += (double)acc[x] * TAMC_FX_INV;
      er += (double)(acc[x] + accq[x]) * TAMC_FX_INV;
      acc[x] = 0;
      accq[x] = 0;
    }
    S.Ec[x] = ec;
    S.Er[x] = er;
  }
  __syncthreads();
  uint32_t m_cur = ctl->m_cur, s_cur = ctl->s_cur;
  if (mode != 2 && ctl->pending) {
    const uint32_t ip = ctl->i - 1;
    if (ip >= J.meas_init) measure_phase(J, F, S, ip, m_cur, s_cur);
  }
  __syncthreads();
  if (mode == 0) {  // start round i: ICM, then exchange; the sweeps follow
    const uint32_t i = ctl->i;
    if (J.icm) icm_phase(J, F, S, i);
    exchange_phase(J, S, i);
  }
  for (uint32_t x = tid; x < CN; x += blockDim.x) {
    J.Ec[x] = S.Ec[x];
    J.Er[x] = S.Er[x];
  }
  __syncthreads();
  if (tid == 0) {
    ctl->m_cur = m_cur;
    ctl->s_cur = s_cur;
    if (mode == 0) {
      ctl->i += 1;
      ctl->pending = 1;
    } else {
      ctl->pending = 0;
    }
    if (J.count_out) *J.count_out = *J.log.count;
  }
}

template <bool SELF>
__global__ void __launch_bounds__(256) k_plain_sweep(const PtJob* __restrict__ jp, const PlainCtl* __restrict__ ctl,
                                                     uint32_t color, long long* acc) {
  extern __shared__ uint4 smem_u4[];
  const PtJob& J = *jp;
  const uint32_t CN = J.C * J.ntp;
  long long* sacc = reinterpret_cast<long long*>(smem_u4);
  long long* saccq = sacc + CN;
  float4* b4 = reinterpret_cast<float4*>(saccq + CN + (CN & 1u));
  for (uint32_t x = threadIdx.x; x < 2 * CN; x += blockDim.x) sacc[x] = 0;
  const float L2E = 1.4426950408889634f;
  for (uint32_t k = threadIdx.x; k < J.qps; k += blockDim.x) {
    const uint32_t q = k % J.qpc;
    b4[k] = make_float4(J.betas[4 * q] * L2E, J.betas[4 * q + 1] * L2E, J.betas[4 * q + 2] * L2E,
                        J.betas[4 * q + 3] * L2E);
  }
  __syncthreads();
  const uint32_t i = ctl->i - 1;
  const uint32_t c0 = J.F.color_off[color], nc = J.F.color_off[color + 1] - c0;
  const uint64_t ntask = (uint64_t)nc * J.qps;
  const FastInst F = J.F;
  for (uint64_t task = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; task < ntask;
       task += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t k = (uint32_t)(task % J.qps);
    const uint32_t s = c0 + (uint32_t)(task / J.qps);
    const uint32_t ch = k / J.qpc, q = k % J.qpc;
    const uint32_t wo = ch * J.wpc + (q >> 3), shift = 4 * (q & 7u);
    const uint4 rnd = philox4x32_10(make_uint4(s, i, ch * 16u + q, PTAG_SWEEP), J.key);
    Fx4 a{0, 0, 0, 0};
    const uint32_t m = quad_update<true>(s, shift, F, J.W, J.nw, wo, b4[k], rnd, a);
    if (m) {
      atomicXor(&J.W[s * J.nw + wo], m << shift);
      const uint32_t slot = ch * J.ntp + 4 * q;
      if (m & 1u) atomicAdd((unsigned long long*)&sacc[slot + 0], (unsigned long long)a.x);
      if (m & 2u) atomicAdd((unsigned long long*)&sacc[slot + 1], (unsigned long long)a.y);
      if (m & 4u) atomicAdd((unsigned long long*)&sacc[slot + 2], (unsigned long long)a.z);
      if (m & 8u) atomicAdd((unsigned long long*)&sacc[slot + 3], (unsigned long long)a.w);
      if (SELF) {
        const unsigned long long k2 = (unsigned long long)to_fx(2.0f * F.kd[s]);
        for (uint32_t r = 0; r < 4; ++r)
          if ((m >> r) & 1u) atomicAdd((unsigned long long*)&saccq[slot + r], k2);
      }
    }
  }
  __syncthreads();
  for (uint32_t x = threadIdx.x; x < 2 * CN; x += blockDim.x)
    if (sacc[x]) atomicAdd((unsigned long long*)&acc[x], (unsigned long long)sacc[x]);
}

// Initial replicas (random, as the fused kernel's init) and their energy terms.
__global__ void k_plain_init(const PtJob* __restrict__ jp, long long* acc, int random) {
  const PtJob& J = *jp;
  const uint64_t total = (uint64_t)J.n * J.nw;
  if (random) {
    for (uint64_t x = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; x < total;
         x += (uint64_t)gridDim.x * blockDim.x) {
      const uint32_t s = (uint32_t)(x / J.nw), wo = (uint32_t)(x % J.nw);
      const uint32_t ch = wo / J.wpc, w = wo % J.wpc;
      uint32_t v = 0;
      for (uint32_t qq = 0; qq < 8; ++qq) {
        const uint32_t q = 8 * w + qq;
        if (q >= J.qpc) break;
        v |= init_nibble(philox4x32_10(make_uint4(s, 0xffffffffu, ch * 16u + q, PTAG_INIT), J.key)) << (4 * qq);
      }
      J.W[x] = v;
    }
  }
}
__global__ void k_plain_energy(const PtJob* __restrict__ jp, long long* acc) {
  const PtJob& J = *jp;
  const uint64_t ntask = (uint64_t)J.n * J.qps;
  for (uint64_t task = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; task < ntask;
       task += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t k = (uint32_t)(task % J.qps), s = (uint32_t)(task / J.qps);
    const uint32_t ch = k / J.qpc, q = k % J.qpc;
    const uint32_t wo = ch * J.wpc + (q >> 3), shift = 4 * (q & 7u);
    const float4 e = energy_terms4(s, shift, J.F, J.W, J.nw, wo);
    const uint32_t slot = ch * J.ntp + 4 * q;
    atomicAdd((unsigned long long*)&acc[slot + 0], (unsigned long long)to_fx(e.x));
    atomicAdd((unsigned long long*)&acc[slot + 1], (unsigned long long)to_fx(e.y));
    atomicAdd((unsigned long long*)&acc[slot + 2], (unsigned long long)to_fx(e.z));
    atomicAdd((unsigned long long*)&acc[slot + 3], (unsigned long long)to_fx(e.w));
  }
}

}  // namespace

size_t fused_smem_bytes(const PtJob& j, uint32_t T, bool csr_smem) {
  return carve_all(nullptr, nullptr, j.n, j.nw, j.C, j.ntp, j.qps, T, j.F.nnz, csr_smem);
}

int fused_blocks_per_sm(uint32_t T, size_t smem) {
  TAMC_CUDA(cudaFuncSetAttribute(k_pt_fused, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int nb = 0;
  TAMC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_pt_fused, (int)T, smem));
  return nb;
}

size_t plain_head_bytes(const PtJob& j) { return plain_head_smem(j.n, j.C, j.ntp); }

void plain_launch_head(cudaStream_t st, const PtJob* d_job, PlainCtl* ctl, long long* acc, int mode, size_t smem) {
  TAMC_CUDA(cudaFuncSetAttribute(k_plain_head, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_plain_head<<<1, 1024, smem, st>>>(d_job, ctl, acc, mode);
  TAMC_CUDA(cudaGetLastError());
}

void plain_launch_sweep(cudaStream_t st, const PtJob& j, const PtJob* d_job, const PlainCtl* ctl, uint32_t color,
                        uint32_t ntask, long long* acc, uint32_t grid_cap) {
  const uint32_t T = 256;
  const uint32_t grid = std::max(1u, std::min(grid_cap, (ntask + T - 1) / T));
  const size_t smem = (size_t)(2 * j.C * j.ntp + 2) * 8 + (size_t)j.qps * 16;
  if (j.self_loops) {
    TAMC_CUDA(cudaFuncSetAttribute(k_plain_sweep<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_plain_sweep<true><<<grid, T, smem, st>>>(d_job, ctl, color, acc);
  } else {
    TAMC_CUDA(cudaFuncSetAttribute(k_plain_sweep<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_plain_sweep<false><<<grid, T, smem, st>>>(d_job, ctl, color, acc);
  }
  TAMC_CUDA(cudaGetLastError());
}

void plain_launch_init(cudaStream_t st, const PtJob* d_job, long long* acc, int random, uint32_t grid) {
  if (random) k_plain_init<<<grid, 256, 0, st>>>(d_job, acc, 1);
  k_plain_energy<<<grid, 256, 0, st>>>(d_job, acc);
  TAMC_CUDA(cudaGetLastError());
}

void fused_launch(cudaStream_t st, const PtJob* d_jobs, uint32_t njobs, uint32_t* ctr, uint32_t grid, uint32_t T,
                  size_t smem) {
  TAMC_CUDA(cudaFuncSetAttribute(k_pt_fused, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_pt_fused<<<grid, T, smem, st>>>(d_jobs, njobs, ctr);
  TAMC_CUDA(cudaGetLastError());
}

}  // namespace tamc
