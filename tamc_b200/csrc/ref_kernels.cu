// ref_kernels.cu -- reference-order replay kernels (TAMC_MODE_REF).
//
// These kernels reproduce the reference's Markov chain bit for bit: every
// replica is swept in site order 0..n-1 by one thread that owns the replica's
// Xoshiro256++ stream, ΔE is summed in CSR row order in f32, acceptance uses
// the glibc-identical expf, the ICM seed is drawn with rand's gen_range and
// the cluster is the connected q<0 component of the petgraph node range.
// Parallelism is only across independent streams (chains x temperatures, or
// SA partitions), exactly the parallelism the reference's rayon code has.
#include "ref_kernels.cuh"

namespace tamc {
namespace refk {

// ΔE of flipping site i (src/ising.rs:468-480), f32 in row order.
__device__ __forceinline__ float delta_e(const RefInst& I, const int8_t* s, uint32_t i) {
  float d = 0.0f;
  d = __fadd_rn(d, I.bias[i]);
  const uint32_t e1 = I.rp[i + 1];
  for (uint32_t e = I.rp[i]; e < e1; ++e) d = __fadd_rn(d, __fmul_rn(I.J[e], (float)s[I.col[e]]));
  const float si = (float)s[i];
  return __fmul_rn(d, __fmul_rn(-2.0f, si));
}

// MetropolisSampler::advance_impl (tamc-core/src/metropolis.rs:43-57).
__device__ __forceinline__ bool advance(const RefInst& I, const ExpTable& X, float beta, int8_t* s, uint32_t i,
                                        Xo& rng, float& de) {
  const float d = delta_e(I, s, i);
  if (d < 0.0f) {
    s[i] = (int8_t)-s[i];
    de = d;
    return true;
  }
  const float p = tamc_expf_exact(__fmul_rn(-beta, d), X.off, X.keys, X.vals);
  const float x = rng.std_f32();
  if (x < p) {
    s[i] = (int8_t)-s[i];
    de = d;
    return true;
  }
  return false;
}

// IsingSampler::sweep (src/ising.rs:225-233): returns Σ accepted ΔE in f32 site order.
__device__ float sweep_tracked(const RefInst& I, const ExpTable& X, float beta, int8_t* s, Xo& rng) {
  float de = 0.0f;
  for (uint32_t i = 0; i < I.n; ++i) {
    float d = 0.0f;
    de = __fadd_rn(de, advance(I, X, beta, s, i, rng, d) ? d : 0.0f);
  }
  return de;
}

// energy_ref (src/ising.rs:438-454) sequentially by one thread.
__device__ float energy_ref_seq(const RefInst& I, const int8_t* s) {
  float total = I.offset;
  for (uint32_t i = 0; i < I.n; ++i) {
    float h = 0.0f;
    const float si = (float)s[i];
    h = __fadd_rn(h, I.bias[i]);
    const uint32_t e1 = I.rp[i + 1];
    for (uint32_t e = I.rp[i]; e < e1; ++e) h = __fadd_rn(h, __fmul_rn(I.J[e], (float)s[I.col[e]]) / 2.0f);
    total = __fadd_rn(total, __fmul_rn(h, si));
  }
  return total;
}

// Row terms h_i * s_i of energy_ref, one row per thread; the caller sums them in order.
__device__ void energy_rows(const RefInst& I, const int8_t* s, float* rows) {
  for (uint32_t i = threadIdx.x; i < I.n; i += blockDim.x) {
    float h = 0.0f;
    const float si = (float)s[i];
    h = __fadd_rn(h, I.bias[i]);
    const uint32_t e1 = I.rp[i + 1];
    for (uint32_t e = I.rp[i]; e < e1; ++e) h = __fadd_rn(h, __fmul_rn(I.J[e], (float)s[I.col[e]]) / 2.0f);
    rows[i] = __fmul_rn(h, si);
  }
}

__device__ __forceinline__ uint32_t block_sum_u32(uint32_t v, uint32_t* sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  __syncthreads();
  if ((threadIdx.x & 31) == 0) sh[w] = v;
  __syncthreads();
  uint32_t t = 0;
  for (int k = 0; k < nw; ++k) t += sh[k];
  __syncthreads();
  return t;
}

// ------------------------------------------------------------ init ----
// energy_ref of every replica (rand_ising_state caches it, src/ising.rs:175).
__global__ void k_energy_all(RefInst I, const int8_t* spins, float* energy, uint32_t R) {
  const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r < R) energy[r] = energy_ref_seq(I, spins + (size_t)r * I.n);
}

// ------------------------------------------------------------- ICM ----
// apply_icm (src/pt.rs:521-540) + houdayer_cluster_move (src/pt.rs:31-77), one
// CTA, pairs in the reference's order.  scratch: visited[max(n,1)] u32,
// queue[n] u32, rows[n] f32.
__global__ void __launch_bounds__(512) k_icm(RefInst I, RefPt P, ExpTable X, Xo* rng, int* err) {
  __shared__ uint32_t sh[32];
  __shared__ uint32_t s_k, s_tail, s_found;
  const uint32_t n = I.n;
  for (uint32_t c = 0; c + 1 < P.C; c += 2) {
    for (uint32_t t = P.lo; t < P.nt; ++t) {
      const uint32_t r1 = P.perm[c * P.nt + t], r2 = P.perm[(c + 1) * P.nt + t];
      int8_t* s1 = P.spins + (size_t)r1 * n;
      int8_t* s2 = P.spins + (size_t)r2 * n;
      uint32_t cnt = 0;
      for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) cnt += (s1[i] != s2[i]);
      cnt = block_sum_u32(cnt, sh);
      if (cnt == 0) continue;  // `idxs.choose` returns None: no draw, no invalidation
      if (threadIdx.x == 0) {
        Xo x = *rng;
        s_k = x.gen_range(cnt);
        *rng = x;
        s_found = 0xffffffffu;
      }
      __syncthreads();
      // the k-th site with q<0 (idxs is in increasing site order)
      uint32_t base = 0;
      for (uint32_t i0 = 0; i0 < n; i0 += blockDim.x) {
        const uint32_t i = i0 + threadIdx.x;
        const bool f = i < n && s1[i] != s2[i];
        const uint32_t bal = __ballot_sync(0xffffffffu, f);
        const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
        if (lane == 0) sh[w] = __popc(bal);
        __syncthreads();
        uint32_t before = base;
        for (int k = 0; k < w; ++k) before += sh[k];
        before += __popc(bal & ((1u << lane) - 1u));
        if (f && before == s_k) s_found = i;
        uint32_t tot = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) tot += sh[k];
        base += tot;
        __syncthreads();
        if (s_found != 0xffffffffu) break;
      }
      const uint32_t seed = s_found;
      if (seed >= I.g_nodes) {  // petgraph's FixedBitSet would panic here
        if (threadIdx.x == 0) *err = TAMC_E_REFPANIC;
        return;
      }
      // BFS over the q<0 subgraph (order-free: only the discovered set matters)
      for (uint32_t i = threadIdx.x; i < I.g_nodes; i += blockDim.x) P.visited[i] = 0;
      __syncthreads();
      if (threadIdx.x == 0) {
        P.visited[seed] = 1;
        P.queue[0] = seed;
        s_tail = 1;
      }
      __syncthreads();
      uint32_t lvl_begin = 0;
      for (;;) {
        const uint32_t lvl_end = s_tail;
        __syncthreads();  // everyone has read the level bound before anyone appends
        if (lvl_begin == lvl_end) break;
        for (uint32_t q = lvl_begin + threadIdx.x; q < lvl_end; q += blockDim.x) {
          const uint32_t u = P.queue[q];
          const uint32_t e1 = I.grp[u + 1];
          for (uint32_t e = I.grp[u]; e < e1; ++e) {
            const uint32_t v = I.gcol[e];
            if (s1[v] != s2[v] && atomicExch(&P.visited[v], 1u) == 0u) P.queue[atomicAdd(&s_tail, 1u)] = v;
          }
        }
        __syncthreads();
        lvl_begin = lvl_end;
      }
      const uint32_t csz = s_tail;
      for (uint32_t q = threadIdx.x; q < csz; q += blockDim.x) {
        const uint32_t v = P.queue[q];
        const int8_t a = s1[v];
        s1[v] = s2[v];
        s2[v] = a;
      }
      __syncthreads();
      // invalidated energies are recomputed by energy_ref exactly as the next
      // Macrostate::energy call would (tamc-core/src/pt.rs:126-129)
      for (int rep = 0; rep < 2; ++rep) {
        const int8_t* s = rep ? s2 : s1;
        energy_rows(I, s, P.rows);
        __syncthreads();
        if (threadIdx.x == 0) {
          float total = I.offset;
          for (uint32_t i = 0; i < n; ++i) total = __fadd_rn(total, P.rows[i]);
          P.energy[rep ? r2 : r1] = total;
        }
        __syncthreads();
      }
    }
  }
}

// ------------------------------------------------------- exchange ----
__device__ void update_round_trips(const RefPt& P, uint32_t c) {  // tamc-core/src/pt.rs:54-84
  uint8_t* tg = P.tags + (size_t)c * P.nt;
  uint8_t& lo = tg[0];
  if (lo == 0) lo = 1;
  else if (lo == 4) { P.rtrips[c] += 1; lo = 1; }
  else if (lo == 2) lo = 3;
  uint8_t& hi = tg[P.nt - 1];
  if (hi == 0) hi = 2;
  else if (hi == 3) { P.rtrips[c] += 1; hi = 2; }
  else if (hi == 1) hi = 4;
  for (uint32_t k = 0; k < P.nt; ++k) {
    const uint8_t v = tg[k];
    if (v == 1 || v == 3) P.dhist[((size_t)c * P.nt + k) * 2] += 1;
    else if (v == 2 || v == 4) P.dhist[((size_t)c * P.nt + k) * 2 + 1] += 1;
  }
}

__device__ __forceinline__ void swap_slots(const RefPt& P, uint32_t c, uint32_t j) {  // PTState::swap_states
  uint32_t* pm = P.perm + (size_t)c * P.nt;
  const uint32_t a = pm[j];
  pm[j] = pm[j + 1];
  pm[j + 1] = a;
  uint8_t* tg = P.tags + (size_t)c * P.nt;
  const uint8_t b = tg[j];
  tg[j] = tg[j + 1];
  tg[j + 1] = b;
  P.acc[(size_t)c * P.nt + j] += 1;
}

// ThreadedPTSampler exchange (tamc-core/src/parallel/pt.rs:41-59), one thread per chain,
// uniforms from rng_vec[c][0].
__global__ void k_exchange_threaded(RefPt P, ExpTable X, Xo* rngs) {
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= P.C) return;
  Xo x = rngs[(size_t)c * P.nt];
  const uint32_t* pm = P.perm + (size_t)c * P.nt;
  for (uint32_t j = 0; j + 1 < P.nt; ++j) {
    // stale differences: E taken before any swap of this pass
    const float dlt = __fmul_rn(P.dbeta[j], __fsub_rn(P.e_stale[(size_t)c * P.nt + j + 1], P.e_stale[(size_t)c * P.nt + j]));
    if (dlt >= 0.0f || x.std_f32() < tamc_expf_exact(dlt, X.off, X.keys, X.vals)) swap_slots(P, c, j);
  }
  (void)pm;
  update_round_trips(P, c);
  rngs[(size_t)c * P.nt] = x;
}
// snapshot of the slot energies for the stale-difference exchange
__global__ void k_snapshot_energies(RefPt P) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < P.C * P.nt) P.e_stale[k] = P.energy[P.perm[k]];
}

// --------------------------------------------------------- sweeps ----
// ThreadedPTSampler sweeps (parallel/pt.rs:63-68): slot (c,t) with rng_vec[c][t].
__global__ void k_sweep_threaded(RefInst I, RefPt P, ExpTable X, Xo* rngs) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= P.C * P.nt) return;
  const uint32_t t = k % P.nt;
  const uint32_t r = P.perm[k];
  Xo x = rngs[k];
  const float de = sweep_tracked(I, X, P.betas[t], P.spins + (size_t)r * I.n, x);
  P.energy[r] = __fadd_rn(P.energy[r], de);
  rngs[k] = x;
}

// Serial mode (src/pt.rs:493-497, EnsembleSampler over ParallelTemperingSampler):
// one stream, per chain: exchange with ΔE propagation, then sweeps t = 0..nt-1.
__global__ void k_serial_round(RefInst I, RefPt P, ExpTable X, Xo* rng) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  Xo x = *rng;
  for (uint32_t c = 0; c < P.C; ++c) {
    uint32_t* pm = P.perm + (size_t)c * P.nt;
    float* des = P.e_stale;  // scratch [nt]
    for (uint32_t k = 0; k + 1 < P.nt; ++k) des[k] = __fsub_rn(P.energy[pm[k + 1]], P.energy[pm[k]]);
    for (uint32_t j = 0; j + 1 < P.nt; ++j) {
      const float dlt = __fmul_rn(P.dbeta[j], des[j]);
      if (dlt >= 0.0f || x.std_f32() < tamc_expf_exact(dlt, X.off, X.keys, X.vals)) {
        swap_slots(P, c, j);
        if (j + 2 < P.nt) des[j + 1] = __fadd_rn(des[j + 1], des[j]);
        des[j] = -des[j];
      }
    }
    update_round_trips(P, c);
    for (uint32_t t = 0; t < P.nt; ++t) {
      const uint32_t r = pm[t];
      const float de = sweep_tracked(I, X, P.betas[t], P.spins + (size_t)r * I.n, x);
      P.energy[r] = __fadd_rn(P.energy[r], de);
    }
  }
  *rng = x;
}

// ---------------------------------------------------- measurements ----
// PtIcmThermalSamples::measure / sample_states (src/pt.rs:167-226) for one
// measurement index; grid (nt, C).
__global__ void k_measure(RefInst I, RefPt P, MeasOut O, uint32_t m, int do_measure, uint32_t smp, int do_sample) {
  __shared__ uint32_t sh[32];
  const uint32_t t = blockIdx.x, c = blockIdx.y;
  const uint32_t n = I.n;
  const uint32_t r = P.perm[(size_t)c * P.nt + t];
  const int8_t* s1 = P.spins + (size_t)r * n;
  const uint32_t npair = P.C / 2;
  if (do_measure) {
    if (threadIdx.x == 0) O.e[(size_t)t * O.M * P.C + (size_t)m * P.C + c] = P.energy[r];
    if ((c & 1u) == 0 && c / 2 < npair) {
      const uint32_t p = c / 2;
      const int8_t* s2 = P.spins + (size_t)P.perm[(size_t)(c + 1) * P.nt + t] * n;
      uint32_t neg = 0;
      for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) neg += (s1[i] != s2[i]);
      neg = block_sum_u32(neg, sh);
      if (threadIdx.x == 0) O.q[(size_t)t * O.M * npair + (size_t)m * npair + p] = (int32_t)n - 2 * (int32_t)neg;
      for (uint32_t k = threadIdx.x; k < O.nchi; k += blockDim.x) {
        const double* w = I.sus + (size_t)k * n;
        double chi = 0.0;
        for (uint32_t i = 0; i < n; ++i) chi = __dadd_rn(chi, __dmul_rn(w[i], (double)(s1[i] * s2[i])));
        O.sus[((size_t)t * O.nchi + k) * O.M * npair + (size_t)m * npair + p] = (float)chi;
      }
    }
  }
  if (do_sample) {
    int z = -1;
    if (O.level == 0) z = (int)t;
    else if (O.level == 1) { if (t >= P.nt - P.nt / 2) z = (int)(P.nt - 1 - t); }
    else if (t == P.nt - 1) z = 0;
    if (z >= 0) {
      const uint32_t nb = (n + 7) / 8;
      uint8_t* dst = O.samp + (((size_t)z * O.S + smp) * P.C + c) * nb;
      for (uint32_t b = threadIdx.x; b < nb; b += blockDim.x) {
        uint32_t v = 0;
        for (uint32_t k = 0; k < 8 && b * 8 + k < n; ++k) v |= (uint32_t)(s1[b * 8 + k] <= 0) << k;
        dst[b] = (uint8_t)v;
      }
    }
  }
}

// Ground-state tracking of apply_measurements (src/pt.rs:559-581): first
// minimum over slots, then over chains, strictly below the running minimum.
__global__ void k_gs_track(RefInst I, RefPt P, GsLog L, uint32_t step) {
  __shared__ int s_new;
  __shared__ uint32_t s_rep, s_slot;
  if (threadIdx.x == 0) {
    float best = 0.0f;
    uint32_t br = 0;
    for (uint32_t c = 0; c < P.C; ++c) {
      uint32_t i1 = 0;
      float e1 = P.energy[P.perm[(size_t)c * P.nt]];
      for (uint32_t t = 1; t < P.nt; ++t) {
        const float e = P.energy[P.perm[(size_t)c * P.nt + t]];
        if (e < e1) { e1 = e; i1 = t; }
      }
      if (c == 0 || e1 < best) { best = e1; br = P.perm[(size_t)c * P.nt + i1]; }
    }
    s_new = 0;
    if (!*L.have || best < *L.minE) {
      *L.have = 1;
      *L.minE = best;
      const uint32_t k = *L.count;
      if (k < L.cap) {
        L.steps[k] = step;
        L.E[k] = best;
        s_new = 1;
        s_slot = k;
        s_rep = br;
      }
      *L.count = k + 1;
    }
  }
  __syncthreads();
  if (!s_new) return;
  const int8_t* s = P.spins + (size_t)s_rep * I.n;
  const uint32_t nw = (I.n + 63) / 64;
  for (uint32_t w = threadIdx.x; w < nw; w += blockDim.x) {
    uint64_t v = 0;
    for (uint32_t k = 0; k < 64 && w * 64 + k < I.n; ++k) v |= (uint64_t)(s[w * 64 + k] <= 0) << k;
    L.words[(size_t)s_slot * nw + w] = v;
  }
}

// ------------------------------------------------------------- SA ----
// sa_loop over one partition (src/sa.rs:167-199, tamc-core/src/sa.rs:27-48):
// for each beta, each replica of the partition is swept in turn with the
// partition's stream.  One thread per partition.
__global__ void k_sa(RefInst I, ExpTable X, int8_t* spins, Xo* rngs, uint32_t parts, uint32_t per,
                     const float* betas, uint32_t nbeta) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= parts) return;
  Xo x = rngs[p];
  for (uint32_t b = 0; b < nbeta; ++b) {
    const float beta = betas[b];
    for (uint32_t r = 0; r < per; ++r) {
      int8_t* s = spins + ((size_t)p * per + r) * I.n;
      for (uint32_t i = 0; i < I.n; ++i) {
        float d;
        advance(I, X, beta, s, i, x, d);
      }
    }
  }
  rngs[p] = x;
}

}  // namespace refk

// ----------------------------------------------------------- launchers ----
void ref_energy_all(cudaStream_t st, const RefInst& I, const int8_t* spins, float* energy, uint32_t R) {
  if (!R) return;
  refk::k_energy_all<<<(R + 63) / 64, 64, 0, st>>>(I, spins, energy, R);
}
void ref_icm(cudaStream_t st, const RefInst& I, const RefPt& P, const ExpTable& X, Xo* rng, int* err) {
  refk::k_icm<<<1, 512, 0, st>>>(I, P, X, rng, err);
}
void ref_exchange_threaded(cudaStream_t st, const RefPt& P, const ExpTable& X, Xo* rngs) {
  const uint32_t k = P.C * P.nt;
  refk::k_snapshot_energies<<<(k + 127) / 128, 128, 0, st>>>(P);
  refk::k_exchange_threaded<<<(P.C + 31) / 32, 32, 0, st>>>(P, X, rngs);
}
void ref_sweep_threaded(cudaStream_t st, const RefInst& I, const RefPt& P, const ExpTable& X, Xo* rngs) {
  const uint32_t k = P.C * P.nt;
  refk::k_sweep_threaded<<<(k + 31) / 32, 32, 0, st>>>(I, P, X, rngs);
}
void ref_serial_round(cudaStream_t st, const RefInst& I, const RefPt& P, const ExpTable& X, Xo* rng) {
  refk::k_serial_round<<<1, 1, 0, st>>>(I, P, X, rng);
}
void ref_measure(cudaStream_t st, const RefInst& I, const RefPt& P, const MeasOut& O, uint32_t m, bool meas,
                 uint32_t smp, bool samp) {
  refk::k_measure<<<dim3(P.nt, P.C), 128, 0, st>>>(I, P, O, m, meas ? 1 : 0, smp, samp ? 1 : 0);
}
void ref_gs_track(cudaStream_t st, const RefInst& I, const RefPt& P, const GsLog& L, uint32_t step) {
  refk::k_gs_track<<<1, 128, 0, st>>>(I, P, L, step);
}
void ref_sa(cudaStream_t st, const RefInst& I, const ExpTable& X, int8_t* spins, Xo* rngs, uint32_t parts,
            uint32_t per, const float* betas, uint32_t nbeta) {
  refk::k_sa<<<(parts + 31) / 32, 32, 0, st>>>(I, X, spins, rngs, parts, per, betas, nbeta);
}

}  // namespace tamc
