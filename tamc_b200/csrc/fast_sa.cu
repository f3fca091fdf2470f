// fast_sa.cu -- colour-ordered simulated annealing (TAMC_MODE_FAST).
//
// One CTA owns G = 4*NQ replicas for the whole schedule; their spins live in
// shared memory as one 32-bit word per site (bits 0..G-1), and, when it fits,
// so does the colour-ordered CSR of the instance.  A sweep visits the colour
// classes in order; inside a class the sites are independent, so every
// (site, quad) task runs in parallel and the sweep is a sequential sweep in
// colour order.  HBM is touched only to load the instance and to write the
// final states and energies: the kernel is bound by issue (ΔE, Philox, exp),
// not by memory.
#include "fast_common.cuh"
#include "fast_sa.cuh"

#include <cstdio>
#include <map>
#include <mutex>
#include <tuple>

namespace tamc {

namespace {

template <int NQ, bool SMEM, uint32_t DEG>
__global__ void __launch_bounds__(1024) k_sa_fast(SaFastArgs a) {
  extern __shared__ uint4 smem_u4[];
  constexpr uint32_t G = 4 * NQ;
  const uint32_t T = blockDim.x, tid = threadIdx.x;
  const uint32_t n = a.F.n;
  uint32_t* W = reinterpret_cast<uint32_t*>(smem_u4);
  FastInst F = a.F;
  if (SMEM) {
    // [W: n words][rp: n+1][bias: n][pad to 8][ent: nnz uint2]
    uint32_t* rp = W + n;
    float* bias = reinterpret_cast<float*>(rp + n + 1);
    uint2* ent = reinterpret_cast<uint2*>(W + ((3u * n + 1u + 1u) & ~1u));
    for (uint32_t i = tid; i <= n; i += T) rp[i] = a.F.rp[i];
    for (uint32_t i = tid; i < n; i += T) bias[i] = a.F.bias[i];
    for (uint32_t i = tid; i < a.F.nnz; i += T) ent[i] = a.F.ent[i];
    F.rp = rp;
    F.bias = bias;
    F.ent = ent;
  }
  const uint32_t r0 = blockIdx.x * G;
  const uint2 key = a.key;
  for (uint32_t s = tid; s < n; s += T) {
    uint32_t w = 0;
    if (a.init_words) {
      w = a.init_words[(size_t)(r0 >> 5) * n + a.F.perm[s]] >> (r0 & 31u);
      if (G < 32) w &= (1u << G) - 1u;
    } else {
#pragma unroll
      for (uint32_t q = 0; q < NQ; ++q)
        w |= init_nibble(philox4x32_10(make_uint4(s, 0xffffffffu, (r0 >> 2) + q, PTAG_INIT), key)) << (4 * q);
    }
    W[s] = w;
  }
  __syncthreads();
  const uint32_t q = tid % NQ;
  const uint32_t shift = 4 * q;
  const uint32_t qid = (r0 >> 2) + q;
  const uint32_t stride = T / NQ;
  Fx4 acc{0, 0, 0, 0};  // unused: SA energies are computed once at the end
  const PhiloxKeys PK = philox_schedule(key);
  for (uint32_t sw = 0; sw < a.nbeta; ++sw) {
    const float b = a.betas[sw] * TAMC_2LOG2E;  // 2 beta log2(e)
    const float4 beta = make_float4(b, b, b, b);
    for (uint32_t c = 0; c < F.ncolors; ++c) {
      const uint32_t c1 = a.F.color_off[c + 1];
      for (uint32_t s = a.F.color_off[c] + tid / NQ; s < c1; s += stride) {
        const uint4 rnd = philox4x32_10(make_uint4(s, sw, qid, PTAG_SWEEP), PK);
        const uint32_t m = quad_update<false, DEG>(s, shift, F, W, 1, 0, beta, rnd, acc);
        if (m) {
          if (NQ == 1) W[s] ^= m;
          else atomicXor(&W[s], m << shift);
        }
      }
      __syncthreads();
    }
  }
  // energy_ref of every replica: f32 row terms accumulated in fixed point
  long long e0 = 0, e1 = 0, e2 = 0, e3 = 0;
  for (uint32_t s = tid / NQ; s < n; s += stride) {
    const float4 t = energy_terms4(s, shift, F, W, 1, 0);
    e0 += to_fx(t.x);
    e1 += to_fx(t.y);
    e2 += to_fx(t.z);
    e3 += to_fx(t.w);
  }
#pragma unroll
  for (uint32_t off = 16; off >= NQ; off >>= 1) {
    e0 += __shfl_xor_sync(0xffffffffu, e0, off);
    e1 += __shfl_xor_sync(0xffffffffu, e1, off);
    e2 += __shfl_xor_sync(0xffffffffu, e2, off);
    e3 += __shfl_xor_sync(0xffffffffu, e3, off);
  }
  __syncthreads();  // W is still read below; reuse a separate region for the reduction
  long long* red = reinterpret_cast<long long*>(smem_u4) + ((SMEM ? (3u * n + 2u + 2u * a.F.nnz) : n) + 1u) / 2u + 1u;
  const uint32_t lane = tid & 31u, warp = tid >> 5, nw = T >> 5;
  if (lane < NQ) {
    red[(warp * NQ + lane) * 4 + 0] = e0;
    red[(warp * NQ + lane) * 4 + 1] = e1;
    red[(warp * NQ + lane) * 4 + 2] = e2;
    red[(warp * NQ + lane) * 4 + 3] = e3;
  }
  __syncthreads();
  if (tid < G) {
    long long E = 0;
    for (uint32_t w = 0; w < nw; ++w) E += red[(w * NQ + tid / 4) * 4 + (tid & 3u)];
    const uint32_t r = r0 + tid;
    if (r < a.R) a.energies_out[r] = (float)((double)a.F.offset + (double)E * TAMC_FX_INV);
  }
  // states back in original site order
  const uint32_t keep = (a.R - r0 >= 32u) ? 0xffffffffu : ((1u << (a.R - r0)) - 1u);
  for (uint32_t s = tid; s < n; s += T) {
    const uint32_t v = (W[s] & (G < 32 ? ((1u << G) - 1u) : 0xffffffffu) & keep) << (r0 & 31u);
    uint32_t* dst = a.words_out + (size_t)(r0 >> 5) * n + a.F.perm[s];
    if (G == 32) *dst = v;
    else atomicOr(dst, v);
  }
}

// words [ceil(R/32)][n] (bit r%32 = replica r) -> packed [R][ceil(n/8)] bytes
// (bit i%8 of byte i/8 = site i), the IsingState::write_to_bytes layout
// (src/ising.rs:102-115).  One thread per output byte.
__global__ void k_pack_states(const uint32_t* __restrict__ words, uint32_t n, uint32_t R, uint8_t* __restrict__ out) {
  const uint32_t nb = (n + 7) / 8;
  const uint64_t x = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= (uint64_t)R * nb) return;
  const uint32_t r = (uint32_t)(x / nb), b = (uint32_t)(x % nb);
  const uint32_t* w = words + (size_t)(r >> 5) * n;
  uint32_t v = 0;
  for (uint32_t k = 0; k < 8 && 8 * b + k < n; ++k) v |= ((w[8 * b + k] >> (r & 31u)) & 1u) << k;
  out[x] = (uint8_t)v;
}

template <int NQ, bool SMEM, uint32_t DEG>
void launch_d(cudaStream_t st, const SaFastArgs& a, uint32_t ncta, uint32_t T, size_t smem) {
  auto k = k_sa_fast<NQ, SMEM, DEG>;
  TAMC_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k<<<ncta, T, smem, st>>>(a);
  TAMC_CUDA(cudaGetLastError());
}

// rows of uniform length 3, 4 or 6 (random regular graphs, square and cubic
// lattices) get an unrolled local field without row-pointer loads
template <int NQ, bool SMEM>
void launch_t(cudaStream_t st, const SaFastArgs& a, uint32_t ncta, uint32_t T, size_t smem) {
  switch (a.F.udeg) {
    case 3: launch_d<NQ, SMEM, 3>(st, a, ncta, T, smem); break;
    case 4: launch_d<NQ, SMEM, 4>(st, a, ncta, T, smem); break;
    case 6: launch_d<NQ, SMEM, 6>(st, a, ncta, T, smem); break;
    default: launch_d<NQ, SMEM, 0>(st, a, ncta, T, smem); break;
  }
}

}  // namespace

size_t sa_fast_smem(const FastInst& F, uint32_t nq, uint32_t T, bool smem_csr) {
  const size_t words = smem_csr ? (3ull * F.n + 2ull + 2ull * F.nnz) : (size_t)F.n;
  return ((words + 1) / 2 + 1) * 8 + (size_t)(T / 32) * nq * 4 * 8 + 16;
}

void sa_pack_states(cudaStream_t st, const uint32_t* words, uint32_t n, uint32_t R, uint8_t* out) {
  const uint64_t total = (uint64_t)R * ((n + 7) / 8);
  if (!total) return;
  k_pack_states<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(words, n, R, out);
  TAMC_CUDA(cudaGetLastError());
}

// Heuristic tile: 256 threads and the smallest replica group (quads per CTA)
// that gives no SM more than two CTAs.  (On 1024 restarts of a 2000-spin
// instance: 256 CTAs of 4 restarts, measured fastest of the 12 tiles.)
static SaTile heuristic(const tamc_gpu* g, const FastInst& F, uint32_t R) {
  SaTile t;
  t.T = 256;
  t.smem_csr = sa_fast_smem(F, 8, 1024, true) <= g->smem_optin;
  t.nq = 8;
  for (uint32_t nq : {1u, 2u, 4u, 8u}) {
    const uint32_t ncta = (R + 4 * nq - 1) / (4 * nq);
    if (ncta <= 2u * (uint32_t)g->num_sms) { t.nq = nq; break; }
  }
  t.smem = sa_fast_smem(F, t.nq, t.T, t.smem_csr);
  return t;
}

// Autotuner: times a short anneal (a few sweeps) of each candidate tile --
// replicas per CTA (4*nq) x CTA size -- on scratch buffers the first time a
// (device, n, nnz, R) shape is seen, and caches the fastest.  The choice does
// not change results: spins depend only on (seed, site, sweep, replica) and
// energies are fixed-point sums.
static std::mutex g_sa_mu;
static std::map<std::tuple<int, uint32_t, uint32_t, uint32_t>, SaTile> g_sa_tune;

SaTile sa_fast_choose(tamc_gpu* g, const FastInst& F, uint32_t R) {
  const auto key = std::make_tuple(g->device, F.n, F.nnz, R);
  {
    std::lock_guard<std::mutex> lk(g_sa_mu);
    auto it = g_sa_tune.find(key);
    if (it != g_sa_tune.end()) return it->second;
  }
  SaTile best = heuristic(g, F, R);
  const char* env = getenv("TAMC_AUTOTUNE");
  if ((!env || env[0] != '0') && R >= 64) {
    // long enough that the per-sweep cost, not the start-up, decides
    const uint32_t nb = 64;
    float* d_b = nullptr;
    float* d_e = nullptr;
    uint32_t* d_w = nullptr;
    TAMC_CUDA(cudaMalloc((void**)&d_b, nb * 4));
    TAMC_CUDA(cudaMalloc((void**)&d_e, (size_t)R * 4));
    TAMC_CUDA(cudaMalloc((void**)&d_w, (size_t)((R + 31) / 32) * F.n * 4));
    std::vector<float> hb(nb);
    for (uint32_t k = 0; k < nb; ++k) hb[k] = 0.1f + 9.9f * (float)k / (float)(nb - 1);  // an annealing ramp
    TAMC_CUDA(copy_sync(d_b, hb.data(), nb * 4, cudaMemcpyHostToDevice));
    cudaEvent_t e0, e1;
    TAMC_CUDA(cudaEventCreate(&e0));
    TAMC_CUDA(cudaEventCreate(&e1));
    float best_ms = 1e30f;
    for (uint32_t nq : {1u, 2u, 4u, 8u}) {
      for (uint32_t T : {128u, 256u, 512u, 1024u}) {
        SaTile t;
        t.nq = nq;
        t.T = T;
        t.smem_csr = best.smem_csr;
        t.smem = sa_fast_smem(F, nq, T, t.smem_csr);
        if (t.smem > g->smem_optin) continue;
        const uint32_t ncta = (R + 4 * nq - 1) / (4 * nq);
        if (ncta * 4 < (uint32_t)g->num_sms && nq > 1) continue;  // too few CTAs to fill the GPU
        SaFastArgs a;
        a.F = F;
        a.betas = d_b;
        a.nbeta = nb;
        a.key = make_uint2(1u, 2u);
        a.R = R;
        a.init_words = nullptr;
        a.words_out = d_w;
        a.energies_out = d_e;
        float ms = 1e30f;
        for (int rep = 0; rep < 3; ++rep) {  // the first run warms up; keep the fastest of the rest
          float m = 0.0f;
          TAMC_CUDA(cudaMemsetAsync(d_w, 0, (size_t)((R + 31) / 32) * F.n * 4, g->stream));
          TAMC_CUDA(cudaEventRecord(e0, g->stream));
          sa_fast_launch(g->stream, a, t);
          TAMC_CUDA(cudaEventRecord(e1, g->stream));
          g->count();
          TAMC_CUDA(cudaEventSynchronize(e1));
          TAMC_CUDA(cudaEventElapsedTime(&m, e0, e1));
          if (rep > 0) ms = std::min(ms, m);
        }
        if (ms < best_ms) {
          best_ms = ms;
          best = t;
        }
      }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(d_b);
    cudaFree(d_e);
    cudaFree(d_w);
  }
  if (const char* e = getenv("TAMC_SA_NQ")) {  // manual override (profiling)
    const int v = atoi(e);
    if (v == 1 || v == 2 || v == 4 || v == 8) best.nq = (uint32_t)v;
  }
  if (const char* e = getenv("TAMC_SA_T")) {
    const int v = atoi(e);
    if (v == 128 || v == 256 || v == 512 || v == 1024) best.T = (uint32_t)v;
  }
  best.smem = sa_fast_smem(F, best.nq, best.T, best.smem_csr);
  if (best.smem > g->smem_optin) fail(TAMC_E_UNSUPPORTED, "instance too large for the fast SA kernel");
  if (getenv("TAMC_DEBUG"))
    fprintf(stderr, "[tamc] SA tile n=%u R=%u: replicas/CTA=%u threads=%u csr_smem=%d smem=%zu\n", F.n, R,
            4 * best.nq, best.T, (int)best.smem_csr, best.smem);
  std::lock_guard<std::mutex> lk(g_sa_mu);
  g_sa_tune[key] = best;
  return best;
}

void sa_fast_launch(cudaStream_t st, const SaFastArgs& a, const SaTile& t) {
  const uint32_t G = 4 * t.nq;
  const uint32_t ncta = (a.R + G - 1) / G;
  if (!ncta) return;
  switch (t.nq * 2 + (t.smem_csr ? 1 : 0)) {
    case 2: launch_t<1, false>(st, a, ncta, t.T, t.smem); break;
    case 3: launch_t<1, true>(st, a, ncta, t.T, t.smem); break;
    case 4: launch_t<2, false>(st, a, ncta, t.T, t.smem); break;
    case 5: launch_t<2, true>(st, a, ncta, t.T, t.smem); break;
    case 8: launch_t<4, false>(st, a, ncta, t.T, t.smem); break;
    case 9: launch_t<4, true>(st, a, ncta, t.T, t.smem); break;
    case 16: launch_t<8, false>(st, a, ncta, t.T, t.smem); break;
    case 17: launch_t<8, true>(st, a, ncta, t.T, t.smem); break;
    default: fail(TAMC_E_INVAL, "bad SA tile");
  }
}

SaTile sa_fast_peek(const tamc_gpu* g, const FastInst& F, uint32_t R) {
  {
    std::lock_guard<std::mutex> lk(g_sa_mu);
    auto it = g_sa_tune.find(std::make_tuple(g->device, F.n, F.nnz, R));
    if (it != g_sa_tune.end()) return it->second;
  }
  return heuristic(g, F, R);
}

}  // namespace tamc
