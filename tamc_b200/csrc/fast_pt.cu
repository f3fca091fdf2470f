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

#include <cooperative_groups.h>
#include <map>
#include <mutex>
#include <numeric>

namespace cg = cooperative_groups;

namespace tamc {
namespace {

__device__ __forceinline__ uint64_t bitperm(uint64_t v, uint64_t D) {
  const uint64_t S = D & ~(D << 1);
  const uint64_t E = (D << 1) & ~D;
  return ((v >> 1) & D) | (((v & S) + D) & E) | (v & ~(D | (D << 1)));
}

// Phase cycle accounting (thread 0, after the phase's closing barrier).
struct PhaseClock {
  unsigned long long* out;
  long long t;
  __device__ __forceinline__ void start(unsigned long long* o) {
    out = o;
    if (out && threadIdx.x == 0) t = clock64();
  }
  __device__ __forceinline__ void lap(int phase) {
    if (out && threadIdx.x == 0) {
      const long long now = clock64();
      atomicAdd(&out[phase], (unsigned long long)(now - t));
      t = now;
    }
  }
};

__device__ __forceinline__ float u24(uint32_t r) { return (float)(r >> 8) * (1.0f / 16777216.0f); }

// Scratch of one ICM group (all in shared memory).
struct IcmScratch {
  uint32_t* D;     // [n] disagreement bits of the group's slots
  uint32_t* Cl;    // [n] cluster bits
  uint32_t* L;     // union-find: [G][n] labels; several-slot BFS: [n] level marks, then two frontiers
                   // and the visited list as 16-bit site lists; one-slot BFS: [n] queue; propagation: unused
  uint32_t* cnt;   // [32] q<0 counts per bit
  uint32_t* seed;  // [32] seed site per bit
  uint32_t* gidx;  // [32] label-array index per bit
  unsigned long long* dE;  // [2][32] fixed-point energy change per chain and bit
  uint32_t* red;   // [32] block reduction scratch
  long long* part; // [32 warps][2] per-warp partial sums
  uint32_t* q;     // [4] BFS counters: frontier sizes (three, by level mod 3), visited count
};

struct Smem {
  uint32_t* W;
  IcmScratch X;
  double* Ec;
  double* Er;
  float4* beta4;
  float4* red;
  float4* redq;
  unsigned long long* Dm;
  uint32_t* rp;
  float* bias;
  uint2* ent;
  uint32_t* msc;  // multi-spin coding: per word [3][32] threshold planes, then [3] always, [3] never
  // fused kernel: the exchange bookkeeping and the ground-state log's running
  // minimum in shared memory for a range of rounds (XchgSm below); null in the
  // plain form, which uses the job's global arrays
  char* xb;
};

// Shared-memory copies of a fused job's exchange bookkeeping and of its
// ground-state minimum, loaded at the start of a range of rounds and stored at
// its end (no global round trips inside a round).  One base pointer: the
// fields are found by offsets, which keeps the kernel's register budget.
struct GsMin {
  int have;
  float minE;
  uint32_t count;
};
struct XchgSm {
  uint8_t* tags;    // [C][nt]
  uint32_t* acc;    // [C][nt]
  uint32_t* dhist;  // [C][nt][2]
  uint32_t* rtrips; // [C]
  float* dbeta;     // [nt - 1] beta[j + 1] - beta[j] (f32)
  GsMin* gs;
};
__host__ __device__ inline size_t xchg_layout(XchgSm* X, char* base, uint32_t C, uint32_t nt) {
  size_t o = 0;
  auto take = [&](size_t bytes) {
    char* p = base ? base + o : nullptr;
    o = (o + bytes + 15) & ~(size_t)15;
    return p;
  };
  const size_t CT = (size_t)C * nt;
  char* tags = take(CT);
  char* acc = take(CT * 4);
  char* dhist = take(CT * 8);
  char* rtrips = take((size_t)C * 4);
  char* dbeta = take((size_t)nt * 4);
  char* gs = take(sizeof(GsMin));
  if (X) {
    X->tags = (uint8_t*)tags;
    X->acc = (uint32_t*)acc;
    X->dhist = (uint32_t*)dhist;
    X->rtrips = (uint32_t*)rtrips;
    X->dbeta = (float*)dbeta;
    X->gs = (GsMin*)gs;
  }
  return o;
}

// words of multi-spin-coding thresholds per replica word (levels x < 3):
// [3][32] planes, [3] always, [3] never, padded so that every word's planes
// start on a 16-byte boundary (msc_step4 loads four planes at once)
constexpr uint32_t MSC_WORDS = 3 * 32 + 3 + 3 + 2;
static_assert(MSC_WORDS % 4 == 0, "16-byte aligned threshold planes");

__host__ __device__ inline size_t al16(size_t x) { return (x + 15) & ~(size_t)15; }

// Label region (32-bit words) by cluster search:
//   ICM_UF       G label arrays of n words;
//   ICM_BFS      (several slots) level marks [n] u32, then two frontiers and the
//                visited list as 16-bit site indices (n <= 65536);
//   ICM_BFS_ONE  (one slot) the queue of visited sites [n] u32.
enum { ICM_UF = 0, ICM_BFS = 1, ICM_BFS_ONE = 2 };
__host__ __device__ inline size_t icm_n16(uint32_t n) { return ((size_t)n + 7) / 8 * 8; }
// (ICM_UF and ICM_BFS also hold the several-slot seed scan's transposed chunk
// masks first: at least 32 words per chunk of 32 sites.)
__host__ __device__ inline size_t icm_label_words(uint32_t n, uint32_t G, int mode) {
  const size_t chunks = ((size_t)n + 31) / 32 * 32;
  if (mode == ICM_UF) return (size_t)G * n > chunks ? (size_t)G * n : chunks;
  if (mode == ICM_BFS) return (size_t)n + 3 * icm_n16(n) / 2 > chunks ? (size_t)n + 3 * icm_n16(n) / 2 : chunks;
  return n;
}

__host__ __device__ inline size_t carve_icm(IcmScratch* X, char* base, size_t o, uint32_t n, uint32_t G, int mode) {
  auto take = [&](size_t bytes) {
    char* p = base ? base + o : nullptr;
    o = al16(o + bytes);
    return p;
  };
  char* D = take((size_t)n * 4);
  char* Cl = take((size_t)n * 4);
  char* L = take(icm_label_words(n, G, mode) * 4);
  char* cnt = take(32 * 4);
  char* seed = take(32 * 4);
  char* gidx = take(32 * 4);
  char* dE = take(64 * 8);
  char* red = take(32 * 4);
  char* part = take(64 * 8);
  char* q = take(4 * 4);
  if (X) {
    X->D = (uint32_t*)D;
    X->Cl = (uint32_t*)Cl;
    X->L = (uint32_t*)L;
    X->cnt = (uint32_t*)cnt;
    X->seed = (uint32_t*)seed;
    X->gidx = (uint32_t*)gidx;
    X->dE = (unsigned long long*)dE;
    X->red = (uint32_t*)red;
    X->part = (long long*)part;
    X->q = (uint32_t*)q;
  }
  return o;
}

__host__ __device__ inline size_t carve_all(Smem* S, char* base, uint32_t n, uint32_t nw, uint32_t C, uint32_t ntp,
                                            uint32_t qps, uint32_t T, uint32_t nnz, bool csr, uint32_t G,
                                            bool uf) {
  size_t o = 0;
  auto take = [&](size_t bytes) {
    char* p = base ? base + o : nullptr;
    o = al16(o + bytes);
    return p;
  };
  char* W = take((size_t)n * nw * 4);
  IcmScratch X;
  o = carve_icm(&X, base, o, n, G, uf ? ICM_UF : ICM_BFS);
  char* Ec = take((size_t)C * ntp * 8);
  char* Er = take((size_t)C * ntp * 8);
  char* b4 = take((size_t)qps * 16);
  char* red = take((size_t)T * 16);
  char* redq = take((size_t)T * 16);
  char* Dm = take((size_t)C * 8);
  char* msc = take((size_t)nw * MSC_WORDS * 4);
  char* xb = take(xchg_layout(nullptr, nullptr, C, ntp));
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
    S->X = X;
    S->Ec = (double*)Ec;
    S->Er = (double*)Er;
    S->beta4 = (float4*)b4;
    S->red = (float4*)red;
    S->redq = (float4*)redq;
    S->Dm = (unsigned long long*)Dm;
    S->msc = (uint32_t*)msc;
    S->xb = xb;
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

// ------------------------------------------------------------------ ICM ----
// Connected components of the subgraph where the two replicas of a slot
// disagree, by union-find in rounds (Shiloach-Vishkin style): labels are site
// indices, every label points to a smaller-or-equal index (a root is its own
// label), pointer jumping turns the trees into stars, and hooking links the
// larger of two adjacent roots under the smaller with atomicMin.  A hook that
// lands on a root another thread has already hooked in the same round may
// drop that link; the edge still joins two labels afterwards and is hooked
// again in the next round.  Every round removes at least one root, so the
// rounds end within n + 1, and the final labels are the smallest site index
// of each component whatever the thread schedule was.

// Houdayer move (src/pt.rs:31-77) for the slots of `gmask` (bits of word w)
// of chain pair (c0, c1) at sweep i: count the q<0 sites of every slot, draw
// the seed index from Philox, find the seed's component of the q<0 subgraph,
// accumulate the energy change of flipping it in both replicas (boundary
// terms, fixed point), and flip.  The component is found either by a
// level-synchronous BFS from the seeds of all slots at once (bit-parallel:
// the cluster word of a site carries one bit per slot, and only cluster
// sites and their edges are touched) or by union-find labelling of the whole
// subgraph (J.icm_uf).  Both give the exact component, so the result depends
// only on the replica state, the seed and the sweep index -- not on the
// algorithm, the number of threads or how slots are grouped -- and the fused
// and plain forms agree.
// Instances of at most 4 sites per thread use in-place propagation instead of
// a BFS (whole-graph passes, no frontier lists).
// PLAIN: the one-slot-per-CTA kernel of the plain form, which gets the
// single-slot queue search and batched edge loads; the fused kernel keeps the
// general paths (it runs at its register limit).
// OR of the cluster words of the DEG neighbours of s (rows of DEG entries).
template <uint32_t DEG, typename Col>
__device__ __forceinline__ uint32_t nb_or(uint32_t s, const uint32_t* XC, Col col) {
  uint32_t j[DEG];
#pragma unroll
  for (uint32_t k = 0; k < DEG; ++k) j[k] = col(DEG * s + k);
  uint32_t nb = 0;
#pragma unroll
  for (uint32_t k = 0; k < DEG; ++k) nb |= XC[j[k]];
  return nb;
}

// In-place propagation passes (see icm_group) for rows of DEG entries and at
// most PS sites per thread.  What does not change between passes stays in
// registers: each site's disagreement word, its cluster word (only this
// thread writes it) and its neighbours' columns, two 16-bit columns per
// register (n <= 4 T <= 4096).  A pass then loads only the neighbours'
// cluster words and stores the words that grew.  CHAIN: site after site, so
// a site sees what this thread's earlier sites gained in the same pass (with
// checkerboard colour order a thread's sites alternate colours, and a pass
// then advances two hops; measured faster than issuing all loads first).
template <uint32_t DEG, uint32_t PS, bool CHAIN, typename Col>
__device__ __forceinline__ void prop_passes(uint32_t n, uint32_t T, uint32_t tid, const uint32_t* XD, uint32_t* XC,
                                            Col col) {
  constexpr uint32_t NP = DEG / 2;
  uint32_t d[PS], c[PS], jp[PS][NP];
#pragma unroll
  for (uint32_t k = 0; k < PS; ++k) {
    const uint32_t s = tid + k * T;
    d[k] = 0;
    c[k] = 0;
#pragma unroll
    for (uint32_t m = 0; m < NP; ++m) jp[k][m] = 0;
    if (s < n) {
      d[k] = XD[s];
      c[k] = XC[s];
#pragma unroll
      for (uint32_t m = 0; m < NP; ++m) jp[k][m] = col(DEG * s + 2 * m) | (col(DEG * s + 2 * m + 1) << 16);
    }
  }
  for (uint32_t pass = 0; pass < 32u * n + 2u; ++pass) {
    uint32_t nb[PS];
    int grew = 0;
#pragma unroll
    for (uint32_t k = 0; k < PS; ++k) {
      nb[k] = 0;
      if ((c[k] & d[k]) != d[k]) {
#pragma unroll
        for (uint32_t m = 0; m < NP; ++m) nb[k] |= XC[jp[k][m] & 0xffffu] | XC[jp[k][m] >> 16];
      }
      if (CHAIN) {
        const uint32_t nc = c[k] | (nb[k] & d[k]);
        if (nc != c[k]) {
          XC[tid + k * T] = nc;
          c[k] = nc;
          grew = 1;
        }
      }
    }
    if (!CHAIN) {
#pragma unroll
      for (uint32_t k = 0; k < PS; ++k) {
        const uint32_t nc = c[k] | (nb[k] & d[k]);
        if (nc != c[k]) {
          XC[tid + k * T] = nc;
          c[k] = nc;
          grew = 1;
        }
      }
    }
    if (!__syncthreads_or(grew)) break;
  }
}

// Energy change of flipping the clusters XC of the slots in gmask, for +-J
// instances (rows of DEG entries, J = +-1, no field): a boundary bond (s in
// the slot's cluster, j outside) that is unsatisfied in replica 0
// (J s_s s_j = +1) changes by -2 when the cluster flips, a satisfied one by
// +2.  Each lane takes a site; per slot bit, the counts of both kinds over the
// site's bonds are bit-sliced (3 planes each), transposed across the warp
// (lane b then holds slot b's counts over the warp's 32 sites) and added to
// X.dE[b] (64-bit shared atomics; integer sums, so in any order); replica 1's
// change is the negative.  X.dE must be zero on entry.
template <uint32_t DEG, typename R0>
__device__ __noinline__ void icm_energy_msc(uint32_t n, const uint32_t* XC, const uint2* __restrict__ ent, R0 r0,
                                               uint32_t gmask, IcmScratch& X) {
  const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5, nwarp = blockDim.x >> 5;
  long long acc = 0;
  for (uint32_t base = warp * 32u; base < n; base += nwarp * 32u) {
    const uint32_t s = base + lane;
    uint32_t p0 = 0, p1 = 0, p2 = 0, q0 = 0, q1 = 0, q2 = 0;  // satisfied / unsatisfied boundary bonds
    const uint32_t cs = s < n ? XC[s] : 0u;
    if (cs) {
      const uint32_t rs = r0(s);
#pragma unroll
      for (uint32_t m = 0; m < DEG; ++m) {
        const uint2 ce = ent[s * DEG + m];
        const uint32_t B = cs & ~XC[ce.x];
        const uint32_t U = ~(rs ^ r0(ce.x) ^ (0u - (ce.y >> 31)));
        const uint32_t a = B & ~U, b = B & U;
        uint32_t c = p0 & a;
        p0 ^= a;
        p2 ^= p1 & c;
        p1 ^= c;
        c = q0 & b;
        q0 ^= b;
        q2 ^= q1 & c;
        q1 ^= c;
      }
    }
    const int dp = __popc(transpose32(p0, lane)) + 2 * __popc(transpose32(p1, lane)) +
                   4 * __popc(transpose32(p2, lane));
    const int dq = __popc(transpose32(q0, lane)) + 2 * __popc(transpose32(q1, lane)) +
                   4 * __popc(transpose32(q2, lane));
    acc += (long long)(2 * (dp - dq)) * 4294967296ll;
  }
  if (((gmask >> lane) & 1u) && acc) atomicAdd(&X.dE[lane], (unsigned long long)acc);
  __syncthreads();
  if (tid < 32 && ((gmask >> tid) & 1u)) X.dE[32 + tid] = (unsigned long long)(-(long long)X.dE[tid]);
  __syncthreads();
}

template <bool PLAIN>
__device__ void icm_group(const PtJob& J, const FastInst& F, uint32_t* W, IcmScratch& X, uint32_t i, uint32_t p,
                          uint32_t w, uint32_t gmask, const uint16_t* cols = nullptr, uint32_t* wstage = nullptr,
                          PhaseClock* pc = nullptr) {
  const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5, nwarp = blockDim.x >> 5;
  const uint32_t n = J.n, T = blockDim.x, nw = J.nw;
  const uint32_t o0 = 2 * p * J.wpc + w, o1 = (2 * p + 1) * J.wpc + w, tb = 32 * w;
  // loop-invariant pointers in registers (stores through the label arrays
  // would otherwise force reloads of the descriptors)
  const uint32_t* __restrict__ rp = F.rp;
  const uint2* __restrict__ ent = F.ent;
  const float* __restrict__ bias = F.bias;
  uint32_t* const XD = X.D;
  uint32_t* const XC = X.Cl;
  uint32_t* const XL = X.L;
  const bool uf = J.icm_uf != 0;
  const bool prop = !uf && n <= 4 * T;  // propagation instead of BFS on small instances
  // replica 0's words, read once (kept in shared memory when W is not); the
  // energy change needs no other replica words
  auto r0 = [&](uint32_t s) -> uint32_t { return wstage ? wstage[s] : W[s * nw + o0]; };
  if (pc) pc->lap(PHASE_OTHER);
  for (uint32_t s = tid; s < n; s += T) {
    const uint32_t v0 = W[s * nw + o0], v1 = W[s * nw + o1];
    if (wstage) wstage[s] = v0;
    XD[s] = (v0 ^ v1) & gmask;
    XC[s] = 0;
    if (!uf && !PLAIN) XL[s] = 0;  // level marks of the multi-slot search (ICM_BFS layout)
  }
  if (tid < 4) X.q[tid] = 0;
  if (tid < 32) {
    X.cnt[tid] = 0;
    X.seed[tid] = 0xffffffffu;
    X.gidx[tid] = __popc(gmask & ((1u << tid) - 1u));
  }
  if (tid < 64) X.dE[tid] = 0;
  __syncthreads();
  if (pc && !uf) pc->lap(PHASE_ICM_INIT);
  const uint32_t G = __popc(gmask);
  if (G == 1) {
    // one slot: each warp counts a contiguous segment of sites with ballots,
    // one warp-wide prefix sum over the segment counts orders them, and the
    // warp whose segment holds the k-th q<0 site finds it
    const uint32_t b = __ffs(gmask) - 1;
    const uint32_t seg = ((n + nwarp - 1) / nwarp + 31u) & ~31u;
    const uint32_t w0 = min(n, warp * seg), w1 = min(n, w0 + seg);
    uint32_t wc = 0;
    for (uint32_t base = w0; base < w1; base += 32) {
      const uint32_t s = base + lane;
      wc += __popc(__ballot_sync(0xffffffffu, s < w1 && ((XD[s] >> b) & 1u)));
    }
    if (lane == 0) X.red[warp] = wc;
    __syncthreads();
    const uint32_t v = lane < nwarp ? X.red[lane] : 0u;
    uint32_t incl = v;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= (uint32_t)o) incl += y;
    }
    const uint32_t cnt = __shfl_sync(0xffffffffu, incl, 31);
    const uint32_t before = __shfl_sync(0xffffffffu, incl - v, warp);
    if (cnt) {
      const uint32_t u = philox4x32_10(make_uint4(tb + b, i, p, PTAG_ICM), J.key).x;
      const uint32_t k = (uint32_t)(((uint64_t)u * cnt) >> 32);
      if (k >= before && k < before + wc) {
        uint32_t r = k - before;
        for (uint32_t base = w0; base < w1; base += 32) {
          const uint32_t s = base + lane;
          const uint32_t bal = __ballot_sync(0xffffffffu, s < w1 && ((XD[s] >> b) & 1u));
          const uint32_t c = __popc(bal);
          if (r < c) {
            if (lane == 0) X.seed[b] = base + __fns(bal, 0, (int)r + 1);
            break;
          }
          r -= c;
        }
      }
      if (tid == 0) X.cnt[b] = cnt;
    }
  } else {
    // several slots: the (gmask-masked) disagreement words of 32 consecutive
    // sites are transposed in a warp, so lane b holds slot b's bits of those
    // sites; the masks go to XL as [chunk][32].  Then one warp per slot counts
    // its sites (lane = chunk, in groups of 32 chunks), draws k and finds the
    // chunk holding the k-th site by a prefix sum over the lanes and the site
    // by __fns: the site a scan in site order would find.
    const uint32_t nchunk = (n + 31) / 32;
    uint32_t* const M = XL;  // 32 * nchunk words (icm_label_words)
    for (uint32_t ch = warp; ch < nchunk; ch += nwarp) {
      const uint32_t s = ch * 32 + lane;
      M[ch * 32 + lane] = transpose32(s < n ? XD[s] : 0u, lane);
    }
    __syncthreads();
    for (uint32_t b = warp; b < 32; b += nwarp) {
      if (!((gmask >> b) & 1u)) continue;
      const uint32_t u = philox4x32_10(make_uint4(tb + b, i, p, PTAG_ICM), J.key).x;  // needed only if cnt > 0
      uint32_t cnt = 0;
      for (uint32_t c0 = 0; c0 < nchunk; c0 += 32) {
        const uint32_t ch = c0 + lane;
        cnt += ch < nchunk ? (uint32_t)__popc(M[ch * 32 + b]) : 0u;
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
      if (cnt == 0) continue;
      uint32_t k = (uint32_t)(((uint64_t)u * cnt) >> 32);
      for (uint32_t c0 = 0; c0 < nchunk; c0 += 32) {
        const uint32_t ch = c0 + lane;
        const uint32_t m = ch < nchunk ? M[ch * 32 + b] : 0u;
        const uint32_t cc = __popc(m);
        uint32_t incl = cc;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= (uint32_t)o) incl += v;
        }
        const uint32_t tot = __shfl_sync(0xffffffffu, incl, 31);
        if (k < tot) {  // warp-uniform
          const uint32_t excl = incl - cc;
          if (k >= excl && k < incl) {  // exactly one lane
            X.seed[b] = ch * 32 + __fns(m, 0, (int)(k - excl) + 1);
            X.cnt[b] = cnt;
          }
          break;
        }
        k -= tot;
      }
    }
  }
  __syncthreads();
  if (!PLAIN && G > 1 && !uf && !prop) {
    // the breadth-first search's level marks, which the scan's masks overwrote
    for (uint32_t s = tid; s < n; s += T) XL[s] = 0;
    __syncthreads();
  }
  if (pc) pc->lap(PHASE_ICM_SCAN);
  auto col = [&](uint32_t e) -> uint32_t { return cols ? cols[e] : ent[e].x; };
  // BFS: the cluster sites (16-bit list for several slots, 32-bit for one);
  // union-find: all sites
  const uint16_t* vlist16 = nullptr;
  const uint32_t* vlist = nullptr;
  if (uf) {
    // union-find labelling of the q<0 subgraph of every slot of the group:
    // (1) every site starts as a child of its smallest lower-index neighbour in
    //     the subgraph, or as its own root;
    // (2) rounds of pointer jumping (until every tree is a star) and hooking
    //     (each subgraph edge whose ends carry different labels links the
    //     larger label under the smaller), until no edge joins two labels.
    for (uint32_t x = tid; x < G * n; x += T) XL[x] = x % n;
    __syncthreads();
    for (uint32_t s = tid; s < n; s += T) {
      const uint32_t d = XD[s];
      if (!d) continue;
      const uint32_t e1 = rp[s + 1];
      for (uint32_t e = rp[s]; e < e1; ++e) {
        const uint32_t j = col(e);
        if (j >= s) continue;  // only this thread writes row s of every label array
        uint32_t m = d & XD[j];
        while (m) {
          const uint32_t b = __ffs(m) - 1;
          m &= m - 1;
          uint32_t* l = XL + X.gidx[b] * n + s;
          if (j < *l) *l = j;
        }
      }
    }
    __syncthreads();
    if (pc) pc->lap(PHASE_ICM_INIT);
    for (uint32_t round = 0; round <= n; ++round) {
      for (uint32_t it = 0; it <= n; ++it) {
        int ch = 0;
        for (uint32_t x = tid; x < G * n; x += T) {
          const uint32_t l = XL[x];
          const uint32_t base = x - x % n;
          const uint32_t ll = XL[base + l];
          if (ll != l) {
            XL[x] = ll;
            ch = 1;
          }
        }
        if (!__syncthreads_or(ch)) break;
      }
      if (pc) pc->lap(PHASE_ICM_JUMP);
      int ch = 0;
      for (uint32_t s = tid; s < n; s += T) {
        const uint32_t d = XD[s];
        if (!d) continue;
        const uint32_t e1 = rp[s + 1];
        for (uint32_t e = rp[s]; e < e1; ++e) {
          const uint32_t j = col(e);
          if (j <= s) continue;  // every undirected edge once; self-loops skipped
          uint32_t m = d & XD[j];
          while (m) {
            const uint32_t b = __ffs(m) - 1;
            m &= m - 1;
            uint32_t* L = XL + X.gidx[b] * n;
            const uint32_t a = L[s], c = L[j];
            if (a != c) {
              atomicMin(L + max(a, c), min(a, c));
              ch = 1;
            }
          }
        }
      }
      const int any = __syncthreads_or(ch);
      if (pc) pc->lap(PHASE_ICM_GROW);
      if (!any) break;
    }
    // root of every seed, then the cluster: q<0 sites in the seed's component
    if (tid < 32 && ((gmask >> tid) & 1u) && X.cnt[tid]) X.seed[tid] = XL[X.gidx[tid] * n + X.seed[tid]];
    __syncthreads();
    for (uint32_t s = tid; s < n; s += T) {
      uint32_t d = XD[s], c = 0;
      while (d) {
        const uint32_t b = __ffs(d) - 1;
        d &= d - 1;
        if (X.cnt[b] && XL[X.gidx[b] * n + s] == X.seed[b]) c |= 1u << b;
      }
      XC[s] = c;
    }
    __syncthreads();
    if (pc) pc->lap(PHASE_ICM_MARK);
  } else if (prop) {
    // Small instances (at most 4 sites per thread): in-place propagation.  Each
    // pass, every site still missing some of its q<0 slots takes the cluster
    // bits of its neighbours (C[s] |= D[s] & OR_j C[j]); only the site's thread
    // writes C[s], and a neighbour's word can only have gained bits, so reading
    // it mid-pass is safe and lets a pass advance more than one hop.  Passes end
    // when one changes nothing (each changing pass adds a bit: at most 32 n).
    // Whole-graph passes cost a fixed few loads per thread, where a frontier
    // level pays a chain of shared atomics and appends.
    if (tid < 32 && ((gmask >> tid) & 1u) && X.cnt[tid]) atomicOr(&XC[X.seed[tid]], 1u << tid);
    __syncthreads();
    // Square and cubic lattices: per-thread state in registers (the fused
    // kernel has registers for 2 sites of 4 entries per thread); otherwise
    // rows of 4 or 6 entries still load all their columns, then all the
    // neighbours' words, before use.
    const uint32_t udeg = F.udeg;
    if (PLAIN && udeg == 4) {
      prop_passes<4, 4, true>(n, T, tid, XD, XC, col);
    } else if (PLAIN && udeg == 6) {
      prop_passes<6, 4, true>(n, T, tid, XD, XC, col);
    } else if (!PLAIN && udeg == 4 && n <= 2 * T) {
      prop_passes<4, 2, true>(n, T, tid, XD, XC, col);
    } else {
      for (uint32_t pass = 0; pass < 32u * n + 2u; ++pass) {
        int grew = 0;
        for (uint32_t s = tid; s < n; s += T) {
          const uint32_t d = XD[s];
          const uint32_t c = XC[s];
          if ((c & d) == d) continue;
          uint32_t nb = 0;
          if (udeg == 4) {
            nb = nb_or<4>(s, XC, col);
          } else if (udeg == 6) {
            nb = nb_or<6>(s, XC, col);
          } else {
            const uint32_t e1 = rp[s + 1];
            for (uint32_t e = rp[s]; e < e1; ++e) nb |= XC[col(e)];
          }
          const uint32_t nc = c | (nb & d);
          if (nc != c) {
            XC[s] = nc;
            grew = 1;
          }
        }
        if (!__syncthreads_or(grew)) break;
      }
    }
    if (pc) pc->lap(PHASE_ICM_GROW);
  } else if (PLAIN && G == 1) {
    // One slot: a site joins the cluster exactly once (the atomicOr that sets
    // its bit tells which thread got there first), so the levels are
    // consecutive segments of one queue V, which ends up listing the cluster.
    // Counters rotate over three entries as in the multi-slot search below.
    uint32_t* const V = XL;
    const uint32_t b = __ffs(gmask) - 1, bit = 1u << b;
    if (tid == 0 && X.cnt[b]) {
      XC[X.seed[b]] = bit;
      V[0] = X.seed[b];
      X.q[0] = 1;
    }
    __syncthreads();
    constexpr uint32_t BFS_LANES = 4;
    const uint32_t lt = (1u << lane) - 1u;
    uint32_t lo = 0;
    for (uint32_t lvl = 0; lvl < n + 2u; ++lvl) {
      const uint32_t ncur = X.q[lvl % 3u];
      if (ncur == 0) break;
      uint32_t* qn = &X.q[(lvl + 1u) % 3u];
      uint32_t* nxt = V + lo + ncur;
      const uint32_t items = ncur * BFS_LANES;
      for (uint32_t base = warp * 32u; base < items; base += T) {  // warp-uniform trip count
        const uint32_t x = base + lane;
        uint32_t e = 0, e1 = 0;
        if (x < items) {
          const uint32_t s = V[lo + x / BFS_LANES];
          e = rp[s] + x % BFS_LANES;
          e1 = rp[s + 1];
        }
        const uint32_t steps = __reduce_max_sync(0xffffffffu, e < e1 ? (e1 - e + BFS_LANES - 1) / BFS_LANES : 0u);
        for (uint32_t r = 0; r < steps; ++r, e += BFS_LANES) {
          uint32_t j = 0;
          bool pq = false;
          if (e < e1) {
            j = col(e);
            if ((XD[j] & bit) && !(XC[j] & bit)) pq = !(atomicOr(&XC[j], bit) & bit);
          }
          const uint32_t bq = __ballot_sync(0xffffffffu, pq);
          uint32_t oq = 0;
          if (lane == 0 && bq) oq = atomicAdd(qn, (uint32_t)__popc(bq));
          oq = __shfl_sync(0xffffffffu, oq, 0);
          if (pq) nxt[oq + __popc(bq & lt)] = j;
        }
      }
      lo += ncur;
      if (tid == 0) X.q[(lvl + 2u) % 3u] = 0;
      __syncthreads();
    }
    if (tid == 0) X.q[3] = lo;
    __syncthreads();
    vlist = V;
    if (pc) pc->lap(PHASE_ICM_GROW);
  } else {
    // BFS from the seeds of all slots, one level per barrier.  XC[s] holds the
    // slots whose cluster contains s; a site is queued for the next level when
    // it gains a slot bit (at most once per level: level marks), and listed
    // in V the first time it gains any.  Frontier counters rotate over three
    // entries so that one barrier per level separates reading, filling and
    // clearing them.  A level runs only if the previous one added a (site,
    // slot) pair, so the levels end within 32 n.
    uint32_t* const MK = XL;
    uint16_t* const F0 = reinterpret_cast<uint16_t*>(XL + n);
    uint16_t* const F1 = F0 + icm_n16(n);
    uint16_t* const V = F1 + icm_n16(n);
    if (tid < 32 && ((gmask >> tid) & 1u) && X.cnt[tid]) {
      const uint32_t s0 = X.seed[tid];
      const uint32_t old = atomicOr(&XC[s0], 1u << tid);
      if (old == 0) V[atomicAdd(&X.q[3], 1u)] = (uint16_t)s0;
      if (atomicMax(&MK[s0], 1u) < 1u) F0[atomicAdd(&X.q[0], 1u)] = (uint16_t)s0;
    }
    __syncthreads();
    // Each frontier site is expanded by a team of BFS_LANES lanes (one edge
    // each per step), and the appends to the next frontier and to V are
    // aggregated per warp (one shared atomic per warp and step).
    constexpr uint32_t BFS_LANES = 4;
    const uint32_t lt = (1u << lane) - 1u;
    for (uint32_t lvl = 0; lvl < 32u * n + 2u; ++lvl) {
      const uint32_t ncur = X.q[lvl % 3u];
      if (ncur == 0) break;
      const uint16_t* cur = (lvl & 1u) ? F1 : F0;
      uint16_t* nxt = (lvl & 1u) ? F0 : F1;
      uint32_t* qn = &X.q[(lvl + 1u) % 3u];
      const uint32_t mark = lvl + 2u;
      const uint32_t items = ncur * BFS_LANES;
      for (uint32_t base = warp * 32u; base < items; base += T) {  // warp-uniform trip count
        const uint32_t x = base + lane;
        uint32_t c = 0, e = 0, e1 = 0;
        if (x < items) {
          const uint32_t s = cur[x / BFS_LANES];
          c = XC[s];
          e = rp[s] + x % BFS_LANES;
          e1 = rp[s + 1];
        }
        const uint32_t steps = __reduce_max_sync(0xffffffffu, e < e1 ? (e1 - e + BFS_LANES - 1) / BFS_LANES : 0u);
        for (uint32_t r = 0; r < steps; ++r, e += BFS_LANES) {
          uint32_t j = 0;
          bool pq = false, pv = false;
          if (e < e1) {
            j = col(e);
            const uint32_t nb = c & XD[j] & ~XC[j];
            if (nb) {
              const uint32_t old = atomicOr(&XC[j], nb);
              if (nb & ~old) {
                pv = old == 0;
                pq = atomicMax(&MK[j], mark) < mark;
              }
            }
          }
          const uint32_t bq = __ballot_sync(0xffffffffu, pq), bv = __ballot_sync(0xffffffffu, pv);
          uint32_t oq = 0, ov = 0;
          if (lane == 0) {
            if (bq) oq = atomicAdd(qn, (uint32_t)__popc(bq));
            if (bv) ov = atomicAdd(&X.q[3], (uint32_t)__popc(bv));
          }
          oq = __shfl_sync(0xffffffffu, oq, 0);
          ov = __shfl_sync(0xffffffffu, ov, 0);
          if (pq) nxt[oq + __popc(bq & lt)] = (uint16_t)j;
          if (pv) V[ov + __popc(bv & lt)] = (uint16_t)j;
        }
      }
      if (tid == 0) X.q[(lvl + 2u) % 3u] = 0;
      __syncthreads();
    }
    vlist16 = V;
    if (pc) pc->lap(PHASE_ICM_GROW);
  }
  const uint32_t nlist = (uf || prop) ? n : X.q[3];
  if (!PLAIN && F.pmj) {
    // +-J instances: the boundary terms of every slot of the group at once,
    // 32 sites per warp step (exact integers, so the same fixed-point sums)
    if (F.udeg == 4) icm_energy_msc<4>(n, XC, ent, r0, gmask, X);
    else icm_energy_msc<6>(n, XC, ent, r0, gmask, X);
  } else
  // energy change of flipping each cluster in both replicas: boundary terms
  // -2 s_i (h_i + sum_{j not in cluster} J_ij s_j), f32 per site, summed in
  // fixed point per slot.  The slots are dealt to teams of warps (all warps
  // for one slot, one warp per slot for many); each warp reduces by shuffles
  // and a team combines its warps in a fixed order.
  // Only replica 0's sum is formed: the cluster is the whole component of the
  // seed among the sites where the replicas differ, so every neighbour j
  // outside it has the same spin in both replicas while every cluster site
  // has opposite spins.  Replica 1's field at i is therefore the same float
  // sum in the same order and its term is the exact negative (conversion to
  // fixed point rounds symmetrically), so its sum is -a0, bit for bit.
  {
    const uint32_t team = max(1u, nwarp / G), teams = nwarp / team;
    const uint32_t tw = warp % team, tid_team = warp / team;
    const uint32_t iters = (G + teams - 1) / teams;
    for (uint32_t it = 0; it < iters; ++it) {
      const uint32_t g = it * teams + tid_team;
      long long a0 = 0, a1 = 0;
      uint32_t b = 32;
      if (g < G && tid_team < teams) {
        b = __fns(gmask, 0, (int)g + 1);
        if (X.cnt[b]) {
          for (uint32_t x = tw * 32 + lane; x < nlist; x += team * 32) {
            const uint32_t s = vlist ? vlist[x] : vlist16 ? (uint32_t)vlist16[x] : x;
            if (!((XC[s] >> b) & 1u)) continue;
            float f0 = bias[s];
            const uint32_t e1 = rp[s + 1];
            if (!PLAIN && F.udeg == 4) {
              // square-lattice rows: all four entries, cluster words and spins
              // loaded before use, then summed in row order
              uint2 ce[4];
              uint32_t xc[4], wv[4];
#pragma unroll
              for (uint32_t k = 0; k < 4; ++k) ce[k] = ent[4 * s + k];
#pragma unroll
              for (uint32_t k = 0; k < 4; ++k) {
                xc[k] = XC[ce[k].x];
                wv[k] = r0(ce[k].x);
              }
#pragma unroll
              for (uint32_t k = 0; k < 4; ++k) {
                if (ce[k].x == s || ((xc[k] >> b) & 1u)) continue;
                const float Jv = __uint_as_float(ce[k].y);
                f0 += ((wv[k] >> b) & 1u) ? -Jv : Jv;
              }
            } else if (!PLAIN) {
              // other rows: one entry at a time (the fused kernel has no
              // registers for batched loads)
              for (uint32_t e = rp[s]; e < e1; ++e) {
                const uint2 ce = ent[e];
                if (ce.x == s || ((XC[ce.x] >> b) & 1u)) continue;
                const float Jv = __uint_as_float(ce.y);
                f0 += ((r0(ce.x) >> b) & 1u) ? -Jv : Jv;
              }
            } else for (uint32_t e = rp[s]; e < e1; e += 4) {
              // up to 4 entries, their cluster words and spins loaded before
              // use (independent loads in flight), then summed in row order
              uint2 ce[4];
              uint32_t xc[4], wv[4];
#pragma unroll
              for (uint32_t k = 0; k < 4; ++k)
                if (e + k < e1) ce[k] = ent[e + k];
#pragma unroll
              for (uint32_t k = 0; k < 4; ++k)
                if (e + k < e1) {
                  xc[k] = XC[ce[k].x];
                  wv[k] = r0(ce[k].x);
                }
#pragma unroll
              for (uint32_t k = 0; k < 4; ++k) {
                if (e + k >= e1 || ce[k].x == s || ((xc[k] >> b) & 1u)) continue;
                const float Jv = __uint_as_float(ce[k].y);
                f0 += ((wv[k] >> b) & 1u) ? -Jv : Jv;
              }
            }
            const float s0 = ((r0(s) >> b) & 1u) ? -1.0f : 1.0f;
            a0 += to_fx(-2.0f * s0 * f0);
          }
          a1 = -a0;
        }
      }
      for (int off = 16; off > 0; off >>= 1) {
        a0 += __shfl_xor_sync(0xffffffffu, a0, off);
        a1 += __shfl_xor_sync(0xffffffffu, a1, off);
      }
      if (lane == 0) {
        X.part[warp * 2] = a0;
        X.part[warp * 2 + 1] = a1;
      }
      __syncthreads();
      if (tw == 0 && lane < 2 && b < 32 && X.cnt[b]) {
        long long t = 0;
        for (uint32_t k = 0; k < team; ++k) t += X.part[(warp + k) * 2 + lane];
        X.dE[lane * 32 + b] = (unsigned long long)t;
      }
      __syncthreads();
    }
  }
  if (pc && prop) pc->lap(PHASE_ICM_MARK);  // (propagation: the energy change ends here, the flip follows)
  for (uint32_t x = tid; x < nlist; x += T) {
    const uint32_t s = vlist ? vlist[x] : vlist16 ? (uint32_t)vlist16[x] : x;
    const uint32_t c = XC[s];
    if (c) {
      atomicXor(&W[s * nw + o0], c);
      atomicXor(&W[s * nw + o1], c);
    }
  }
}

// ICM phase of the fused kernel: all chain pairs, all slots >= lo, in groups
// of at most J.icm_group slots (the label arrays that fit in shared memory).
__device__ void icm_phase(const PtJob& J, const FastInst& F, Smem& S, uint32_t i, PhaseClock& pc) {
  const uint32_t tid = threadIdx.x;
  for (uint32_t p = 0; 2 * p + 1 < J.C; ++p) {
    const uint32_t c0 = 2 * p, c1 = 2 * p + 1;
    for (uint32_t w = 0; w < J.wpc; ++w) {
      const uint32_t tb = 32 * w;
      // slots lo <= tb + b < nt of this word
      const uint32_t lo_b = J.lo > tb ? min(J.lo - tb, 32u) : 0u;
      const uint32_t hi_b = J.nt > tb ? min(J.nt - tb, 32u) : 0u;
      const uint32_t below_hi = hi_b >= 32 ? 0xffffffffu : (1u << hi_b) - 1u;
      const uint32_t below_lo = lo_b >= 32 ? 0xffffffffu : (1u << lo_b) - 1u;
      uint32_t lomask = below_hi & ~below_lo;
      while (lomask) {
        // next group: the lowest `icm_group` set bits
        uint32_t gmask = lomask;
        if ((uint32_t)__popc(lomask) > J.icm_group) {
          gmask = 0;
          uint32_t m = lomask;
          for (uint32_t g = 0; g < J.icm_group && m; ++g) {
            gmask |= m & (~m + 1u);
            m &= m - 1;
          }
        }
        lomask &= ~gmask;
        icm_group<false>(J, F, S.W, S.X, i, p, w, gmask, nullptr, nullptr, &pc);
        __syncthreads();
        pc.lap(PHASE_ICM_APPLY);
        if (tid < 32 && ((gmask >> tid) & 1u) && S.X.cnt[tid]) {
          // the reference invalidates both caches; the next energy() is energy_ref
          const uint32_t x0 = c0 * J.ntp + tb + tid, x1 = c1 * J.ntp + tb + tid;
          S.Er[x0] += (double)(long long)S.X.dE[tid] * TAMC_FX_INV;
          S.Er[x1] += (double)(long long)S.X.dE[32 + tid] * TAMC_FX_INV;
          S.Ec[x0] = S.Er[x0];
          S.Ec[x1] = S.Er[x1];
        }
        __syncthreads();
        pc.lap(PHASE_ICM_APPLY);
      }
    }
  }
}

// Exchange decisions of round i (threaded or serial semantics), acceptance
// counts, the slot permutation of energies and tags, round trips; S.Dm[c]
// receives the swapped pairs of chain c.
__device__ void exchange_decide(const PtJob& J, Smem& S, uint32_t i) {
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  const uint32_t nt = J.nt;
  XchgSm XS{J.tags, J.acc, J.dhist, J.rtrips, nullptr, nullptr};
  if (S.xb) xchg_layout(&XS, S.xb, J.C, J.ntp);
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
          const float dlt = (S.xb ? XS.dbeta[j] : J.betas[j + 1] - J.betas[j]) * des;
          d[h] = dlt >= 0.0f ||
                 u24(philox4x32_10(make_uint4(j, i, c, PTAG_EXCH), J.key).x) < __expf(dlt);
        }
      }
      D = (uint64_t)__ballot_sync(0xffffffffu, d[0]) | ((uint64_t)__ballot_sync(0xffffffffu, d[1]) << 32);
    } else {
      // Serial semantics: pair j sees ΔE_j plus the carried ΔE_{j-1} when pair
      // j - 1 swapped (tamc-core/src/pt.rs:138-141).  The draws, Δβ, ΔE_j and
      // the decisions without a carry do not depend on earlier pairs, so lane
      // j % 32 computes them for pair j in parallel; the walk over the pairs
      // then redoes only the decisions whose lower pair swapped, with the same
      // float operations as a plain sequential loop (same decisions).
      float des0[2], db[2], u[2];
      bool d0[2];
      for (int h = 0; h < 2; ++h) {
        const uint32_t j = lane + 32u * h;
        des0[h] = 0.0f;
        db[h] = 0.0f;
        u[h] = 1.0f;
        d0[h] = false;
        if (j + 1 < nt) {
          des0[h] = (float)Ec[j + 1] - (float)Ec[j];
          db[h] = S.xb ? XS.dbeta[j] : J.betas[j + 1] - J.betas[j];
          u[h] = u24(philox4x32_10(make_uint4(j, i, c, PTAG_EXCH), J.key).x);
          const float dlt = db[h] * des0[h];
          d0[h] = dlt >= 0.0f || u[h] < __expf(dlt);
        }
      }
      const uint64_t D0 =
          (uint64_t)__ballot_sync(0xffffffffu, d0[0]) | ((uint64_t)__ballot_sync(0xffffffffu, d0[1]) << 32);
      float carry = 0.0f;
      bool prev = false;
      for (uint32_t j = 0; j + 1 < nt; ++j) {  // warp-uniform: every lane walks the same values
        const bool hi = j >= 32u;
        const float e = __shfl_sync(0xffffffffu, hi ? des0[1] : des0[0], j & 31u);
        const float b = __shfl_sync(0xffffffffu, hi ? db[1] : db[0], j & 31u);
        const float uj = __shfl_sync(0xffffffffu, hi ? u[1] : u[0], j & 31u);
        float des = e;
        bool dj;
        if (prev) {
          des = e + carry;
          const float dlt = b * des;
          dj = dlt >= 0.0f || uj < __expf(dlt);
        } else {
          dj = (D0 >> j) & 1ull;
        }
        if (dj) D |= 1ull << j;
        prev = dj;
        carry = des;
      }
    }
    // acceptance counts, slot permutation of energies and tags, round trips
    uint32_t* acc = XS.acc + (size_t)c * nt;
    uint8_t* tg = XS.tags + (size_t)c * nt;
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
      else if (lo == 4) { XS.rtrips[c] += 1; lo = 1; }
      else if (lo == 2) lo = 3;
      tg[0] = lo;
      uint8_t hi = tg[nt - 1];
      if (hi == 0) hi = 2;
      else if (hi == 3) { XS.rtrips[c] += 1; hi = 2; }
      else if (hi == 1) hi = 4;
      tg[nt - 1] = hi;
    }
    __syncwarp();
    for (uint32_t k = lane; k < nt; k += 32) {
      const uint8_t v = tg[k];
      if (v == 1 || v == 3) XS.dhist[((size_t)c * nt + k) * 2] += 1;
      else if (v == 2 || v == 4) XS.dhist[((size_t)c * nt + k) * 2 + 1] += 1;
    }
    if (lane == 0) S.Dm[c] = D;
  }
  __syncthreads();
}

__device__ void permute_words(const PtJob& J, Smem& S);
__device__ __forceinline__ void exchange_phase(const PtJob& J, Smem& S, uint32_t i) {
  exchange_decide(J, S, i);
  permute_words(J, S);
}

// Moves the spins after the exchange decisions: one bit permutation per chain
// word (Dm[c] marks the swapped slot pairs of chain c).
__device__ void permute_words(const PtJob& J, Smem& S) {
  const uint32_t tid = threadIdx.x;
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

// The sites of colour class [c0, c1) for this thread's quad; DEG > 0 when
// every row has DEG entries (unrolled local field, no row pointers).
template <bool SELF, uint32_t DEG>
__device__ __forceinline__ void sweep_class(const PtJob& J, const FastInst& F, Smem& S, uint32_t i, uint32_t c0,
                                            uint32_t c1, uint32_t stride, uint32_t shift, uint32_t wo, uint32_t qid,
                                            float4 beta, Fx4& acc, Fx4& qacc) {
  for (uint32_t s = c0; s < c1; s += stride) {
    const uint4 rnd = philox4x32_10(make_uint4(s, i, qid, PTAG_SWEEP), J.key);
    const uint32_t m = quad_update<true, DEG>(s, shift, F, S.W, J.nw, wo, beta, rnd, acc);
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
      const uint32_t c0 = J.F.color_off[c] + tid / J.qps, c1 = J.F.color_off[c + 1];
      if (F.udeg == 4) sweep_class<SELF, 4>(J, F, S, i, c0, c1, stride, shift, wo, qid, beta, acc, qacc);
      else sweep_class<SELF, 0>(J, F, S, i, c0, c1, stride, shift, wo, qid, beta, acc, qacc);
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

// Multi-spin-coded sweep of a +-J job (J.msc): warp w updates replica word
// wo = w % nw of 32 consecutive sites of the colour class per step (lane =
// site), the whole word at once (msc_flip); a lane owns its word, so no
// atomics.  Per-replica energy changes are reduced over the warp's sites by
// bit transposes and summed over warps in fixed point.  The threshold planes
// of every word are in S.msc (msc_fill_planes).
template <uint32_t DEG>
__device__ __noinline__ void sweep_phase_msc(const PtJob& J, const FastInst& F, Smem& S, uint32_t i) {
  const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5, nwarp = blockDim.x >> 5;
  const uint32_t nw = J.nw;
  // words in pairs (wo, wo + 1) per lane when nw is even: two independent
  // random streams in flight per lane; nw == 1 takes the single-word path
  const uint32_t per = nw == 1 ? 1u : 2u, ng = nw / per;
  const uint32_t g = warp % ng, step = nwarp / ng;
  const uint32_t wo = g * per;
  const uint32_t* pl = S.msc + wo * MSC_WORDS;
  // sub-phase cycles per warp (lane 0) when profiling
  unsigned long long* const prof = J.prof;
  long long tl = (prof && lane == 0) ? clock64() : 0;
  auto stamp = [&](int ph) {
    if (prof && lane == 0) {
      const long long t = clock64();
      atomicAdd(&prof[ph], (unsigned long long)(t - tl));
      tl = t;
    }
  };
  long long e0 = 0, e1 = 0;
  for (uint32_t c = 0; c < F.ncolors; ++c) {
    const uint32_t c0 = J.F.color_off[c], c1 = J.F.color_off[c + 1];
    for (uint32_t base = c0 + (warp / ng) * 32u; base < c1; base += step * 32u) {
      const uint32_t s = base + lane;
      uint32_t f0 = 0, f1 = 0;
      MscLevels L0{}, L1{};
      uint32_t S0 = 0, S1 = 0;
      if (s < c1) {
        uint32_t Wj0[DEG], Wj1[DEG], neg = 0;
        S0 = S.W[s * nw + wo];
        S1 = per == 2 ? S.W[s * nw + wo + 1] : 0u;
#pragma unroll
        for (uint32_t m = 0; m < DEG; ++m) {
          const uint2 ce = F.ent[s * DEG + m];
          Wj0[m] = S.W[ce.x * nw + wo];
          Wj1[m] = per == 2 ? S.W[ce.x * nw + wo + 1] : 0u;
          neg |= (ce.y >> 31) << m;
        }
        L0 = msc_levels<DEG>(S0, Wj0, neg);
        if (per == 2) L1 = msc_levels<DEG>(S1, Wj1, neg);
      }
      if (prof) __syncwarp();
      stamp(PHASE_SW_LEVELS);
      if (s < c1) {
        if (per == 2) msc_flip2<DEG>(L0, L1, pl, pl + MSC_WORDS, s, i, wo, J.key, f0, f1);
        else f0 = msc_flip<DEG>(L0, pl, pl + 96, pl + 99, s, i, wo, J.key);
      }
      if (prof) __syncwarp();
      stamp(PHASE_SW_FLIP);
      if (s < c1) {
        if (per == 2) S.W[s * nw + wo + 1] = S1 ^ f1;
        S.W[s * nw + wo] = S0 ^ f0;
      }
      e0 += msc_energy<DEG>(f0, L0, lane);
      if (per == 2) e1 += msc_energy<DEG>(f1, L1, lane);
      stamp(PHASE_SW_ENERGY);
    }
    __syncthreads();
    stamp(PHASE_SW_WAIT);
  }
  long long* red = reinterpret_cast<long long*>(S.red);  // nwarp * 64 entries (the 2 T * 16 bytes of red, redq)
  red[(warp * 2) * 32 + lane] = e0;
  red[(warp * 2 + 1) * 32 + lane] = e1;
  __syncthreads();
  for (uint32_t x = tid; x < nw * 32; x += blockDim.x) {
    const uint32_t w2 = x / 32, r = x % 32;
    const uint32_t gg = w2 / per, k = w2 % per;  // word w2 is member k of pair gg
    long long sum = 0;
    for (uint32_t ww = gg; ww < nwarp; ww += ng) sum += red[(ww * 2 + k) * 32 + r];
    const uint32_t c = w2 / J.wpc, t = (w2 % J.wpc) * 32 + r;
    if (t < J.ntp) {
      const uint32_t xx = c * J.ntp + t;
      S.Ec[xx] += (double)sum * TAMC_FX_INV;
      S.Er[xx] += (double)sum * TAMC_FX_INV;
    }
  }
  __syncthreads();
}

// Threshold planes of every replica word of the job (warp w < nw fills word w).
template <uint32_t DEG>
__device__ __noinline__ void msc_fill_planes(const PtJob& J, uint32_t* msc) {
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  for (uint32_t wo = warp; wo < J.nw; wo += blockDim.x >> 5) {
    const uint32_t t = (wo % J.wpc) * 32 + lane;
    const float beta = t < J.ntp ? J.betas[t] : 0.0f;
    uint32_t* pl = msc + wo * MSC_WORDS;
    msc_planes<DEG>(beta, lane, pl, pl + 96, pl + 99);
  }
}

__device__ __forceinline__ bool sched(int64_t period, uint32_t i, uint32_t meas_init, uint32_t num_sweeps) {
  return period >= 0 && i >= meas_init && ((i - meas_init) % (uint32_t)period == 0 || i == num_sweeps - 1);
}

// A new running minimum found by gs_track: its log entry, chain and slot.
struct GsSnap {
  int fresh;
  uint32_t k, c, t;
};

// Ground-state tracking (apply_measurements, src/pt.rs:542-583): the
// reference takes the first minimum over slots, then the first over chains
// (lexicographic (E, chain, slot)), and records it when strictly below the
// running minimum.  Warp 0 reduces; every thread gets the result.
__device__ GsSnap gs_track(const PtJob& J, Smem& S, uint32_t i) {
  __shared__ GsSnap s_g;
  const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
  const uint32_t nt = J.nt, C = J.C;
  if (warp == 0) {
    float be = INFINITY;
    uint32_t bx = 0xffffffffu;
    for (uint32_t x = lane; x < C * nt; x += 32) {
      const float e = (float)S.Ec[(x / nt) * J.ntp + (x % nt)];
      if (e < be || (e == be && x < bx)) { be = e; bx = x; }
    }
    for (int off = 16; off > 0; off >>= 1) {
      const float oe = __shfl_xor_sync(0xffffffffu, be, off);
      const uint32_t ox = __shfl_xor_sync(0xffffffffu, bx, off);
      if (oe < be || (oe == be && ox < bx)) { be = oe; bx = ox; }
    }
    if (lane == 0) {
      GsSnap g{0, 0, 0, 0};
      XchgSm XS{};
      if (S.xb) xchg_layout(&XS, S.xb, J.C, J.ntp);
      int* have = S.xb ? &XS.gs->have : J.log.have;
      float* minE = S.xb ? &XS.gs->minE : J.log.minE;
      uint32_t* count = S.xb ? &XS.gs->count : J.log.count;
      if (!*have || be < *minE) {
        *have = 1;
        *minE = be;
        const uint32_t k = *count;
        if (k < J.log.cap) {
          J.log.steps[k] = i;
          J.log.E[k] = be;
          g = GsSnap{1, k, bx / nt, bx % nt};
        }
        *count = k + 1;
      }
      s_g = g;
    }
  }
  __syncthreads();
  return s_g;
}

// The rest of a round's measurements, after gs_track: the new minimum's
// state, and on the sampling schedule e / q / suscept (weights `sus`,
// [nchi][n] in colour order) and packed state samples.  `xs` (n words of
// shared memory, or null) holds one chain pair's disagreement word per site
// while its overlaps are summed.
// Shared-memory access pattern: the site words are W[s * nw + o], so lanes on
// consecutive sites read with a stride of nw words (nw-way bank conflicts), and
// the packed outputs gather through the site permutation.  Bits are therefore
// packed per 32 consecutive original sites (one gather per replica word, then
// a ballot or a bit transpose), and the overlap sums first copy each pair's
// disagreement word to the dense array xs.  Sums keep the order of a warp over sites s = lane +
// 32 k followed by a shuffle tree, so results do not depend on the CTA size.
__device__ void measure_rest(const PtJob& J, const FastInst& F, Smem& S, const double* sus, const uint32_t* iperm,
                             uint32_t i, uint32_t& m_cur, uint32_t& s_cur, GsSnap g, uint32_t* xs) {
  const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5, nwarp = blockDim.x >> 5;
  const uint32_t n = J.n, nt = J.nt, C = J.C;
  if (g.fresh) {
    // 64-bit words of the new minimum's spins in original site order, as
    // 32-bit halves: bit x of half h is site 32 h + x
    const uint32_t nw64 = (n + 63) / 64;
    const uint32_t o = g.c * J.wpc + (g.t >> 5), b = g.t & 31u;
    uint32_t* dst = reinterpret_cast<uint32_t*>(J.log.words + (size_t)g.k * nw64);
    for (uint32_t h = warp; h < 2 * nw64; h += nwarp) {
      const uint32_t s = h * 32 + lane;
      const uint32_t bit = s < n ? (S.W[iperm[s] * J.nw + o] >> b) & 1u : 0u;
      const uint32_t bits = __ballot_sync(0xffffffffu, bit);
      if (lane == 0) dst[h] = bits;
    }
  }
  const uint32_t P = C / 2;
  if (sched(J.sample, i, J.meas_init, J.num_sweeps)) {
    const uint32_t m = m_cur++;
    for (uint32_t x = tid; x < C * nt; x += blockDim.x) {
      const uint32_t c = x / nt, t = x % nt;
      J.out.e[(size_t)t * J.out.M * C + (size_t)m * C + c] = (float)S.Ec[c * J.ntp + t];
    }
    const uint32_t nchi = J.out.nchi;
    for (uint32_t p = 0; p < P; ++p) {
      for (uint32_t wd = 0; wd < J.wpc; ++wd) {
        const uint32_t o0 = 2 * p * J.wpc + wd, o1 = (2 * p + 1) * J.wpc + wd;
        const uint32_t tn = min(32u, nt - 32 * wd);  // temperatures in this word
        if (xs) {
          __syncthreads();  // xs free (previous word's sums done)
          for (uint32_t s = tid; s < n; s += blockDim.x) xs[s] = S.W[s * J.nw + o0] ^ S.W[s * J.nw + o1];
          __syncthreads();
        }
        auto xword = [&](uint32_t s) -> uint32_t {
          return xs ? xs[s] : (S.W[s * J.nw + o0] ^ S.W[s * J.nw + o1]);
        };
        // one warp per temperature of the word: q, then the weights in pairs
        for (uint32_t tb = warp; tb < tn; tb += nwarp) {
          const uint32_t t = 32 * wd + tb;
          uint32_t neg = 0;
          for (uint32_t s = lane; s < n; s += 32) neg += (xword(s) >> tb) & 1u;
          for (int off = 16; off > 0; off >>= 1) neg += __shfl_xor_sync(0xffffffffu, neg, off);
          if (lane == 0) J.out.q[(size_t)t * J.out.M * P + (size_t)m * P + p] = (int32_t)n - 2 * (int32_t)neg;
          for (uint32_t k0 = 0; k0 < nchi; k0 += 2) {
            double chi[2] = {0.0, 0.0};
            for (uint32_t s = lane; s < n; s += 32) {
              const bool flip = (xword(s) >> tb) & 1u;
#pragma unroll
              for (uint32_t j = 0; j < 2; ++j)
                if (k0 + j < nchi) {
                  const double wv = sus[(size_t)(k0 + j) * n + s];
                  chi[j] += flip ? -wv : wv;
                }
            }
#pragma unroll
            for (uint32_t j = 0; j < 2; ++j) {
              if (k0 + j >= nchi) break;
              double v = chi[j];
              for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
              if (lane == 0)
                J.out.sus[((size_t)t * nchi + k0 + j) * J.out.M * P + (size_t)m * P + p] = (float)v;
            }
          }
        }
      }
    }
  }
  if (sched(J.sample_states, i, J.meas_init, J.num_sweeps)) {
    // bytes of 8 original sites (bit k = site 8 byte + k).  A warp takes 8
    // blocks of 32 consecutive original sites for one chain and replica word,
    // gathers each site's word once and transposes each 32x32 bit block, so
    // that lane t holds 32 bytes of temperature t's row: two 16-byte stores
    // per row where the rows are 16-byte aligned, else byte stores.
    const uint32_t smp = s_cur++;
    const uint32_t nb = (n + 7) / 8;
    const uint32_t Z = J.level == 0 ? nt : (J.level == 1 ? nt / 2 : 1);
    const uint32_t nblk = ((n + 31) / 32 + 7) / 8;
    const bool wide = nb % 16 == 0;  // row starts 16-byte aligned (the buffer itself is)
    for (uint32_t it = warp; it < C * J.wpc * nblk; it += nwarp) {
      const uint32_t hb = it % nblk, cw = it / nblk, c = cw / J.wpc, wd = cw % J.wpc;
      uint32_t xv[8];
#pragma unroll
      for (uint32_t j = 0; j < 8; ++j) {
        const uint32_t s = (8 * hb + j) * 32 + lane;
        xv[j] = transpose32(s < n ? S.W[iperm[s] * J.nw + c * J.wpc + wd] : 0u, lane);
      }
      const uint32_t t = 32 * wd + lane;
      uint32_t z = 0xffffffffu;  // sample slot of temperature t, if sampled
      if (t < nt) {
        if (J.level == 0) z = t;
        else if (J.level == 1) z = nt - 1 - t < Z ? nt - 1 - t : 0xffffffffu;
        else z = t == nt - 1 ? 0u : 0xffffffffu;
      }
      if (z != 0xffffffffu) {
        uint8_t* dst = J.out.samp + (((size_t)z * J.out.S + smp) * C + c) * nb + 32 * hb;
        if (wide && 32 * hb + 32 <= nb) {
          reinterpret_cast<uint4*>(dst)[0] = make_uint4(xv[0], xv[1], xv[2], xv[3]);
          reinterpret_cast<uint4*>(dst)[1] = make_uint4(xv[4], xv[5], xv[6], xv[7]);
        } else {
#pragma unroll
          for (uint32_t j = 0; j < 8; ++j)
            for (uint32_t k = 0; k < 4; ++k)
              if (32 * hb + 4 * j + k < nb) dst[4 * j + k] = (uint8_t)(xv[j] >> (8 * k));
        }
      }
    }
  }
  __syncthreads();
}

__device__ void measure_phase(const PtJob& J, const FastInst& F, Smem& S, uint32_t i, uint32_t& m_cur,
                              uint32_t& s_cur) {
  const GsSnap g = gs_track(J, S, i);
  measure_rest(J, F, S, F.sus, F.iperm, i, m_cur, s_cur, g, S.X.D);  // the ICM arrays are free here
}

// Copy of the job descriptor in shared memory: the phase functions read its
// fields inside their loops, and shared-memory loads stay short where global
// reloads of a descriptor evicted from L1 would go to L2.
__device__ __forceinline__ void load_job(PtJob& dst, const PtJob* src) {
  static_assert(sizeof(PtJob) % 8 == 0, "job descriptor copied as 8-byte words");
  const uint2* a = reinterpret_cast<const uint2*>(src);
  uint2* b = reinterpret_cast<uint2*>(&dst);
  for (uint32_t x = threadIdx.x; x < sizeof(PtJob) / 8; x += blockDim.x) b[x] = a[x];
  __syncthreads();
}

// The fused job's bookkeeping into shared memory (start of a range of rounds)
// and back (its end); the end also reports the log count.
// Threads from t0 on copy (the ones below t0 may be loading something else
// meanwhile); every thread meets the closing barrier.
__device__ __noinline__ void xchg_load(const PtJob& J, char* xb, bool gs = true, uint32_t t0 = 0) {
  XchgSm X;
  xchg_layout(&X, xb, J.C, J.ntp);
  const uint32_t CT = J.C * J.nt;
  if (threadIdx.x >= t0) {
    const uint32_t tid = threadIdx.x - t0, T = blockDim.x - t0;
    for (uint32_t x = tid; x < CT; x += T) {
      X.tags[x] = J.tags[x];
      X.acc[x] = J.acc[x];
      X.dhist[2 * x] = J.dhist[2 * x];
      X.dhist[2 * x + 1] = J.dhist[2 * x + 1];
    }
    for (uint32_t c = tid; c < J.C; c += T) X.rtrips[c] = J.rtrips[c];
    for (uint32_t j = tid; j + 1 < J.nt; j += T) X.dbeta[j] = J.betas[j + 1] - J.betas[j];
    if (gs && tid == 0) {
      X.gs->have = *J.log.have;
      X.gs->minE = *J.log.minE;
      X.gs->count = *J.log.count;
    }
  }
  __syncthreads();
}
__device__ __noinline__ void xchg_store(const PtJob& J, char* xb, bool gs = true) {
  XchgSm X;
  xchg_layout(&X, xb, J.C, J.ntp);
  const uint32_t CT = J.C * J.nt;
  for (uint32_t x = threadIdx.x; x < CT; x += blockDim.x) {
    J.tags[x] = X.tags[x];
    J.acc[x] = X.acc[x];
    J.dhist[2 * x] = X.dhist[2 * x];
    J.dhist[2 * x + 1] = X.dhist[2 * x + 1];
  }
  for (uint32_t c = threadIdx.x; c < J.C; c += blockDim.x) J.rtrips[c] = X.rtrips[c];
  if (gs && threadIdx.x == 0) {
    *J.log.have = X.gs->have;
    *J.log.minE = X.gs->minE;
    *J.log.count = X.gs->count;
    if (J.count_out) *J.count_out = X.gs->count;
  }
  __syncthreads();
}

template <bool SELF>
__device__ void run_job(const PtJob& J, char* smem_base) {
  Smem S;
  carve_all(&S, smem_base, J.n, J.nw, J.C, J.ntp, J.qps, blockDim.x, J.F.nnz, J.csr_smem != 0, J.icm_group,
            J.icm_uf != 0);
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
    const float L2E = TAMC_2LOG2E;  // 2 beta log2(e) for ex2
    S.beta4[k] = make_float4(J.betas[4 * q] * L2E, J.betas[4 * q + 1] * L2E, J.betas[4 * q + 2] * L2E,
                             J.betas[4 * q + 3] * L2E);
  }
  const uint32_t Teff = (T / J.qps) * J.qps;
  if (J.msc) {
    if (F.udeg == 4) msc_fill_planes<4>(J, S.msc);
    else msc_fill_planes<6>(J, S.msc);
  }
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
  // exchange bookkeeping and the ground-state minimum stay in shared memory
  // for the range of rounds (no global round trips inside a round)
  xchg_load(J, S.xb);
  uint32_t m_cur = J.m_base, s_cur = J.s_base;
  PhaseClock pc;
  pc.start(J.prof);
  for (uint32_t i = J.sweep_begin; i < J.sweep_end; ++i) {
    if (J.icm) icm_phase(J, F, S, i, pc);
    exchange_phase(J, S, i);
    pc.lap(PHASE_EXCH);
    if (J.msc) {
      if (F.udeg == 4) sweep_phase_msc<4>(J, F, S, i);
      else sweep_phase_msc<6>(J, F, S, i);
    } else {
      sweep_phase<SELF>(J, F, S, i, Teff);
    }
    pc.lap(PHASE_SWEEP);
    if (i >= J.meas_init) measure_phase(J, F, S, i, m_cur, s_cur);
    pc.lap(PHASE_MEASURE);
  }
  for (uint32_t x = tid; x < n * J.nw; x += T) J.W[x] = S.W[x];
  for (uint32_t x = tid; x < J.C * J.ntp; x += T) {
    J.Ec[x] = S.Ec[x];
    J.Er[x] = S.Er[x];
  }
  xchg_store(J, S.xb);
}

__global__ void __launch_bounds__(512, 1) k_pt_fused(const PtJob* __restrict__ jobs, uint32_t njobs, uint32_t* ctr) {
  extern __shared__ uint4 smem_u4[];
  __shared__ uint32_t s_job;
  __shared__ PtJob s_J;
  for (;;) {
    if (threadIdx.x == 0) s_job = atomicAdd(ctr, 1u);
    __syncthreads();
    const uint32_t jid = s_job;
    __syncthreads();
    if (jid >= njobs) break;
    load_job(s_J, jobs + jid);
    if (s_J.self_loops) run_job<true>(s_J, reinterpret_cast<char*>(smem_u4));
    else run_job<false>(s_J, reinterpret_cast<char*>(smem_u4));
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
  (void)n;
  return al16((size_t)C * ntp * 8) * 2 + al16((size_t)C * 8) + 64;
}
// The exchange body's shared memory: the head's energies and masks, then the
// bookkeeping staged from global memory (XchgSm).
__host__ __device__ inline size_t plain_exch_smem(uint32_t n, uint32_t C, uint32_t ntp) {
  return plain_head_smem(n, C, ntp) + xchg_layout(nullptr, nullptr, C, ntp);
}

// Close the previous round (add its fixed-point sweep sums, measurements), or
// (mode 2) set the initial energies from the energy kernel's sums.
__global__ void __launch_bounds__(1024, 1) k_plain_head(const PtJob* __restrict__ jp, PlainCtl* ctl,
                                                       long long* acc, int mode, int stage) {
  pdl_enter();
  extern __shared__ uint4 smem_u4[];
  __shared__ PtJob s_J;
  load_job(s_J, jp);
  const PtJob& J = s_J;
  const uint32_t tid = threadIdx.x;
  // rounds without measurements were closed by the last sweep launch
  if (mode != 2 && !ctl->pending) return;
  char* base = reinterpret_cast<char*>(smem_u4);
  Smem S{};
  S.Ec = (double*)base;
  S.Er = (double*)(base + al16((size_t)J.C * J.ntp * 8));
  S.W = J.W;
  const FastInst F = J.F;
  const uint32_t CN = J.C * J.ntp;
  long long* accq = acc + CN;
  const bool pending = mode != 2 && ctl->pending;
  for (uint32_t x = tid; x < CN; x += blockDim.x) {
    double ec = J.Ec[x], er = J.Er[x];
    if (mode == 2) {
      ec = (double)J.F.offset + (double)acc[x] * TAMC_FX_INV;
      er = ec;
      acc[x] = 0;
    } else if (pending) {  // IsingSampler::sweep: energy += sum of accepted dE
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
  PhaseClock pc;
  pc.start(J.prof);
  if (pending) {
    const uint32_t ip = ctl->i - 1;
    if (ip >= J.meas_init) {
      const GsSnap g = gs_track(J, S, ip);
      const bool meas = sched(J.sample, ip, J.meas_init, J.num_sweeps);
      const bool snap = sched(J.sample_states, ip, J.meas_init, J.num_sweeps);
      const double* sus = F.sus;
      const uint32_t* iperm = F.iperm;
      uint32_t* xs = nullptr;
      if (stage && (g.fresh || meas || snap)) {
        // the measurements gather bits of every site: read the replica words,
        // the weights and the site permutation once into shared memory
        // instead of gathering from L2
        char* st = base + plain_head_smem(J.n, J.C, J.ntp);
        uint32_t* Ws = reinterpret_cast<uint32_t*>(st);
        const uint32_t nwords = J.n * J.nw;
        for (uint32_t x = tid; x < nwords / 4; x += blockDim.x)
          reinterpret_cast<uint4*>(Ws)[x] = reinterpret_cast<const uint4*>(J.W)[x];
        for (uint32_t x = nwords / 4 * 4 + tid; x < nwords; x += blockDim.x) Ws[x] = J.W[x];
        st += al16((size_t)nwords * 4);
        if (g.fresh || snap) {
          uint32_t* ip_s = reinterpret_cast<uint32_t*>(st);
          for (uint32_t x = tid; x < J.n; x += blockDim.x) ip_s[x] = F.iperm[x];
          iperm = ip_s;
        }
        st += al16((size_t)J.n * 4);
        if (meas && F.nchi) {
          double* ss = reinterpret_cast<double*>(st);
          for (uint32_t x = tid; x < F.nchi * J.n; x += blockDim.x) ss[x] = F.sus[x];
          sus = ss;
        }
        st += al16((size_t)F.nchi * J.n * 8);
        xs = reinterpret_cast<uint32_t*>(st);  // one pair's disagreement words for the overlaps
        __syncthreads();
        S.W = Ws;
      }
      measure_rest(J, F, S, sus, iperm, ip, m_cur, s_cur, g, xs);
    }
  }
  for (uint32_t x = tid; x < CN; x += blockDim.x) {
    J.Ec[x] = S.Ec[x];
    J.Er[x] = S.Er[x];
  }
  __syncthreads();
  pc.lap(PHASE_MEASURE);
  if (tid == 0) {
    ctl->m_cur = m_cur;
    ctl->s_cur = s_cur;
    ctl->pending = 0;
    if (J.count_out) *J.count_out = *J.log.count;
  }
}

__device__ void plain_exchange_body(const PtJob& J, PlainCtl* ctl, const long long* icm_dE, uint32_t* icm_valid,
                                    char* base, unsigned long long* dm, bool staged = false);

// Houdayer moves of round ctl->i: one CTA per (chain pair, slot >= lo).
__global__ void __launch_bounds__(1024, 1) k_plain_icm(const PtJob* __restrict__ jp, PlainCtl* ctl, long long* icm_dE,
                                                       uint32_t* icm_valid, int stage, unsigned long long* dm) {
  pdl_enter();
  extern __shared__ uint4 smem_u4[];
  __shared__ PtJob s_J;
  load_job(s_J, jp);
  const PtJob& J = s_J;
  const uint32_t nact = J.nt - J.lo;
  const uint32_t p = blockIdx.x / nact, t = J.lo + blockIdx.x % nact;
  char* base = reinterpret_cast<char*>(smem_u4);
  IcmScratch X;
  const size_t o = carve_icm(&X, base, 0, J.n, 1, J.icm_uf ? ICM_UF : ICM_BFS_ONE);
  FastInst F = J.F;
  const uint16_t* cols = nullptr;
  // stage bit 1: replica 0's words [n]; bit 0: row pointers and columns
  uint32_t* wstage = (stage & 2) ? reinterpret_cast<uint32_t*>(base + o) : nullptr;
  const size_t o2 = o + ((stage & 2) ? al16((size_t)J.n * 4) : 0);
  if (stage & 1) {
    // row pointers and 16-bit column indices in shared memory for the cluster search
    uint32_t* rp = reinterpret_cast<uint32_t*>(base + o2);
    uint16_t* cl = reinterpret_cast<uint16_t*>(base + o2 + al16((size_t)(J.n + 1) * 4));
    // 16-byte copies: rp (n + 1 words, tail by words) and the padded 16-bit columns
    const uint32_t nrp4 = (J.n + 1) / 4;
    for (uint32_t x = threadIdx.x; x < nrp4; x += blockDim.x)
      reinterpret_cast<uint4*>(rp)[x] = reinterpret_cast<const uint4*>(J.F.rp)[x];
    for (uint32_t x = 4 * nrp4 + threadIdx.x; x <= J.n; x += blockDim.x) rp[x] = J.F.rp[x];
    const uint32_t ncl8 = (J.F.nnz + 7) / 8;
    for (uint32_t x = threadIdx.x; x < ncl8; x += blockDim.x)
      reinterpret_cast<uint4*>(cl)[x] = reinterpret_cast<const uint4*>(J.F.col16)[x];
    __syncthreads();
    F.rp = rp;
    cols = cl;
  }
  const uint32_t b = t & 31u;
  PhaseClock pc;  // with profiling on, cycles are summed over the CTAs
  pc.start(J.prof);
  icm_group<true>(J, F, J.W, X, ctl->i, p, t >> 5, 1u << b, cols, wstage, &pc);
  __syncthreads();
  if (threadIdx.x == 0) {
    const uint32_t x0 = 2 * p * J.ntp + t, x1 = (2 * p + 1) * J.ntp + t;
    const uint32_t v = X.cnt[b] != 0;
    icm_valid[x0] = v;
    icm_valid[x1] = v;
    icm_dE[x0] = (long long)X.dE[b];
    icm_dE[x1] = (long long)X.dE[32 + b];
  }
  pc.lap(PHASE_ICM_APPLY);
  // the last CTA to finish runs the exchange of the round (no waiting: the
  // others have published their results before counting themselves done)
  __shared__ int s_last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    s_last = atomicAdd(&ctl->icm_done, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  if (threadIdx.x == 0) ctl->icm_done = 0;
  plain_exchange_body(J, ctl, icm_dE, icm_valid, base, dm);
}

// Houdayer moves of round ctl->i on a periodic square or cubic lattice of
// side L = 16 or 32 in file order (FastInst::lat_L): one CTA per (chain pair,
// slot >= lo), as k_plain_icm, with the slot's disagreement set and cluster
// held as bitmaps over the original site order (n / 32 words; a lattice row
// fills half or all of a word).  A growth pass is word-parallel: each of the
// first n / 32 threads owns one word and first closes it under the moves
// inside the word (z +-1 within each row; for L = 16 also between the word's
// two rows), then adds the D sites next to cluster sites of the words of the
// neighbouring rows and planes; a warp repeats this while its words grow, and
// passes (a barrier over the growth threads) end when one changes nothing, so
// the result is the exact component of the seed.  Meanwhile the other threads
// stage the couplings, columns, fields and permutation for the energy change.  The seed is the k-th q<0 site
// in colour order with k drawn as in icm_group, and the energy change sums
// each cluster site's boundary terms in its colour-ordered row order with the
// couplings and columns staged in shared memory, so the move, the flips and
// the fixed-point sums are those of k_plain_icm bit for bit.
struct LatScratch {
  float* Jf;         // [DEG][n] couplings: entry m of colour row s at m n + s
  uint16_t* cols;    // [DEG][n] columns, same layout
  uint32_t* Dcol;    // [NW] q<0 bits of the slot, colour order
  uint32_t* R0col;   // [NW] replica 0's spin bits of the slot, colour order
  uint32_t* Do;      // [NW] q<0 bits, original order
  uint32_t* Co;      // [NW] cluster bits, original order
  uint32_t* Ccol;    // [NW] cluster bits, colour order
  float* bias;       // [n] fields, colour order
  uint32_t* perm;    // [n] colour -> file order
  long long* part;   // [32] per-warp energy sums
  uint32_t* misc;    // [4] seed count, seed site, pass flag
};
__host__ __device__ inline size_t carve_lat(LatScratch* X, char* base, uint32_t n, uint32_t nnz) {
  size_t o = 0;
  auto take = [&](size_t bytes) {
    char* p = base ? base + o : nullptr;
    o = al16(o + bytes);
    return p;
  };
  const size_t NW = (n + 31) / 32;
  char* Jf = take((size_t)nnz * 4);
  char* cols = take((size_t)nnz * 2);
  char* Dcol = take(NW * 4);
  char* R0col = take(NW * 4);
  char* Do = take(NW * 4);
  char* Co = take(NW * 4);
  char* Ccol = take(NW * 4);
  char* bias = take((size_t)n * 4);
  char* perm = take((size_t)n * 4);
  char* part = take(32 * 8);
  char* misc = take(4 * 4);
  if (X) {
    X->Jf = (float*)Jf;
    X->cols = (uint16_t*)cols;
    X->Dcol = (uint32_t*)Dcol;
    X->R0col = (uint32_t*)R0col;
    X->Do = (uint32_t*)Do;
    X->Co = (uint32_t*)Co;
    X->Ccol = (uint32_t*)Ccol;
    X->bias = (float*)bias;
    X->perm = (uint32_t*)perm;
    X->part = (long long*)part;
    X->misc = (uint32_t*)misc;
  }
  return o;
}

// Closure of the cluster bits c under the moves inside one bitmap word of the
// q<0 bits d: along each row (periodic in L), and for L = 16 between the
// word's two rows.  A row is filled from its seeds with one addition each
// way: on the row written twice in a row, the carry of d + c runs from every
// seed through the run of d above it (past the row's end into the copy: the
// periodic wrap), and bit reversal gives the other direction.
__device__ __forceinline__ uint32_t lat_fill32(uint32_t c, uint32_t d) {
  const uint64_t dd = (uint64_t)d | ((uint64_t)d << 32);
  uint64_t up = (((dd + c) ^ dd) & dd) | c;
  const uint32_t rd = __brev(d), rc = __brev(c);
  const uint64_t rdd = (uint64_t)rd | ((uint64_t)rd << 32);
  uint64_t dn = (((rdd + rc) ^ rdd) & rdd) | rc;
  return (uint32_t)(up | (up >> 32)) | __brev((uint32_t)(dn | (dn >> 32)));
}
__device__ __forceinline__ uint32_t lat_fill16(uint32_t c, uint32_t d) {  // c, d < 2^16
  const uint32_t dd = d | (d << 16);
  uint32_t up = (((dd + c) ^ dd) & dd) | c;
  const uint32_t rd = __brev(dd), rc = __brev(c) >> 16;
  uint32_t dn = (((rd + rc) ^ rd) & rd) | rc;
  return ((up | (up >> 16)) & 0xffffu) | (__brev((dn | (dn >> 16)) & 0xffffu) >> 16);
}
// (For L = 16 two rounds of row fill and row coupling, a fixed cost per call:
// what remains to couple is added by the next call of the growth loop.)
__device__ __forceinline__ uint32_t lat_fill_rows16(uint32_t c, uint32_t d) {
  return lat_fill16(c & 0xffffu, d & 0xffffu) | (lat_fill16(c >> 16, d >> 16) << 16);
}
template <uint32_t L>
__device__ __forceinline__ uint32_t lat_close(uint32_t c, uint32_t d) {
  if (L == 32) return lat_fill32(c, d);
  c = lat_fill_rows16(c, d);
  c |= d & ((c >> 16) | (c << 16));  // the word's two rows are neighbours
  c = lat_fill_rows16(c, d);
  return c | (d & ((c >> 16) | (c << 16)));
}

// Barrier over the first `count` threads (a multiple of 32) on barrier 1,
// returning whether any of them passed a non-zero `pred`.
__device__ __forceinline__ int bar1_or(int pred, uint32_t count) {
  int r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\tsetp.ne.s32 q, %1, 0;\n\tbar.red.or.pred p, 1, %2, q;\n\tselp.s32 %0, 1, 0, p;\n\t}"
      : "=r"(r)
      : "r"(pred), "r"(count)
      : "memory");
  return r;
}

// Stages the exchange's inputs into `base` in plain_exchange_body's layout:
// the energies as the round started (the Houdayer changes are added at the
// exchange) and the bookkeeping that xchg_load copies, by the threads tid of
// T (part of the CTA; no barrier).
__device__ void plain_exch_stage(const PtJob& J, char* base, uint32_t tid, uint32_t T) {
  const uint32_t CN = J.C * J.ntp, CT = J.C * J.nt;
  double* Ec = (double*)base;
  double* Er = (double*)(base + al16((size_t)CN * 8));
  for (uint32_t x = tid; x < CN; x += T) {
    Ec[x] = J.Ec[x];
    Er[x] = J.Er[x];
  }
  XchgSm X;
  xchg_layout(&X, base + plain_head_smem(J.n, J.C, J.ntp), J.C, J.ntp);
  for (uint32_t x = tid; x < CT; x += T) {
    X.tags[x] = J.tags[x];
    X.acc[x] = J.acc[x];
    X.dhist[2 * x] = J.dhist[2 * x];
    X.dhist[2 * x + 1] = J.dhist[2 * x + 1];
  }
  for (uint32_t c = tid; c < J.C; c += T) X.rtrips[c] = J.rtrips[c];
  for (uint32_t j = tid; j + 1 < J.nt; j += T) X.dbeta[j] = J.betas[j + 1] - J.betas[j];
}

template <uint32_t L, uint32_t DIM>
__global__ void __launch_bounds__(1024, 1) k_plain_icm_lat(const PtJob* __restrict__ jp, PlainCtl* ctl,
                                                           long long* icm_dE, uint32_t* icm_valid,
                                                           unsigned long long* dm, int stage_exch) {
  pdl_enter();
  extern __shared__ uint4 smem_u4[];
  __shared__ PtJob s_J;
  load_job(s_J, jp);
  const PtJob& J = s_J;
  constexpr uint32_t DEG = 2 * DIM;
  constexpr uint32_t n = DIM == 2 ? L * L : L * L * L;
  constexpr uint32_t NW = n / 32;                  // bitmap words
  constexpr uint32_t WPP = L * L / 32;             // words per plane of L rows
  constexpr uint32_t G = (NW + 31) / 32 * 32;      // threads of the growth group
  static_assert(G < 1024, "the growth group leaves threads for the staging");
  const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5, nwarp = blockDim.x >> 5;
  const uint32_t T = blockDim.x;
  const uint32_t nact = J.nt - J.lo;
  const uint32_t p = blockIdx.x / nact, t = J.lo + blockIdx.x % nact;
  const uint32_t b = t & 31u, w = t >> 5, tb = 32 * w;
  const uint32_t nw = J.nw, o0 = 2 * p * J.wpc + w, o1 = (2 * p + 1) * J.wpc + w;
  const uint32_t nnz = J.F.nnz;
  char* base = reinterpret_cast<char*>(smem_u4);
  LatScratch X;
  char* const xbase = base + carve_lat(&X, base, n, nnz);  // the exchange's staged inputs (stage_exch)
  uint32_t* const Wg = J.W;
  PhaseClock pc;  // with profiling on, cycles are summed over the CTAs
  pc.start(J.prof);
  // the slot's q<0 bits and replica 0's spin bits in colour order (ballots;
  // a warp's words at most NW / 32 <= 4, their loads issued together)
  constexpr uint32_t WPW = NW >= 32 * 32 ? 32 : (NW + 31) / 32;  // words per warp
  {
    uint32_t v0[WPW], v1[WPW];
#pragma unroll
    for (uint32_t k = 0; k < WPW; ++k) {
      const uint32_t wc = warp + k * nwarp;
      const uint32_t s = 32 * wc + lane;
      v0[k] = wc < NW ? Wg[(size_t)s * nw + o0] : 0u;
      v1[k] = wc < NW ? Wg[(size_t)s * nw + o1] : 0u;
    }
#pragma unroll
    for (uint32_t k = 0; k < WPW; ++k) {
      const uint32_t wc = warp + k * nwarp;
      const uint32_t dq = __ballot_sync(0xffffffffu, ((v0[k] ^ v1[k]) >> b) & 1u);
      const uint32_t r0 = __ballot_sync(0xffffffffu, (v0[k] >> b) & 1u);
      if (lane == 0 && wc < NW) {
        X.Dcol[wc] = dq;
        X.R0col[wc] = r0;
      }
    }
  }
  uint32_t ip[WPW];  // file order -> colour order of this lane's sites
#pragma unroll
  for (uint32_t k = 0; k < WPW; ++k) {
    const uint32_t wo = warp + k * nwarp;
    ip[k] = wo < NW ? J.F.iperm[32 * wo + lane] : 0u;
  }
  __syncthreads();
  // the q<0 bits in original order; the cluster starts empty
#pragma unroll
  for (uint32_t k = 0; k < WPW; ++k) {
    const uint32_t wo = warp + k * nwarp;
    const uint32_t s = ip[k];
    const uint32_t dq = __ballot_sync(0xffffffffu, wo < NW && ((X.Dcol[s >> 5] >> (s & 31u)) & 1u));
    if (lane == 0 && wo < NW) {
      X.Do[wo] = dq;
      X.Co[wo] = 0;
    }
  }
  // seed (warp 0): the k-th q<0 site in colour order, k = floor(u cnt / 2^32)
  if (warp == 0) {
    uint32_t cnt = 0;
    for (uint32_t c0 = 0; c0 < NW; c0 += 32)
      cnt += c0 + lane < NW ? (uint32_t)__popc(X.Dcol[c0 + lane]) : 0u;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    uint32_t seed = 0xffffffffu;
    if (cnt) {
      const uint32_t u = philox4x32_10(make_uint4(tb + b, ctl->i, p, PTAG_ICM), J.key).x;
      uint32_t k = (uint32_t)(((uint64_t)u * cnt) >> 32);
      for (uint32_t c0 = 0; c0 < NW; c0 += 32) {
        const uint32_t m = c0 + lane < NW ? X.Dcol[c0 + lane] : 0u;
        const uint32_t cc = __popc(m);
        uint32_t incl = cc;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= (uint32_t)o) incl += v;
        }
        const uint32_t tot = __shfl_sync(0xffffffffu, incl, 31);
        if (k < tot) {
          const uint32_t excl = incl - cc;
          const uint32_t hit = __ballot_sync(0xffffffffu, k >= excl && k < incl);
          const uint32_t src = __ffs(hit) - 1;
          seed = (c0 + src) * 32 + __fns(__shfl_sync(0xffffffffu, m, src), 0,
                                         (int)(k - __shfl_sync(0xffffffffu, excl, src)) + 1);
          break;
        }
        k -= tot;
      }
    }
    if (lane == 0) {
      X.misc[0] = cnt;
      X.misc[1] = seed;
    }
  }
  __syncthreads();
  pc.lap(PHASE_ICM_SCAN);
  const uint32_t cnt = X.misc[0];
  if (tid < G) {
    // growth group: thread tid owns bitmap word tid.  Inside a pass a warp
    // repeats its words' updates while any of them grows (its words are
    // neighbouring rows and planes), then the group's barrier
    if (cnt && tid == 0) {
      const uint32_t o = J.F.perm[X.misc[1]];
      X.Co[o >> 5] = 1u << (o & 31u);
    }
    bar1_or(0, G);
    const uint32_t wi = tid;
    const bool own = cnt && wi < NW;
    const uint32_t d = own ? X.Do[wi] : 0u;
    uint32_t c = own ? X.Co[wi] : 0u;
    const uint32_t j = wi % WPP, plane0 = wi - j;
    const uint32_t wym = plane0 + (j + WPP - 1) % WPP, wyp = plane0 + (j + 1) % WPP;
    const uint32_t wxm = (wi + NW - WPP) % NW, wxp = (wi + WPP) % NW;
    for (uint32_t pass = 0; cnt && pass < n + 2u; ++pass) {
      int grew = 0;
      for (uint32_t rep = 0; rep < 64u; ++rep) {
        int g = 0;
        if (own && d != c) {
          const uint32_t c_in = c;
          uint32_t nb = L == 16 ? (X.Co[wym] >> 16) | (X.Co[wyp] << 16) : X.Co[wym] | X.Co[wyp];
          if (DIM == 3) nb |= X.Co[wxm] | X.Co[wxp];
          c = lat_close<L>(c | (d & nb), d);  // the neighbours' bits, then the closure inside the word
          if (c != c_in) {
            X.Co[wi] = c;
            g = 1;
          }
        }
        grew |= g;
        if (!__any_sync(0xffffffffu, g)) break;
        __syncwarp();
      }
      if (!bar1_or(grew, G)) break;
    }
  } else {
    // staging group: couplings, columns, fields and the colour -> file order
    // permutation into shared memory while the cluster grows
    // (asynchronous 16-byte copies, all in flight at once)
    const uint32_t st = tid - G, ns = T - G;
    auto copy16 = [&](void* dst, const void* src, uint32_t n16) {
      const uint32_t d0 = (uint32_t)__cvta_generic_to_shared(dst);
      const char* s0 = static_cast<const char*>(src);
      for (uint32_t x = st; x < n16; x += ns)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d0 + 16 * x), "l"(s0 + 16 * (size_t)x)
                     : "memory");
    };
    copy16(X.Jf, J.F.fJt, nnz / 4);
    copy16(X.cols, J.F.fcolt, nnz / 8);
    copy16(X.bias, J.F.bias, n / 4);
    copy16(X.perm, J.F.perm, n / 4);
    // every CTA stages the exchange's inputs (only the last one uses them), so
    // that the exchange reads just the Houdayer changes from L2
    if (stage_exch) plain_exch_stage(J, xbase, st, ns);
    asm volatile("cp.async.wait_all;\n" ::: "memory");
  }
  __syncthreads();
  pc.lap(PHASE_ICM_GROW);
  long long a0 = 0;
  if (cnt) {
    // the cluster in colour order
    for (uint32_t wc = warp; wc < NW; wc += nwarp) {
      const uint32_t o = X.perm[32 * wc + lane];
      const uint32_t cb = __ballot_sync(0xffffffffu, (X.Co[o >> 5] >> (o & 31u)) & 1u);
      if (lane == 0) X.Ccol[wc] = cb;
    }
    __syncthreads();
    // energy change of flipping the cluster in replica 0: boundary terms
    // -2 s_i (h_i + sum_{j not in cluster} J_ij s_j), f32 in row order, summed
    // in fixed point (replica 1's sum is the exact negative)
    auto bit = [](const uint32_t* m, uint32_t s) { return (m[s >> 5] >> (s & 31u)) & 1u; };
    for (uint32_t s = tid; s < n; s += T) {
      if (!bit(X.Ccol, s)) continue;
      // every neighbour's column, coupling and bits loaded before the sum
      uint32_t jj[DEG], cw[DEG], rw[DEG];
      float Jv[DEG];
#pragma unroll
      for (uint32_t m = 0; m < DEG; ++m) {
        jj[m] = X.cols[m * n + s];
        Jv[m] = X.Jf[m * n + s];
      }
#pragma unroll
      for (uint32_t m = 0; m < DEG; ++m) {
        cw[m] = X.Ccol[jj[m] >> 5];
        rw[m] = X.R0col[jj[m] >> 5];
      }
      float f0 = X.bias[s];
#pragma unroll
      for (uint32_t m = 0; m < DEG; ++m) {
        const uint32_t sh = jj[m] & 31u;
        if (jj[m] == s || ((cw[m] >> sh) & 1u)) continue;
        f0 += ((rw[m] >> sh) & 1u) ? -Jv[m] : Jv[m];
      }
      const float s0 = bit(X.R0col, s) ? -1.0f : 1.0f;
      a0 += to_fx(-2.0f * s0 * f0);
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) a0 += __shfl_xor_sync(0xffffffffu, a0, off);
    if (lane == 0) X.part[warp] = a0;
    __syncthreads();
    if (warp == 0) {  // only thread 0 uses the total (integers: any order)
      a0 = 0;
      for (uint32_t k = lane; k < nwarp; k += 32) a0 += X.part[k];
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) a0 += __shfl_xor_sync(0xffffffffu, a0, off);
    }
    pc.lap(PHASE_ICM_MARK);
    // flip the cluster in both replicas
    for (uint32_t s = tid; s < n; s += T)
      if (bit(X.Ccol, s)) {
        atomicXor(&Wg[(size_t)s * nw + o0], 1u << b);
        atomicXor(&Wg[(size_t)s * nw + o1], 1u << b);
      }
  }
  __syncthreads();
  if (tid == 0) {
    const uint32_t x0 = 2 * p * J.ntp + t, x1 = (2 * p + 1) * J.ntp + t;
    icm_valid[x0] = cnt != 0;
    icm_valid[x1] = cnt != 0;
    icm_dE[x0] = a0;
    icm_dE[x1] = -a0;
  }
  pc.lap(PHASE_ICM_APPLY);
  // the last CTA to finish runs the exchange of the round (as k_plain_icm)
  __shared__ int s_last;
  __syncthreads();
  if (tid == 0) {
    __threadfence();
    s_last = atomicAdd(&ctl->icm_done, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  if (tid == 0) ctl->icm_done = 0;
  plain_exchange_body(J, ctl, icm_dE, icm_valid, stage_exch ? xbase : base, dm, stage_exch != 0);
}

// Houdayer moves of round ctl->i on thread-block clusters: one cluster of CL
// CTAs per (chain pair, slot >= lo), each CTA owning the sites of one
// contiguous colour-order range (on square and cubic lattices a slab of the
// lattice).  Every CTA keeps full copies of the disagreement words XD, the
// cluster words XC and replica 0's words R0 in its shared memory; a site's
// owner updates it and, when a neighbour lives in another range, stores the
// new word into the other CTAs' copies through distributed shared memory.
//   seed    each CTA counts the q<0 sites of its range (ballots), the counts
//           are exchanged, and the CTA holding the k-th site in colour order
//           (the rule of icm_group) publishes it;
//   growth  in-place propagation passes (icm_group's rule C[s] |= D[s] & OR_j C[j],
//           the site state and columns in registers), a cluster barrier per
//           pass, each CTA's "grew" flag stored into every CTA before it;
//   apply   each CTA sums the boundary terms of its cluster sites (fixed
//           point, integer sums) and flips them; CTA 0 adds the partial sums.
// The cluster is the exact component of the seed, the sums are integers, so
// the result equals the one-CTA kernel's bit for bit.  Rows of DEG entries
// (uniform degree); at most PS sites per thread and range.
struct IcmClScratch {
  uint32_t *XD, *XC, *R0;
  uint16_t* cols;          // [PS * T][DEG] columns of this CTA's sites
  uint32_t* cnt;           // [CL] q<0 counts per range
  uint32_t* seed;          // [1]
  uint32_t* flags;         // [2][CL] per-pass "grew" flags, by pass parity
  long long* part;         // [CL] partial energy sums (in CTA 0)
  long long* wsum;         // [32] per-warp sums
  uint32_t* wcnt;          // [32] per-warp counts
};
__host__ __device__ inline size_t carve_icm_cl(IcmClScratch* X, char* base, uint32_t n, uint32_t T, uint32_t PS,
                                               uint32_t DEG, uint32_t CL) {
  size_t o = 0;
  auto take = [&](size_t bytes) {
    char* p = base ? base + o : nullptr;
    o = al16(o + bytes);
    return p;
  };
  char* XD = take((size_t)n * 4);
  char* XC = take((size_t)n * 4);
  char* R0 = take((size_t)n * 4);
  char* cols = take((size_t)PS * T * DEG * 2);
  char* cnt = take((size_t)CL * 4);
  char* seed = take(4);
  char* flags = take((size_t)2 * CL * 4);
  char* part = take((size_t)CL * 8);
  char* wsum = take(32 * 8);
  char* wcnt = take(32 * 4);
  if (X) {
    X->XD = (uint32_t*)XD;
    X->XC = (uint32_t*)XC;
    X->R0 = (uint32_t*)R0;
    X->cols = (uint16_t*)cols;
    X->cnt = (uint32_t*)cnt;
    X->seed = (uint32_t*)seed;
    X->flags = (uint32_t*)flags;
    X->part = (long long*)part;
    X->wsum = (long long*)wsum;
    X->wcnt = (uint32_t*)wcnt;
  }
  return o;
}

template <uint32_t CL, uint32_t DEG, uint32_t PS>
__global__ void __launch_bounds__(1024, 1) k_plain_icm_cl(const PtJob* __restrict__ jp, PlainCtl* ctl,
                                                          long long* icm_dE, uint32_t* icm_valid,
                                                          unsigned long long* dm) {
  pdl_enter();
  extern __shared__ uint4 smem_u4[];
  __shared__ PtJob s_J;
  load_job(s_J, jp);
  const PtJob& J = s_J;
  cg::cluster_group cluster = cg::this_cluster();
  const uint32_t r = cluster.block_rank();
  const uint32_t tid = threadIdx.x, T = blockDim.x, lane = tid & 31u, warp = tid >> 5, nwarp = T >> 5;
  const uint32_t n = J.n, nw = J.nw, nact = J.nt - J.lo;
  const uint32_t cid = blockIdx.x / CL;
  const uint32_t p = cid / nact, t = J.lo + cid % nact;
  const uint32_t b = t & 31u, bit = 1u << b, w = t >> 5;
  const uint32_t o0 = 2 * p * J.wpc + w, o1 = (2 * p + 1) * J.wpc + w;
  const uint32_t i = ctl->i;
  char* base = reinterpret_cast<char*>(smem_u4);
  IcmClScratch X;
  carve_icm_cl(&X, base, n, T, PS, DEG, CL);
  const uint32_t span = (n + CL - 1) / CL;
  const uint32_t lo = min(n, r * span), hi = min(n, lo + span);
  uint32_t* const W = J.W;
  PhaseClock pc;
  pc.start(r == 0 ? J.prof : nullptr);
  // full copies of the disagreement and replica-0 words; columns of own sites
  for (uint32_t s = tid; s < n; s += T) {
    const uint32_t v0 = W[s * nw + o0], v1 = W[s * nw + o1];
    X.XD[s] = (v0 ^ v1) & bit;
    X.R0[s] = v0;
    X.XC[s] = 0;
  }
  for (uint32_t x = tid; x < (hi - lo) * DEG; x += T) X.cols[x] = J.F.col16[lo * DEG + x];
  if (tid < 2 * CL) X.flags[tid] = 0;
  __syncthreads();
  cluster.sync();  // every CTA of the cluster has started and cleared its copies
  // ---- seed: q<0 counts of every range, then the k-th site in colour order
  const uint32_t seg = ((hi - lo + nwarp - 1) / nwarp + 31u) & ~31u;
  const uint32_t w0 = min(hi, lo + warp * seg), w1 = min(hi, w0 + seg);
  uint32_t wc = 0;
  for (uint32_t s0 = w0; s0 < w1; s0 += 32) {
    const uint32_t s = s0 + lane;
    wc += __popc(__ballot_sync(0xffffffffu, s < w1 && X.XD[s]));
  }
  if (lane == 0) X.wcnt[warp] = wc;
  __syncthreads();
  const uint32_t v = lane < nwarp ? X.wcnt[lane] : 0u;
  uint32_t incl = v;
  for (int off = 1; off < 32; off <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, incl, off);
    if (lane >= (uint32_t)off) incl += y;
  }
  const uint32_t cnt_r = __shfl_sync(0xffffffffu, incl, 31);
  const uint32_t before_w = __shfl_sync(0xffffffffu, incl - v, warp);
  if (tid == 0)
    for (uint32_t q = 0; q < CL; ++q) cluster.map_shared_rank(X.cnt, q)[r] = cnt_r;
  cluster.sync();
  uint32_t total = 0, before_r = 0;
  for (uint32_t q = 0; q < CL; ++q) {
    const uint32_t c = X.cnt[q];
    if (q < r) before_r += c;
    total += c;
  }
  if (total) {
    const uint32_t u = philox4x32_10(make_uint4(32 * w + b, i, p, PTAG_ICM), J.key).x;
    const uint32_t k = (uint32_t)(((uint64_t)u * total) >> 32);
    const uint32_t kb = before_r + before_w;
    if (k >= kb && k < kb + wc) {
      uint32_t rem = k - kb;
      for (uint32_t s0 = w0; s0 < w1; s0 += 32) {
        const uint32_t s = s0 + lane;
        const uint32_t bal = __ballot_sync(0xffffffffu, s < w1 && X.XD[s]);
        const uint32_t c = __popc(bal);
        if (rem < c) {
          if (lane == 0) {
            const uint32_t sd = s0 + __fns(bal, 0, (int)rem + 1);
            for (uint32_t q = 0; q < CL; ++q) *cluster.map_shared_rank(X.seed, q) = sd;
          }
          break;
        }
        rem -= c;
      }
    }
  }
  cluster.sync();
  pc.lap(PHASE_ICM_SCAN);
  if (total) {
    if (tid == 0) X.XC[*X.seed] = bit;
    __syncthreads();
    // ---- growth: propagation passes over this CTA's sites
    // two 16-bit columns per register
    constexpr uint32_t NP = DEG / 2;
    uint32_t d[PS], c[PS], jp[PS][NP];
    bool edge[PS];
#pragma unroll
    for (uint32_t k = 0; k < PS; ++k) {
      const uint32_t s = lo + tid + k * T;
      d[k] = 0;
      c[k] = 0;
      edge[k] = false;
#pragma unroll
      for (uint32_t m = 0; m < NP; ++m) jp[k][m] = 0;
      if (s < hi) {
        d[k] = X.XD[s];
        c[k] = X.XC[s];
#pragma unroll
        for (uint32_t m = 0; m < NP; ++m) {
          const uint32_t ja = X.cols[(s - lo) * DEG + 2 * m], jb = X.cols[(s - lo) * DEG + 2 * m + 1];
          jp[k][m] = ja | (jb << 16);
          edge[k] |= ja < lo || ja >= hi || jb < lo || jb >= hi;
        }
      }
    }
    for (uint32_t pass = 0; pass < 32u * n + 2u; ++pass) {
      int grew = 0;
#pragma unroll
      for (uint32_t k = 0; k < PS; ++k) {
        if ((c[k] & d[k]) == d[k]) continue;
        uint32_t nb = 0;
#pragma unroll
        for (uint32_t m = 0; m < NP; ++m) nb |= X.XC[jp[k][m] & 0xffffu] | X.XC[jp[k][m] >> 16];
        const uint32_t nc = c[k] | (nb & d[k]);
        if (nc != c[k]) {
          const uint32_t s = lo + tid + k * T;
          c[k] = nc;
          X.XC[s] = nc;
          grew = 1;
          if (edge[k])
            for (uint32_t q = 0; q < CL; ++q)
              if (q != r) cluster.map_shared_rank(X.XC, q)[s] = nc;
        }
      }
      const int any_cta = __syncthreads_or(grew);
      const uint32_t par = pass & 1u;
      if (tid == 0) {
        if (any_cta)
          for (uint32_t q = 0; q < CL; ++q) cluster.map_shared_rank(X.flags, q)[par * CL + r] = 1u;
        for (uint32_t q = 0; q < CL; ++q) X.flags[(par ^ 1u) * CL + q] = 0u;  // written no earlier than next pass
      }
      cluster.sync();
      uint32_t any = 0;
      for (uint32_t q = 0; q < CL; ++q) any |= X.flags[par * CL + q];
      if (!any) break;
    }
  }
  pc.lap(PHASE_ICM_GROW);
  // ---- energy change of the flip (replica 0; replica 1's is its negative) and the flip
  long long a0 = 0;
  if (total) {
    const uint2* __restrict__ ent = J.F.ent;
    const float* __restrict__ bias = J.F.bias;
    for (uint32_t s = lo + tid; s < hi; s += T) {
      if (!(X.XC[s] & bit)) continue;
      float f0 = bias[s];
      uint2 ce[DEG];
#pragma unroll
      for (uint32_t m = 0; m < DEG; ++m) ce[m] = ent[s * DEG + m];
#pragma unroll
      for (uint32_t m = 0; m < DEG; ++m) {
        if (ce[m].x == s || (X.XC[ce[m].x] & bit)) continue;
        const float Jv = __uint_as_float(ce[m].y);
        f0 += (X.R0[ce[m].x] & bit) ? -Jv : Jv;
      }
      const float s0 = (X.R0[s] & bit) ? -1.0f : 1.0f;
      a0 += to_fx(-2.0f * s0 * f0);
      atomicXor(&W[s * nw + o0], bit);
      atomicXor(&W[s * nw + o1], bit);
    }
  }
  for (int off = 16; off > 0; off >>= 1) a0 += __shfl_xor_sync(0xffffffffu, a0, off);
  if (lane == 0) X.wsum[warp] = a0;
  __syncthreads();
  if (tid == 0) {
    long long sum = 0;
    for (uint32_t k = 0; k < nwarp; ++k) sum += X.wsum[k];
    cluster.map_shared_rank(X.part, 0)[r] = sum;
  }
  cluster.sync();  // the last access to another CTA's shared memory
  if (r == 0 && tid == 0) {
    long long sum = 0;
    for (uint32_t q = 0; q < CL; ++q) sum += X.part[q];
    const uint32_t x0 = 2 * p * J.ntp + t, x1 = (2 * p + 1) * J.ntp + t;
    const uint32_t valid = total != 0;
    icm_valid[x0] = valid;
    icm_valid[x1] = valid;
    icm_dE[x0] = valid ? sum : 0;
    icm_dE[x1] = valid ? -sum : 0;
  }
  pc.lap(PHASE_ICM_APPLY);
  // the last CTA to finish runs the exchange of the round (as k_plain_icm)
  __shared__ int s_last;
  __syncthreads();
  if (tid == 0) {
    __threadfence();
    s_last = atomicAdd(&ctl->icm_done, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  if (tid == 0) ctl->icm_done = 0;
  plain_exchange_body(J, ctl, icm_dE, icm_valid, base, dm);
}

// Energies after the Houdayer moves and the exchange decisions of round
// ctl->i (the spin permutation follows in k_plain_perm); advances ctl->i.
// `base` is shared memory for Ec, Er and Dm; dm receives Dm for k_plain_perm.
// With `staged`, the energies (without this round's Houdayer changes) and the
// exchange bookkeeping are already in `base`'s layout (plain_exch_stage): only
// the Houdayer changes are read from global memory.
__device__ void plain_exchange_body(const PtJob& J, PlainCtl* ctl, const long long* icm_dE, uint32_t* icm_valid,
                                    char* base, unsigned long long* dm, bool staged) {
  const uint32_t tid = threadIdx.x;
  Smem S{};
  S.Ec = (double*)base;
  S.Er = (double*)(base + al16((size_t)J.C * J.ntp * 8));
  S.Dm = (unsigned long long*)(base + 2 * al16((size_t)J.C * J.ntp * 8));
  S.W = J.W;
  S.xb = base + plain_head_smem(J.n, J.C, J.ntp);
  const uint32_t CN = J.C * J.ntp;
  for (uint32_t x = tid; x < CN; x += blockDim.x) {
    double ec = staged ? S.Ec[x] : J.Ec[x], er = staged ? S.Er[x] : J.Er[x];
    // written by other CTAs of the Houdayer kernel: read through L2
    if (J.icm && __ldcg(icm_valid + x)) {  // invalidated caches are recomputed as energy_ref
      er += (double)__ldcg(icm_dE + x) * TAMC_FX_INV;
      ec = er;
      icm_valid[x] = 0;
    }
    S.Ec[x] = ec;
    S.Er[x] = er;
  }
  if (staged) {
    __syncthreads();
  } else {
    // the exchange bookkeeping in shared memory: one round of parallel global
    // loads and stores instead of dependent global round trips in the decisions;
    // staged by the threads above the energies' so that both sets of loads are
    // in flight together (its closing barrier covers the energies too)
    const uint32_t t0 = (CN + 31) / 32 * 32;
    xchg_load(J, S.xb, false, t0 + 32 <= blockDim.x ? t0 : 0);
  }
  PhaseClock pc;
  pc.start(J.prof);
  const uint32_t i = ctl->i;
  exchange_decide(J, S, i);
  xchg_store(J, S.xb, false);
  for (uint32_t x = tid; x < CN; x += blockDim.x) {
    J.Ec[x] = S.Ec[x];
    J.Er[x] = S.Er[x];
  }
  for (uint32_t c = tid; c < J.C; c += blockDim.x) dm[c] = S.Dm[c];
  __syncthreads();
  pc.lap(PHASE_EXCH);
  if (tid == 0) {
    ctl->i = i + 1;
    ctl->pending = 1;
  }
}

// Exchange of round ctl->i when no Houdayer kernel ran (icm off, or no slot >= lo).
__global__ void __launch_bounds__(1024, 1) k_plain_exch(const PtJob* __restrict__ jp, PlainCtl* ctl,
                                                       const long long* icm_dE, uint32_t* icm_valid,
                                                       unsigned long long* dm) {
  pdl_enter();
  extern __shared__ uint4 smem_u4[];
  __shared__ PtJob s_J;
  load_job(s_J, jp);
  plain_exchange_body(s_J, ctl, icm_dE, icm_valid, reinterpret_cast<char*>(smem_u4), dm);
}

// Spin permutation of the exchange: one thread per (site, chain) word pair.
__global__ void __launch_bounds__(256) k_plain_perm(const PtJob* __restrict__ jp, const unsigned long long* dm) {
  pdl_enter();
  const PtJob& J = *jp;
  const uint32_t C = J.C, wpc = J.wpc, nw = J.nw;
  uint32_t* const W = J.W;
  const uint64_t total = (uint64_t)J.n * C;
  for (uint64_t x = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; x < total;
       x += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t s = (uint32_t)(x / C), c = (uint32_t)(x % C);
    const uint64_t D = dm[c];
    if (!D) continue;
    uint32_t* w = W + (size_t)s * nw + c * wpc;
    uint64_t v = w[0];
    if (wpc > 1) v |= (uint64_t)w[1] << 32;
    v = bitperm(v, D);
    w[0] = (uint32_t)v;
    if (wpc > 1) w[1] = (uint32_t)(v >> 32);
  }
}

// The grid stride is a multiple of qps, so every thread keeps one quad k for
// all its tasks and accumulates its fixed-point ΔE sums in registers; a CTA
// combines its threads per slot and adds one 64-bit atomic per slot.
// Closes round ctl->i - 1 after its last sweep launch, in the launch's last
// CTA, when the round takes no measurement: adds the fixed-point sweep sums to
// the energies and tracks the ground state (a new minimum's state included),
// as k_plain_head would; a measured round is left to k_plain_head.  `base`:
// shared memory for Ec and Er.
__device__ void plain_close_round(const PtJob& J, PlainCtl* ctl, long long* acc, char* base) {
  const uint32_t tid = threadIdx.x;
  const uint32_t ip = ctl->i - 1;
  const bool measured = ip >= J.meas_init && (sched(J.sample, ip, J.meas_init, J.num_sweeps) ||
                                              sched(J.sample_states, ip, J.meas_init, J.num_sweeps));
  if (!measured) {
    Smem S{};
    S.Ec = (double*)base;
    S.Er = (double*)(base + al16((size_t)J.C * J.ntp * 8));
    S.W = J.W;
    const uint32_t CN = J.C * J.ntp;
    for (uint32_t x = tid; x < CN; x += blockDim.x) {
      // written by other CTAs' atomics: read through L2
      const long long a = (long long)__ldcg((const unsigned long long*)acc + x);
      const long long aq = (long long)__ldcg((const unsigned long long*)acc + CN + x);
      S.Ec[x] = J.Ec[x] + (double)a * TAMC_FX_INV;
      S.Er[x] = J.Er[x] + (double)(a + aq) * TAMC_FX_INV;
      acc[x] = 0;
      acc[CN + x] = 0;
    }
    __syncthreads();
    if (ip >= J.meas_init) {
      const GsSnap g = gs_track(J, S, ip);
      uint32_t m_cur = ctl->m_cur, s_cur = ctl->s_cur;  // unchanged: no measurement this round
      measure_rest(J, J.F, S, J.F.sus, J.F.iperm, ip, m_cur, s_cur, g, nullptr);
    }
    for (uint32_t x = tid; x < CN; x += blockDim.x) {
      J.Ec[x] = S.Ec[x];
      J.Er[x] = S.Er[x];
    }
  }
  __syncthreads();
  if (tid == 0) {
    if (!measured) ctl->pending = 0;
    ctl->sweep_done = 0;
  }
}

template <bool SELF, uint32_t DEG, bool CLOSE>
__global__ void __launch_bounds__(256, 3) k_plain_sweep(const PtJob* __restrict__ jp, PlainCtl* ctl, uint32_t color,
                                                     long long* acc) {
  pdl_enter();
  extern __shared__ uint4 smem_u4[];
  const PtJob& J = *jp;
  Fx4* red = reinterpret_cast<Fx4*>(smem_u4);                 // [blockDim.x]
  float4* b4 = reinterpret_cast<float4*>(red + blockDim.x);   // [qps]
  const float L2E = TAMC_2LOG2E;
  for (uint32_t k = threadIdx.x; k < J.qps; k += blockDim.x) {
    const uint32_t q = k % J.qpc;
    b4[k] = make_float4(J.betas[4 * q] * L2E, J.betas[4 * q + 1] * L2E, J.betas[4 * q + 2] * L2E,
                        J.betas[4 * q + 3] * L2E);
  }
  __syncthreads();
  const uint32_t i = ctl->i - 1;
  const uint32_t c0 = J.F.color_off[color], nc = J.F.color_off[color + 1] - c0;
  const uint64_t gtid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t gstride = (uint64_t)gridDim.x * blockDim.x;
  const uint32_t k = (uint32_t)(gtid % J.qps);
  const uint32_t ch = k / J.qpc, q = k % J.qpc;
  const uint32_t wo = ch * J.wpc + (q >> 3), shift = 4 * (q & 7u);
  const float4 b2 = b4[k];
  const FastInst F = J.F;
  const uint2 key = J.key;
  uint32_t* const W = J.W;
  const uint32_t nw = J.nw;
  const uint64_t s_first = gtid / J.qps, s_step = gstride / J.qps;
  Fx4 a{0, 0, 0, 0}, aq{0, 0, 0, 0};
  // two sites of the class per step, all their loads issued before either is
  // decided (sites of one colour class share no bond, so neither update can
  // change what the other reads); the sums are integers, so the order of the
  // updates does not matter
  auto apply = [&](uint32_t s, uint32_t m) {
    if (!m) return;
    atomicXor(&W[s * nw + wo], m << shift);
    if (SELF) {
      const long long k2 = to_fx(2.0f * F.kd[s]);
      aq.x += (m & 1u) ? k2 : 0;
      aq.y += (m & 2u) ? k2 : 0;
      aq.z += (m & 4u) ? k2 : 0;
      aq.w += (m & 8u) ? k2 : 0;
    }
  };
  for (uint64_t site = s_first; site < nc; site += 2 * s_step) {
    const uint32_t sa = c0 + (uint32_t)site;
    const bool two = site + s_step < nc;
    const uint32_t sb = two ? c0 + (uint32_t)(site + s_step) : sa;
    const float4 fa = quad_field<DEG>(sa, shift, F, W, nw, wo);
    const uint32_t oa = W[sa * nw + wo] >> shift;
    float4 fb = fa;
    uint32_t ob = oa;
    if (two) {
      fb = quad_field<DEG>(sb, shift, F, W, nw, wo);
      ob = W[sb * nw + wo] >> shift;
    }
    const uint32_t ma =
        quad_accept<true>(fa, oa, b2, philox4x32_10(make_uint4(sa, i, ch * 16u + q, PTAG_SWEEP), key), a);
    apply(sa, ma);
    if (two) {
      const uint32_t mb =
          quad_accept<true>(fb, ob, b2, philox4x32_10(make_uint4(sb, i, ch * 16u + q, PTAG_SWEEP), key), a);
      apply(sb, mb);
    }
  }
  const uint32_t CN = J.C * J.ntp;
  for (int pass = 0; pass < (SELF ? 2 : 1); ++pass) {
    red[threadIdx.x] = pass ? aq : a;
    __syncthreads();
    // threads of this CTA holding quad kk: tid with (blockIdx.x*blockDim.x + tid) % qps == kk
    for (uint32_t x = threadIdx.x; x < CN; x += blockDim.x) {
      const uint32_t c = x / J.ntp, t = x % J.ntp;
      const uint32_t kk = c * J.qpc + t / 4;
      const uint32_t first = (uint32_t)((kk + J.qps - (uint64_t)blockIdx.x * blockDim.x % J.qps) % J.qps);
      long long sum = 0;
      for (uint32_t th = first; th < blockDim.x; th += J.qps) {
        const Fx4 v = red[th];
        sum += (t & 3u) == 0 ? v.x : (t & 3u) == 1 ? v.y : (t & 3u) == 2 ? v.z : v.w;
      }
      if (sum) atomicAdd((unsigned long long*)&acc[pass * CN + x], (unsigned long long)sum);
    }
    __syncthreads();
  }
  if (CLOSE) {
    __shared__ int s_last;
    if (threadIdx.x == 0) {
      __threadfence();
      s_last = atomicAdd(&ctl->sweep_done, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    plain_close_round(J, ctl, acc, reinterpret_cast<char*>(b4 + J.qps));
  }
}

// Multi-spin-coded sweep of one colour class for a +-J instance (J.msc): the
// fused kernel's sweep_phase_msc spread over the grid -- global warp g updates
// replica word g % nw of 32 consecutive sites per step -- with the same random
// words, so both forms stay identical.  Per-replica energy sums: bit
// transposes per warp, then one 64-bit atomic per replica and CTA.
template <uint32_t DEG, bool CLOSE>
__global__ void __launch_bounds__(256, 3) k_plain_sweep_msc(const PtJob* __restrict__ jp, PlainCtl* ctl, uint32_t color,
                                                         long long* acc) {
  pdl_enter();
  extern __shared__ uint4 smem_u4[];
  const PtJob& J = *jp;
  const uint32_t nw = J.nw;
  uint32_t* msc = reinterpret_cast<uint32_t*>(smem_u4);
  long long* red = reinterpret_cast<long long*>(reinterpret_cast<char*>(smem_u4) + al16((size_t)nw * MSC_WORDS * 4));
  msc_fill_planes<DEG>(J, msc);
  __syncthreads();
  const uint32_t i = ctl->i - 1;
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  const uint32_t gw = blockIdx.x * nwarp + warp, G = gridDim.x * nwarp;  // G % nw == 0
  const uint32_t wo = gw % nw;
  const uint32_t* pl = msc + wo * MSC_WORDS;
  const uint32_t c0 = J.F.color_off[color], c1 = J.F.color_off[color + 1];
  const uint2* __restrict__ ent = J.F.ent;
  uint32_t* const W = J.W;
  long long e = 0;
  for (uint32_t base = c0 + (gw / nw) * 32u; base < c1; base += (G / nw) * 32u) {
    const uint32_t s = base + lane;
    uint32_t flip = 0;
    MscLevels L{};
    if (s < c1) {
      const uint32_t S0 = W[s * nw + wo];
      uint32_t Wj[DEG], neg = 0;
#pragma unroll
      for (uint32_t m = 0; m < DEG; ++m) {
        const uint2 ce = ent[s * DEG + m];
        Wj[m] = W[ce.x * nw + wo];
        neg |= (ce.y >> 31) << m;
      }
      L = msc_levels<DEG>(S0, Wj, neg);
      flip = msc_flip<DEG>(L, pl, pl + 96, pl + 99, s, i, wo, J.key);
      W[s * nw + wo] = S0 ^ flip;
    }
    e += msc_energy<DEG>(flip, L, lane);
  }
  red[warp * 32 + lane] = e;
  __syncthreads();
  for (uint32_t x = threadIdx.x; x < nw * 32; x += blockDim.x) {
    const uint32_t w2 = x / 32, r = x % 32;
    long long sum = 0;
    for (uint32_t ww = w2; ww < nwarp; ww += nw) sum += red[ww * 32 + r];  // warps of word w2 (nwarp % nw == 0)
    const uint32_t c = w2 / J.wpc, t = (w2 % J.wpc) * 32 + r;
    if (t < J.ntp && sum) atomicAdd((unsigned long long*)&acc[c * J.ntp + t], (unsigned long long)sum);
  }
  __syncthreads();
  if (CLOSE) {
    __shared__ int s_last;
    if (threadIdx.x == 0) {
      __threadfence();
      s_last = atomicAdd(&ctl->sweep_done, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    plain_close_round(J, ctl, acc, reinterpret_cast<char*>(red + nwarp * 32));
  }
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
  if (!j.icm_uf && j.n > 65536) return SIZE_MAX;  // the multi-slot search keeps 16-bit site lists
  return carve_all(nullptr, nullptr, j.n, j.nw, j.C, j.ntp, j.qps, T, j.F.nnz, csr_smem, j.icm_group, j.icm_uf != 0);
}

// The fused kernel's dynamic shared-memory limit only grows (per device), so
// that a captured launch stays valid whatever smaller launches ran since.
static void fused_attr(size_t smem) {
  static std::mutex mu;
  static std::map<int, size_t> set;
  int dev = 0;
  TAMC_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  size_t& cur = set[dev];
  if (smem > cur) {
    TAMC_CUDA(cudaFuncSetAttribute(k_pt_fused, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    cur = smem;
  }
}

int fused_blocks_per_sm(uint32_t T, size_t smem) {
  fused_attr(smem);
  int nb = 0;
  TAMC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_pt_fused, (int)T, smem));
  return nb;
}

size_t plain_head_bytes(const PtJob& j, bool stage) {
  size_t b = plain_head_smem(j.n, j.C, j.ntp);
  if (stage)
    b += al16((size_t)j.n * j.nw * 4) + al16((size_t)j.n * 4) + al16((size_t)j.F.nchi * j.n * 8) +
         al16((size_t)j.n * 4);
  return b;
}

// Launches of the plain form's rounds: each kernel may be scheduled while the
// one before it in the stream still runs (programmatic dependent launch; the
// kernels begin with pdl_enter).  TAMC_PDL=0 launches them in plain stream
// order.  Both give the same results: pdl_enter orders every kernel after its
// predecessor.
static bool pdl_on() {
  static const bool on = [] {
    const char* e = getenv("TAMC_PDL");
    return !(e && e[0] == '0');
  }();
  return on;
}

template <typename... KArgs, typename... Args>
static void plain_launch(void (*k)(KArgs...), uint32_t grid, uint32_t block, size_t smem, cudaStream_t st,
                         Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = pdl_on() ? 1 : 0;
  TAMC_CUDA(cudaLaunchKernelEx(&cfg, k, static_cast<KArgs>(args)...));
}

void plain_launch_head(cudaStream_t st, const PtJob* d_job, PlainCtl* ctl, long long* acc, int mode, size_t smem,
                       int stage) {
  TAMC_CUDA(cudaFuncSetAttribute(k_plain_head, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  plain_launch(k_plain_head, 1, 1024, smem, st, d_job, ctl, acc, mode, stage);
}

// Shared memory of the plain Houdayer kernel with the given staging (bit 0:
// adjacency, bit 1: replica words); at least the exchange's.
static size_t plain_icm_smem(const PtJob& j, int stage) {
  size_t b = carve_icm(nullptr, nullptr, 0, j.n, 1, j.icm_uf ? ICM_UF : ICM_BFS_ONE);
  if (stage & 2) b += al16((size_t)j.n * 4);
  if (stage & 1) b += al16((size_t)(j.n + 1) * 4) + al16((size_t)j.F.nnz * 2);
  return std::max(b, plain_exch_smem(j.n, j.C, j.ntp));
}
size_t plain_icm_bytes(const PtJob& j) { return plain_icm_smem(j, 0); }

// Cluster form of the plain Houdayer kernel: CL CTAs per (pair, slot), chosen
// as the largest of 4 or 2 that keeps every CTA of the launch resident at
// once, for rows of 4 or 6 entries with at most 2 sites per thread and range.
// Returns false (and launches nothing) where it does not apply.
template <uint32_t CL, uint32_t DEG, uint32_t PS>
static void launch_icm_cl(cudaStream_t st, uint32_t nclusters, size_t smem, const PtJob* d_job, PlainCtl* ctl,
                          long long* icm_dE, uint32_t* icm_valid, unsigned long long* dm) {
  auto k = k_plain_icm_cl<CL, DEG, PS>;
  TAMC_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(nclusters * CL);
  cfg.blockDim = dim3(1024);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[2];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = CL;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  attr[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[1].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = pdl_on() ? 2 : 1;
  TAMC_CUDA(cudaLaunchKernelEx(&cfg, k, d_job, ctl, icm_dE, icm_valid, dm));
}

template <uint32_t CL, uint32_t DEG>
static void launch_icm_cl_ps(cudaStream_t st, uint32_t ps, uint32_t nclusters, size_t smem, const PtJob* d_job,
                             PlainCtl* ctl, long long* icm_dE, uint32_t* icm_valid, unsigned long long* dm) {
  if (ps == 1) launch_icm_cl<CL, DEG, 1>(st, nclusters, smem, d_job, ctl, icm_dE, icm_valid, dm);
  else launch_icm_cl<CL, DEG, 2>(st, nclusters, smem, d_job, ctl, icm_dE, icm_valid, dm);
}

static bool plain_launch_icm_cluster(cudaStream_t st, const PtJob& j, const PtJob* d_job, PlainCtl* ctl,
                                     long long* icm_dE, uint32_t* icm_valid, size_t smem_limit, uint32_t num_sms,
                                     unsigned long long* dm) {
  // opt-in: on 3-D L=16 (C4) a cluster launch measured 40.6 us against the
  // one-CTA kernel's 36.7 us (one site per thread loses the two-hop chain of
  // the one-CTA passes, and every pass pays a cluster barrier)
  const char* e = getenv("TAMC_PLAIN_CLUSTER");
  if (!e || e[0] != '1') return false;
  const uint32_t deg = j.F.udeg;
  if (j.icm_uf || !j.F.col16 || (deg != 4 && deg != 6)) return false;
  const uint32_t nclusters = (j.C / 2) * (j.nt - j.lo);
  const uint32_t T = 1024;
  for (uint32_t CL : {4u, 2u}) {
    if (nclusters * CL > num_sms) continue;
    const uint32_t span = (j.n + CL - 1) / CL;
    const uint32_t ps = (span + T - 1) / T;
    if (ps > 2) continue;  // more sites per thread spill at 64 registers
    const uint32_t psr = ps <= 1 ? 1 : 2;
    const size_t smem = std::max(carve_icm_cl(nullptr, nullptr, j.n, T, psr, deg, CL),
                                 plain_exch_smem(j.n, j.C, j.ntp));
    if (smem > smem_limit) continue;
    if (CL == 4) {
      if (deg == 4) launch_icm_cl_ps<4, 4>(st, psr, nclusters, smem, d_job, ctl, icm_dE, icm_valid, dm);
      else launch_icm_cl_ps<4, 6>(st, psr, nclusters, smem, d_job, ctl, icm_dE, icm_valid, dm);
    } else {
      if (deg == 4) launch_icm_cl_ps<2, 4>(st, psr, nclusters, smem, d_job, ctl, icm_dE, icm_valid, dm);
      else launch_icm_cl_ps<2, 6>(st, psr, nclusters, smem, d_job, ctl, icm_dE, icm_valid, dm);
    }
    return true;
  }
  return false;
}

// The bitmap Houdayer kernel on periodic square and cubic lattices of side 16
// or 32 (FastInst::lat_L) when its shared memory fits; TAMC_PLAIN_LATTICE=0
// keeps the site-word kernels (same chain).  Returns false where it does not
// apply.
static bool plain_launch_icm_lattice(cudaStream_t st, const PtJob& j, const PtJob* d_job, PlainCtl* ctl,
                                     long long* icm_dE, uint32_t* icm_valid, size_t smem_limit,
                                     unsigned long long* dm) {
  if (const char* e = getenv("TAMC_PLAIN_LATTICE"))
    if (e[0] == '0') return false;
  const uint32_t L = j.F.lat_L, dim = j.F.udeg / 2;
  if (!L || j.icm_uf || !j.F.fJt || !j.F.fcolt || (dim != 2 && dim != 3)) return false;
  const size_t lat = carve_lat(nullptr, nullptr, j.n, j.F.nnz), exch = plain_exch_smem(j.n, j.C, j.ntp);
  if (std::max(lat, exch) > smem_limit || j.n / 32 >= 1024) return false;
  // the exchange's inputs staged beside the search scratch when both fit
  // (TAMC_PLAIN_XSTAGE=0: the exchange loads them itself)
  int stage_exch = lat + exch <= smem_limit;
  if (const char* e = getenv("TAMC_PLAIN_XSTAGE"))
    if (e[0] == '0') stage_exch = 0;
  const size_t smem = stage_exch ? lat + exch : std::max(lat, exch);
  const uint32_t grid = (j.C / 2) * (j.nt - j.lo);
  auto go = [&](auto k) {
    TAMC_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    plain_launch(k, grid, 1024, smem, st, d_job, ctl, icm_dE, icm_valid, dm, stage_exch);
  };
  if (L == 16 && dim == 2) go(k_plain_icm_lat<16, 2>);
  else if (L == 16 && dim == 3) go(k_plain_icm_lat<16, 3>);
  else if (L == 32 && dim == 2) go(k_plain_icm_lat<32, 2>);
  else return false;  // 32^3: the staged couplings do not fit in shared memory
  return true;
}

bool plain_launch_icm(cudaStream_t st, const PtJob& j, const PtJob* d_job, PlainCtl* ctl, long long* icm_dE,
                      uint32_t* icm_valid, size_t smem_limit, uint32_t num_sms, unsigned long long* dm) {
  const uint32_t nact = j.nt - j.lo, grid = (j.C / 2) * nact;
  if (!j.icm || grid == 0) return false;
  if (plain_launch_icm_lattice(st, j, d_job, ctl, icm_dE, icm_valid, smem_limit, dm)) return true;
  if (plain_launch_icm_cluster(st, j, d_job, ctl, icm_dE, icm_valid, smem_limit, num_sms, dm)) return true;
  // as much staging as fits: words and adjacency, words only, nothing
  int stage = j.F.col16 ? 3 : 2;
  if (plain_icm_smem(j, stage) > smem_limit) stage = 2;
  if (plain_icm_smem(j, stage) > smem_limit) stage = 0;
  const size_t smem = plain_icm_smem(j, stage);
  TAMC_CUDA(cudaFuncSetAttribute(k_plain_icm, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  plain_launch(k_plain_icm, grid, 1024, smem, st, d_job, ctl, icm_dE, icm_valid, stage, dm);
  return true;
}

void plain_launch_exch(cudaStream_t st, const PtJob& j, const PtJob* d_job, PlainCtl* ctl, const long long* icm_dE,
                       uint32_t* icm_valid, unsigned long long* dm) {
  const size_t smem = plain_exch_smem(j.n, j.C, j.ntp);
  TAMC_CUDA(cudaFuncSetAttribute(k_plain_exch, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  plain_launch(k_plain_exch, 1, 1024, smem, st, d_job, ctl, icm_dE, icm_valid, dm);
}

void plain_launch_perm(cudaStream_t st, const PtJob& j, const PtJob* d_job, const unsigned long long* dm,
                       uint32_t grid_cap) {
  const uint64_t total = (uint64_t)j.n * j.C;
  const uint32_t grid = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(grid_cap, (total + 255) / 256));
  plain_launch(k_plain_perm, grid, 256, 0, st, d_job, dm);
}

template <bool CLOSE>
static void plain_launch_sweep_t(cudaStream_t st, const PtJob& j, const PtJob* d_job, PlainCtl* ctl,
                                 uint32_t color, uint32_t grid, uint32_t T, size_t smem, long long* acc) {
  auto go = [&](auto k) {
    TAMC_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    plain_launch(k, grid, T, smem, st, d_job, ctl, color, acc);
  };
  const uint32_t deg = j.F.udeg == 4 || j.F.udeg == 6 ? j.F.udeg : 0;
  if (j.self_loops) {
    if (deg == 4) go(k_plain_sweep<true, 4, CLOSE>);
    else if (deg == 6) go(k_plain_sweep<true, 6, CLOSE>);
    else go(k_plain_sweep<true, 0, CLOSE>);
  } else {
    if (deg == 4) go(k_plain_sweep<false, 4, CLOSE>);
    else if (deg == 6) go(k_plain_sweep<false, 6, CLOSE>);
    else go(k_plain_sweep<false, 0, CLOSE>);
  }
}

void plain_launch_sweep(cudaStream_t st, const PtJob& j, const PtJob* d_job, PlainCtl* ctl, uint32_t color,
                        uint32_t ntask, long long* acc, uint32_t grid_cap) {
  const uint32_t T = 256;
  if (j.msc) {
    // one warp per (32 sites, word): ntask / qps sites in the class
    const uint32_t nsites = ntask / j.qps;
    const uint32_t warps = (nsites + 31) / 32 * j.nw;
    const uint32_t grid = std::max(1u, std::min(grid_cap, (warps + T / 32 - 1) / (T / 32)));
    const bool last = color + 1 == j.F.ncolors;
    const size_t smem = al16((size_t)j.nw * MSC_WORDS * 4) + (size_t)(T / 32) * 32 * 8 +
                        (last ? 2 * al16((size_t)j.C * j.ntp * 8) : 0);
    auto go = [&](auto k) {
      TAMC_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      plain_launch(k, grid, T, smem, st, d_job, ctl, color, acc);
    };
    if (j.F.udeg == 4) {
      if (last) go(k_plain_sweep_msc<4, true>);
      else go(k_plain_sweep_msc<4, false>);
    } else {
      if (last) go(k_plain_sweep_msc<6, true>);
      else go(k_plain_sweep_msc<6, false>);
    }
    TAMC_CUDA(cudaGetLastError());
    return;
  }
  uint32_t grid = std::max(1u, std::min(grid_cap, (ntask + T - 1) / T));
  // grid * T must be a multiple of qps (each thread keeps one quad)
  const uint32_t g = j.qps / std::gcd(j.qps, T);
  grid = std::max(g, (grid + g - 1) / g * g);
  const bool last = color + 1 == j.F.ncolors;
  // the last colour's launch also closes the round: Ec and Er in shared memory
  const size_t smem = (size_t)T * sizeof(Fx4) + (size_t)j.qps * 16 + (last ? 2 * al16((size_t)j.C * j.ntp * 8) : 0);
  if (last) plain_launch_sweep_t<true>(st, j, d_job, ctl, color, grid, T, smem, acc);
  else plain_launch_sweep_t<false>(st, j, d_job, ctl, color, grid, T, smem, acc);
  TAMC_CUDA(cudaGetLastError());
}

void plain_launch_init(cudaStream_t st, const PtJob* d_job, long long* acc, int random, uint32_t grid) {
  if (random) k_plain_init<<<grid, 256, 0, st>>>(d_job, acc, 1);
  k_plain_energy<<<grid, 256, 0, st>>>(d_job, acc);
  TAMC_CUDA(cudaGetLastError());
}

void fused_launch(cudaStream_t st, const PtJob* d_jobs, uint32_t njobs, uint32_t* ctr, uint32_t grid, uint32_t T,
                  size_t smem) {
  fused_attr(smem);
  k_pt_fused<<<grid, T, smem, st>>>(d_jobs, njobs, ctr);
  TAMC_CUDA(cudaGetLastError());
}

void fused_launch_prio(cudaStream_t st, const PtJob* d_jobs, uint32_t njobs, uint32_t* ctr, uint32_t grid, uint32_t T,
                       size_t smem, int priority) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(T);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributePriority;
  at[0].val.priority = priority;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  TAMC_CUDA(cudaLaunchKernelEx(&cfg, k_pt_fused, d_jobs, njobs, ctr));
}

void fused_smem_limit(size_t smem) { fused_attr(smem); }

}  // namespace tamc
