// device.cuh -- device-side building blocks shared by every kernel file.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <mutex>
#include <string>
#include <type_traits>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "expf_exact.h"
#include "internal.h"

namespace tamc {

#define TAMC_CUDA(call)                                                                  \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess)                                                               \
      ::tamc::fail(TAMC_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));     \
  } while (0)

// Bytes this library has copied between host and device (all contexts, since
// load), by direction; reported through tamc_copy_bytes.  Every host<->device
// copy goes through copy_async / copy_sync, or calls count_copy where a
// captured graph replays a copy.
extern std::atomic<uint64_t> g_h2d_bytes, g_d2h_bytes;
inline void count_copy(size_t bytes, cudaMemcpyKind kind) {
  if (kind == cudaMemcpyHostToDevice) g_h2d_bytes.fetch_add(bytes, std::memory_order_relaxed);
  else if (kind == cudaMemcpyDeviceToHost) g_d2h_bytes.fetch_add(bytes, std::memory_order_relaxed);
}
inline cudaError_t copy_async(void* dst, const void* src, size_t bytes, cudaMemcpyKind kind, cudaStream_t st) {
  count_copy(bytes, kind);
  return cudaMemcpyAsync(dst, src, bytes, kind, st);
}
inline cudaError_t copy_sync(void* dst, const void* src, size_t bytes, cudaMemcpyKind kind) {
  count_copy(bytes, kind);
  return cudaMemcpy(dst, src, bytes, kind);
}

// A named NVTX range over a host-side scope (nvtx3, header-only: it costs a
// few nanoseconds unless a profiler such as Nsight Systems is attached, which
// then shows the library's uploads, runs and chunks on its timeline).
struct TraceRange {
  explicit TraceRange(const char* name) { nvtxRangePushA(name); }
  ~TraceRange() { nvtxRangePop(); }
  TraceRange(const TraceRange&) = delete;
  TraceRange& operator=(const TraceRange&) = delete;
};

// Device memory of the library's handles (on the current device).  Blocks up
// to a few MiB come from a per-device cache of freed blocks in power-of-two
// size classes: a freed block first waits in a pending list and becomes
// reusable only after one device synchronisation, so memory that work still
// in flight on any stream reads is never handed out again.  Creating and
// destroying many small runs then costs no cudaMalloc / cudaFree each.
void* dev_alloc(size_t bytes);
void dev_free(void* p, size_t bytes);
// Returns the cached blocks of `device` to the driver.
void dev_cache_release(int device);

// Programmatic dependent launch: a kernel launched with
// cudaLaunchAttributeProgrammaticStreamSerialization may be scheduled while
// the kernel before it in the stream still runs.  It calls this first, on
// every path: wait until that kernel has completed and its writes are
// visible, then let the next kernel of the stream be scheduled.  A kernel so
// launched therefore completes only after its predecessor did, and the
// launch latency of each kernel overlaps the one before it.  Launched without
// the attribute, both instructions return at once.
__device__ __forceinline__ void pdl_enter() {
  asm volatile("griddepcontrol.wait;\n" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
}

// ------------------------------------------------------------ RNG ----
// Philox-4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11): ten rounds of the
// multiply-hi/lo Feistel round with multipliers 0xD2511F53 / 0xCD9E8D57 and
// Weyl key increments 0x9E3779B9 / 0xBB67AE85.
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint32_t lo0 = 0xD2511F53u * c.x, hi0 = __umulhi(0xD2511F53u, c.x);
    const uint32_t lo1 = 0xCD9E8D57u * c.z, hi1 = __umulhi(0xCD9E8D57u, c.z);
    c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
    k.x += 0x9E3779B9u;
    k.y += 0xBB67AE85u;
  }
  return c;
}

// The same generator with each round's two products as 32x32->64 multiplies
// (one wide multiply each instead of a low and a high one): the same outputs.
__device__ __forceinline__ uint4 philox4x32_10w(uint4 c, uint2 k) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint64_t p0 = (uint64_t)0xD2511F53u * c.x, p1 = (uint64_t)0xCD9E8D57u * c.z;
    c = make_uint4((uint32_t)(p1 >> 32) ^ c.y ^ k.x, (uint32_t)p1, (uint32_t)(p0 >> 32) ^ c.w ^ k.y, (uint32_t)p0);
    k.x += 0x9E3779B9u;
    k.y += 0xBB67AE85u;
  }
  return c;
}

// The same generator with the ten round keys computed once (they depend only
// on the seed): saves the two key additions per round in hot loops, and each
// multiply is one 32x32->64 product (a wide multiply instead of separate lo
// and hi; it measured 2.5 % faster in the annealing kernel, but costs
// registers that the kernels at their register limit do not have).
struct PhiloxKeys {
  uint32_t x[10], y[10];
};
__host__ __device__ __forceinline__ PhiloxKeys philox_schedule(uint2 k) {
  PhiloxKeys K;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    K.x[r] = k.x + (uint32_t)r * 0x9E3779B9u;
    K.y[r] = k.y + (uint32_t)r * 0xBB67AE85u;
  }
  return K;
}
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, const PhiloxKeys& K) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint64_t p0 = (uint64_t)0xD2511F53u * c.x, p1 = (uint64_t)0xCD9E8D57u * c.z;
    c = make_uint4((uint32_t)(p1 >> 32) ^ c.y ^ K.x[r], (uint32_t)p1, (uint32_t)(p0 >> 32) ^ c.w ^ K.y[r], (uint32_t)p0);
  }
  return c;
}

// Counter tags that keep the Philox streams of different uses disjoint.
enum : uint32_t {
  PTAG_SWEEP = 0x5357u,   // Metropolis uniforms
  PTAG_INIT = 0x494eu,    // initial spins
  PTAG_ICM = 0x4943u,     // ICM seed-site choice
  PTAG_EXCH = 0x4558u,    // replica-exchange uniforms
  PTAG_MSC = 0x4d53u,     // random words of the multi-spin-coded sweep
};

__host__ __device__ __forceinline__ uint2 philox_key(uint64_t seed) {
  return make_uint2((uint32_t)seed, (uint32_t)(seed >> 32));
}

// Xoshiro256++ (Blackman & Vigna 2018) as used by the reference through
// rand_xoshiro::Xoshiro256PlusPlus; next_u32 = upper half (rand_xoshiro).
struct Xo {
  uint64_t s0, s1, s2, s3;
  __host__ __device__ __forceinline__ uint64_t next() {
    const uint64_t r = ((s0 + s3) << 23 | (s0 + s3) >> 41) + s0;
    const uint64_t t = s1 << 17;
    s2 ^= s0;
    s3 ^= s1;
    s1 ^= s2;
    s0 ^= s3;
    s2 ^= t;
    s3 = (s3 << 45) | (s3 >> 19);
    return r;
  }
  __host__ __device__ __forceinline__ uint32_t next_u32() { return (uint32_t)(next() >> 32); }
  // rand 0.8 `Standard` f32: 24 random bits times 2^-24.
  __host__ __device__ __forceinline__ float std_f32() { return (float)(next_u32() >> 8) * (1.0f / 16777216.0f); }
  // rand 0.8 UniformInt<u32>::sample_single over [0, range), range > 0.
  __host__ __device__ __forceinline__ uint32_t gen_range(uint32_t range) {
#if defined(__CUDA_ARCH__)
    const uint32_t zone = (range << __clz(range)) - 1u;
#else
    const uint32_t zone = (range << __builtin_clz(range)) - 1u;
#endif
    for (;;) {
      const uint32_t v = next_u32();
      const uint64_t m = (uint64_t)v * (uint64_t)range;
      if ((uint32_t)m <= zone) return (uint32_t)(m >> 32);
    }
  }
};

// Host-side seeding (rand_xoshiro seed_from_u64 = SplitMix64 fill) and jump.
Xo xo_seed_from_u64(uint64_t seed);
void xo_jump(Xo& x);

// ------------------------------------------------------- contexts ----
struct ExpTable {
  const uint32_t* off;
  const uint32_t* keys;
  const uint32_t* vals;
};

}  // namespace tamc

struct tamc_gpu {
  int device = 0;
  cudaStream_t stream = nullptr;
  int num_sms = 0;
  size_t smem_optin = 0;
  uint32_t* d_exp = nullptr;  // exception table blob
  tamc::ExpTable exp{};
  std::atomic<uint64_t> launches{0};
  // Handles created from this context (instances, batches, servers) hold a
  // reference; tamc_gpu_close only drops the caller's reference, so a
  // context is released after its last child whatever the destruction order.
  std::atomic<int> refs{1};
  // bulk instance uploads: a pinned staging block (grows, kept for the next
  // call) and a copy stream of their own, one bulk upload at a time
  std::mutex up_mu;
  cudaStream_t up_stream = nullptr;
  char* up_pin = nullptr;
  size_t up_pin_bytes = 0;
  void count(uint64_t k = 1) { launches.fetch_add(k, std::memory_order_relaxed); }
};
void tamc_gpu_retain(tamc_gpu* g);
void tamc_gpu_release(tamc_gpu* g);
namespace tamc {
// Frees the batch chunk runners kept for reuse on this context.
void runner_pool_release(tamc_gpu* g);
}  // namespace tamc

// Reusable device buffers of the host-buffer SA entry point.
struct SaScratch {
  uint32_t* words = nullptr;
  float* energies = nullptr;
  uint8_t* packed = nullptr;
  float* betas = nullptr;
  size_t cap_words = 0, cap_e = 0, cap_packed = 0, cap_betas = 0;
  void ensure(size_t nwords, size_t ne, size_t npacked, size_t nbetas) {
    auto grow = [](auto*& p, size_t& cap, size_t want, size_t elt) {
      if (want <= cap) return;
      if (p) tamc::dev_free(p, cap * elt);
      p = nullptr;
      cap = 0;
      p = static_cast<std::remove_reference_t<decltype(p)>>(tamc::dev_alloc(want * elt));
      cap = want;
    };
    grow(words, cap_words, nwords, 4);
    grow(energies, cap_e, ne, 4);
    grow(packed, cap_packed, npacked, 1);
    grow(betas, cap_betas, nbetas, 4);
  }
  void release() {
    if (words) tamc::dev_free(words, cap_words * 4);
    if (energies) tamc::dev_free(energies, cap_e * 4);
    if (packed) tamc::dev_free(packed, cap_packed);
    if (betas) tamc::dev_free(betas, cap_betas * 4);
    words = nullptr;
    energies = nullptr;
    packed = nullptr;
    betas = nullptr;
    cap_words = cap_e = cap_packed = cap_betas = 0;
  }
};

// Device-resident instance.  Two site orders are kept:
//  * reference order (row i = site i, entries sorted by column, self-loops
//    included) for the reference-order kernels and the ICM graph;
//  * colour order for the fast kernels: sites of colour class 0 first, then
//    class 1, ...; fent[e] = (new column index, J bits) in the reference's
//    per-row order so ΔE is summed in the same order as the reference.
struct tamc_inst {
  tamc_gpu* g = nullptr;
  std::atomic<int> refs{1};  // runs created on the instance hold a reference
  uint32_t n = 0;
  uint64_t nnz = 0;
  float offset = 0.0f;
  uint32_t nchi = 0;
  bool self_loops = false;
  uint32_t max_deg = 0;
  // reference order
  uint32_t* d_rp = nullptr;
  uint32_t* d_col = nullptr;
  float* d_J = nullptr;
  float* d_bias = nullptr;
  uint32_t g_nodes = 0;
  uint32_t* d_grp = nullptr;   // ICM graph rows (petgraph node range), off-diagonal
  uint32_t* d_gcol = nullptr;
  double* d_sus = nullptr;     // [nchi][n] reference order
  // colour order
  uint32_t ncolors = 0;
  std::vector<uint32_t> color_off;   // host copy, ncolors + 1
  uint32_t* d_color_off = nullptr;
  uint32_t* d_perm = nullptr;        // new -> original
  uint32_t* d_iperm = nullptr;       // original -> new
  uint32_t* d_frp = nullptr;         // n + 1
  uint2* d_fent = nullptr;           // nnz (col_new, J bits)
  float* d_fJt = nullptr;            // lattice instances: couplings [udeg][n] (entry m of colour row s at m n + s)
  uint16_t* d_fcolt = nullptr;       // lattice instances: columns [udeg][n], same layout
  uint16_t* d_fcol16 = nullptr;      // nnz col_new as 16 bits, padded to 8 entries (n <= 65536 only)
  uint32_t udeg = 0;                 // entries per row when every row has the same count, else 0
  int pmj = 0;                       // +-1 couplings, no field, no self-loop, rows of 4 or 6 entries
  uint32_t lat_L = 0;                // periodic L^d lattice in file order (L 16 or 32, d = udeg / 2), else 0
  float* d_fbias = nullptr;          // n
  void* arena = nullptr;             // one allocation holding every array above
  size_t arena_bytes = 0;
  float* d_fkd = nullptr;            // n: self-loop coefficient (0 if none)
  double* d_fsus = nullptr;          // [nchi][n] colour order
  // host copies used by drivers
  tamc::HostInstance host;
  std::vector<uint32_t> h_perm;
  SaScratch sa_scratch;
};
void tamc_inst_retain(tamc_inst* d);
void tamc_inst_release(tamc_inst* d);
