// sa_noalloc.cu -- simulated annealing (TAMC_MODE_FAST) that allocates no
// device memory: the bit-sliced replica words it needs between the anneal
// kernel and the packing kernel live in a file-scope device array.
//
// tamc_gpu_sa_run (sa_api.cu) keeps the same words in device buffers it
// allocates on first use and caches on the instance; this entry point gives
// the same energies and packed states for callers that must not allocate
// (see the declaration in include/tamc_gpu.h).
#include <mutex>
#include <string>

#include "fast_sa.cuh"
#include "internal.h"

namespace tamc {
FastInst make_fast_inst(const tamc_inst* d);
}
using namespace tamc;

// [ceil(R/32)][n] words of one anneal, bit r%32 of word (r/32, s) = 1 when
// replica r has spin -1 at site s.  One copy per device: each device's
// context loads this module with its own instance of the array.
static __device__ __align__(256) uint32_t g_sa_words[TAMC_SA_NOALLOC_SCRATCH_BYTES / 4];

constexpr int kMaxDevices = 64;
static std::mutex g_words_mu;
static void* g_words_addr[kMaxDevices];  // device address per device, resolved on first use

// Address of g_sa_words on `device`, which must be the current device.
static uint32_t* words_on(int device) {
  if (device < 0 || device >= kMaxDevices) fail(TAMC_E_INVAL, "device index out of range");
  std::lock_guard<std::mutex> lk(g_words_mu);
  if (!g_words_addr[device]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_sa_words);
    if (e != cudaSuccess || !p)
      fail(TAMC_E_CUDA, std::string("cudaGetSymbolAddress(static annealing scratch): ") + cudaGetErrorString(e));
    g_words_addr[device] = p;
  }
  return static_cast<uint32_t*>(g_words_addr[device]);
}

extern "C" {

int tamc_gpu_sa_run_noalloc(tamc_inst* inst, const float* d_betas, uint32_t nbeta, uint32_t num_replicas,
                            uint64_t seed, float* d_energies, uint8_t* d_packed, void* stream) {
  TAMC_API_BEGIN
  if (!inst || (nbeta && !d_betas)) fail(TAMC_E_INVAL, "null argument");
  const uint32_t R = num_replicas;
  if (!R) return TAMC_OK;
  if (!d_energies || !d_packed) fail(TAMC_E_INVAL, "null argument");
  // 64-bit throughout: R + 31 must not wrap for R near 2^32
  const uint64_t need = (((uint64_t)R + 31) / 32) * (uint64_t)inst->n * 4;
  if (need > TAMC_SA_NOALLOC_SCRATCH_BYTES)
    fail(TAMC_E_INVAL, "num_replicas " + std::to_string(R) + " x n " + std::to_string(inst->n) + " needs " +
                           std::to_string(need) + " bytes of replica words, above the static scratch of " +
                           std::to_string((uint64_t)TAMC_SA_NOALLOC_SCRATCH_BYTES) + " bytes");
  tamc_gpu* g = inst->g;
  SaFastArgs a;
  a.F = make_fast_inst(inst);
  // the shared-memory check sa_fast_choose makes, before anything is queued
  const SaTile tile = sa_fast_peek(g, a.F, R);
  if (tile.smem > g->smem_optin) fail(TAMC_E_UNSUPPORTED, "instance too large for the fast SA kernel");
  TAMC_CUDA(cudaSetDevice(g->device));
  uint32_t* words = words_on(g->device);
  cudaStream_t st = stream ? (cudaStream_t)stream : g->stream;
  // the anneal kernel ORs the final spins into the words: they start at zero
  TAMC_CUDA(cudaMemsetAsync(words, 0, need, st));
  a.betas = d_betas;
  a.nbeta = nbeta;
  a.key = philox_key(seed);
  a.R = R;
  a.init_words = nullptr;
  a.words_out = words;
  a.energies_out = d_energies;
  sa_fast_launch(st, a, tile);
  sa_pack_states(st, words, inst->n, R, d_packed);
  g->count(2);
  TAMC_API_END
}

}  // extern "C"
