// fast_sa.cuh -- colour-ordered SA kernel interface.
#pragma once
#include "fast_common.cuh"

namespace tamc {

struct SaFastArgs {
  FastInst F;
  const float* betas;        // [nbeta] device
  uint32_t nbeta;
  uint2 key;                 // Philox key (seed)
  uint32_t R;                // replicas
  const uint32_t* init_words;  // [ceil(R/32)][n] original site order, or null for random
  uint32_t* words_out;       // [ceil(R/32)][n] original site order, zeroed by the caller
  float* energies_out;       // [R]
};

struct SaTile {
  uint32_t nq = 2;       // quads per CTA (replicas per CTA = 4*nq)
  uint32_t T = 512;      // threads per CTA
  bool smem_csr = true;  // instance held in shared memory
  size_t smem = 0;
};

SaTile sa_fast_choose(tamc_gpu* g, const FastInst& F, uint32_t R);
// Device-side conversion of SA words to the reference's packed byte layout.
void sa_pack_states(cudaStream_t st, const uint32_t* words, uint32_t n, uint32_t R, uint8_t* out);
void sa_fast_launch(cudaStream_t st, const SaFastArgs& a, const SaTile& t);
// The tile sa_fast_choose has cached for this shape, else the heuristic tile;
// never times candidates, so it launches and allocates nothing.
SaTile sa_fast_peek(const tamc_gpu* g, const FastInst& F, uint32_t R);

}  // namespace tamc
