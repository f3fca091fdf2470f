// sa_api.cu -- C ABI of simulated annealing: SaRunner::{run, run_parallel}
// (src/sa.rs:110-165) on the device, in reference-order or colour-ordered mode.
#include <chrono>
#include <cstring>

#include "fast_sa.cuh"
#include "pt.cuh"

namespace tamc {

RefInst make_ref_inst(const tamc_inst* d) {
  RefInst I;
  I.n = d->n;
  I.offset = d->offset;
  I.rp = d->d_rp;
  I.col = d->d_col;
  I.J = d->d_J;
  I.bias = d->d_bias;
  I.g_nodes = d->g_nodes;
  I.grp = d->d_grp;
  I.gcol = d->d_gcol;
  I.sus = d->d_sus;
  return I;
}

FastInst make_fast_inst(const tamc_inst* d) {
  FastInst F;
  F.n = d->n;
  F.nnz = (uint32_t)d->nnz;
  F.ncolors = d->ncolors;
  F.offset = d->offset;
  F.color_off = d->d_color_off;
  F.perm = d->d_perm;
  F.iperm = d->d_iperm;
  F.rp = d->d_frp;
  F.ent = d->d_fent;
  F.col16 = d->d_fcol16;
  F.udeg = d->udeg;
  F.pmj = d->pmj;
  F.lat_L = d->lat_L;
  F.fJt = d->d_fJt;
  F.fcolt = d->d_fcolt;
  F.bias = d->d_fbias;
  F.kd = d->d_fkd;
  F.sus = d->d_fsus;
  F.nchi = d->nchi;
  return F;
}


}  // namespace tamc

using namespace tamc;

extern "C" {

int tamc_gpu_sa_run(tamc_inst* inst, const float* betas, uint32_t nbeta, uint32_t num_replicas, uint32_t threads,
                    uint64_t seed, int mode, float* energies_out, uint8_t* packed_out, uint32_t* r_eff) {
  TAMC_API_BEGIN
  TraceRange tr("tamc sa run");
  if (!inst || (nbeta && !betas)) fail(TAMC_E_INVAL, "null argument");
  if (threads == 0) fail(TAMC_E_REFPANIC, "threads must be >= 1 (the reference divides by it)");
  if (num_replicas == 0) fail(TAMC_E_INVAL, "num_replicas must be >= 1");
  for (uint32_t k = 1; k < nbeta; ++k)
    if (!(betas[k] - betas[k - 1] >= 0.0f)) fail(TAMC_E_REFPANIC, "beta array must be non-decreasing");
  tamc_gpu* g = inst->g;
  TAMC_CUDA(cudaSetDevice(g->device));
  cudaStream_t st = g->stream;
  const uint32_t n = inst->n;
  // run_parallel when num_replicas > 1 (src/sa.rs:219-224): `threads` partitions
  // of num_replicas / threads replicas; run otherwise.
  const uint32_t parts = num_replicas > 1 ? threads : 1;
  const uint32_t per = num_replicas > 1 ? num_replicas / threads : 1;
  const uint32_t R = parts * per;
  if (r_eff) *r_eff = R;
  if (R == 0) return TAMC_OK;
  const uint32_t nbytes = (n + 7) / 8;
  if (mode == TAMC_MODE_FAST) {
    // device buffers (schedule, words, energies, packed states) are cached on
    // the instance and reused across calls; results go straight to the caller
    SaScratch& sc = inst->sa_scratch;
    const uint32_t nw = (R + 31) / 32;
    sc.ensure((size_t)nw * n, R, (size_t)R * nbytes, nbeta);
    if (nbeta) TAMC_CUDA(tamc::copy_async(sc.betas, betas, nbeta * 4, cudaMemcpyHostToDevice, st));
    TAMC_CUDA(cudaMemsetAsync(sc.words, 0, (size_t)nw * n * 4, st));
    SaFastArgs a;
    a.F = make_fast_inst(inst);
    a.betas = sc.betas;
    a.nbeta = nbeta;
    a.key = philox_key(seed);
    a.R = R;
    a.init_words = nullptr;
    a.words_out = sc.words;
    a.energies_out = sc.energies;
    const SaTile t = sa_fast_choose(g, a.F, R);
    sa_fast_launch(st, a, t);
    sa_pack_states(st, sc.words, n, R, sc.packed);
    g->count(2);
    if (energies_out) TAMC_CUDA(tamc::copy_async(energies_out, sc.energies, R * 4, cudaMemcpyDeviceToHost, st));
    if (packed_out)
      TAMC_CUDA(tamc::copy_async(packed_out, sc.packed, (size_t)R * nbytes, cudaMemcpyDeviceToHost, st));
    TAMC_CUDA(cudaStreamSynchronize(st));
    return TAMC_OK;
  }
  DBuf<float> d_betas(nbeta);
  if (nbeta) TAMC_CUDA(tamc::copy_async(d_betas.p, betas, nbeta * 4, cudaMemcpyHostToDevice, st));
  std::vector<float> e(R);
  std::vector<uint8_t> packed((size_t)R * nbytes, 0);
  if (mode == TAMC_MODE_REF) {
    // master stream, jumped once per partition (src/sa.rs:142-146); each
    // partition draws its own initial states (src/sa.rs:149-152).
    Xo master = xo_seed_from_u64(seed);
    std::vector<Xo> rv(parts);
    std::vector<int8_t> spins((size_t)R * n);
    for (uint32_t p = 0; p < parts; ++p) {
      rv[p] = master;
      xo_jump(master);
    }
    for (uint32_t p = 0; p < parts; ++p)
      for (uint32_t r = 0; r < per; ++r) {
        int8_t* s = spins.data() + ((size_t)p * per + r) * n;
        for (uint32_t i = 0; i < n; ++i) s[i] = (rv[p].next_u32() >> 31) ? 1 : -1;
      }
    DBuf<int8_t> d_spins((size_t)R * n);
    DBuf<Xo> d_rng(parts);
    DBuf<float> d_e(R);
    TAMC_CUDA(tamc::copy_async(d_spins.p, spins.data(), spins.size(), cudaMemcpyHostToDevice, st));
    TAMC_CUDA(tamc::copy_async(d_rng.p, rv.data(), parts * sizeof(Xo), cudaMemcpyHostToDevice, st));
    const RefInst I = make_ref_inst(inst);
    ref_sa(st, I, g->exp, d_spins.p, d_rng.p, parts, per, d_betas.p, nbeta);
    ref_energy_all(st, I, d_spins.p, d_e.p, R);
    g->count(2);
    TAMC_CUDA(cudaGetLastError());
    TAMC_CUDA(tamc::copy_async(spins.data(), d_spins.p, spins.size(), cudaMemcpyDeviceToHost, st));
    TAMC_CUDA(tamc::copy_async(e.data(), d_e.p, R * 4, cudaMemcpyDeviceToHost, st));
    TAMC_CUDA(cudaStreamSynchronize(st));
    for (uint32_t r = 0; r < R; ++r)
      for (uint32_t i = 0; i < n; ++i)
        if (spins[(size_t)r * n + i] <= 0) packed[(size_t)r * nbytes + i / 8] |= (uint8_t)(1u << (i % 8));
  } else {
    fail(TAMC_E_INVAL, "unknown mode");
  }
  if (energies_out) memcpy(energies_out, e.data(), R * 4);
  if (packed_out) memcpy(packed_out, packed.data(), packed.size());
  TAMC_API_END
}

int tamc_gpu_sa_run_device(tamc_inst* inst, const float* d_betas, uint32_t nbeta, uint32_t num_replicas,
                           uint64_t seed, float* d_energies, uint32_t* d_words, void* stream) {
  TAMC_API_BEGIN
  if (!inst || !d_energies || !d_words || (nbeta && !d_betas)) fail(TAMC_E_INVAL, "null argument");
  tamc_gpu* g = inst->g;
  TAMC_CUDA(cudaSetDevice(g->device));
  cudaStream_t st = stream ? (cudaStream_t)stream : g->stream;
  const uint32_t R = num_replicas;
  if (!R) return TAMC_OK;
  const uint32_t nw = (R + 31) / 32;
  TAMC_CUDA(cudaMemsetAsync(d_words, 0, (size_t)nw * inst->n * 4, st));
  SaFastArgs a;
  a.F = make_fast_inst(inst);
  a.betas = d_betas;
  a.nbeta = nbeta;
  a.key = philox_key(seed);
  a.R = R;
  a.init_words = nullptr;
  a.words_out = d_words;
  a.energies_out = d_energies;
  const SaTile t = sa_fast_choose(g, a.F, R);
  sa_fast_launch(st, a, t);
  g->count();
  TAMC_API_END
}

uint64_t tamc_gpu_sa_scratch_bytes(tamc_inst* inst, uint32_t num_replicas) {
  (void)inst;
  (void)num_replicas;
  return 0;
}

}  // extern "C"
