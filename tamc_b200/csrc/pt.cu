// pt.cu -- C ABI of the PT-ICM runner: PtIcmRunner::{run, run_parallel,
// pt_loop, parallel_pt_loop} (src/pt.rs:354-504) as device launches, with the
// reference's measurement schedule (apply_measurements, src/pt.rs:542-583) and
// result layouts (PtIcmMinResults / PtIcmThermalSamples).
#include <cmath>
#include <cstring>

#include "fast_pt.cuh"
#include "pt.cuh"

namespace tamc {

PtCfg make_cfg(const tamc_pt_params* p) {
  if (!p) fail(TAMC_E_INVAL, "null params");
  PtCfg c;
  c.num_sweeps = p->num_sweeps;
  c.warmup = p->warmup_fraction;
  if (p->num_beta == 0 || !p->betas) fail(TAMC_E_REFPANIC, "beta array must not be empty");
  c.betas.assign(p->betas, p->betas + p->num_beta);
  for (size_t k = 1; k < c.betas.size(); ++k)
    if (!(c.betas[k] - c.betas[k - 1] >= 0.0f)) fail(TAMC_E_REFPANIC, "beta array must be non-decreasing");
  c.nt = p->num_beta;
  c.C = p->num_replica_chains;
  if (c.C == 0) fail(TAMC_E_REFPANIC, "num_replica_chains must be >= 1");
  c.lo = p->lo_beta_idx;
  if (c.lo >= c.nt) fail(TAMC_E_INVAL, "lo_beta_idx must be < num_beta");
  c.icm = p->icm != 0;
  c.threads = p->threads;
  c.sample = p->sample;
  c.sample_states = p->sample_states;
  c.level = p->sample_limiting;
  // `(warmup_fraction * num_sweeps as f64) as u32` (src/pt.rs:348): saturating cast
  const double mi = c.warmup * (double)c.num_sweeps;
  c.meas_init = (mi != mi || mi <= 0.0) ? 0u : (mi >= 4294967295.0 ? 0xffffffffu : (uint32_t)mi);
  if (c.meas_init < c.num_sweeps) {
    if (c.sample == 0) fail(TAMC_E_REFPANIC, "sample must be > 0 (the reference takes `% sample`)");
    if (c.sample_states == 0) fail(TAMC_E_REFPANIC, "sample_states must be > 0");
  }
  for (uint32_t i = c.meas_init; i < c.num_sweeps; ++i) {
    c.M += c.is_meas(i);
    c.S += c.is_snap(i);
  }
  c.Z = c.level == 0 ? c.nt : (c.level == 1 ? c.nt / 2 : 1);
  return c;
}

void PtOutputs::init(const PtCfg& c, uint32_t n_, uint32_t nchi_, cudaStream_t st) {
  n = n_;
  nchi = nchi_;
  const size_t P = c.C / 2;
  e.alloc((size_t)c.nt * c.M * c.C);
  q.alloc((size_t)c.nt * c.M * P);
  sus.alloc((size_t)c.nt * nchi * c.M * P);
  samp.alloc((size_t)c.Z * c.S * c.C * ((n + 7) / 8));
  const uint32_t tracked = c.num_sweeps > c.meas_init ? c.num_sweeps - c.meas_init : 0;
  cap = std::max(1u, std::min(tracked, 1024u));
  // count, have and running minimum start at zero: one block, one memset
  gs_cells.alloc(16);
  gs_count.view(gs_cells.p, 1);
  gs_have.view(gs_cells.p + 4, 1);
  gs_min.view(gs_cells.p + 8, 1);
  gs_cells.zero(st);
  gs_steps.alloc(cap);
  gs_E.alloc(cap);
  gs_words.alloc((size_t)cap * ((n + 63) / 64));
}

MeasOut PtOutputs::meas(const PtCfg& c) const {
  MeasOut o;
  o.M = c.M;
  o.S = c.S;
  o.nchi = nchi;
  o.level = c.level;
  o.e = e.p;
  o.q = q.p;
  o.sus = sus.p;
  o.samp = samp.p;
  return o;
}

GsLog PtOutputs::log() const {
  GsLog L;
  L.cap = cap;
  L.count = gs_count.p;
  L.have = gs_have.p;
  L.minE = gs_min.p;
  L.steps = gs_steps.p;
  L.E = gs_E.p;
  L.words = gs_words.p;
  return L;
}

void PtOutputs::drain(cudaStream_t st) {
  if (!dirty) return;  // nothing has run since the last drain: the host copy is current
  uint32_t cnt = 0;
  TAMC_CUDA(tamc::copy_async(&cnt, gs_count.p, 4, cudaMemcpyDeviceToHost, st));
  TAMC_CUDA(cudaStreamSynchronize(st));
  if (cnt > cap) fail(TAMC_E_INVAL, "ground-state log overflow");
  if (cnt) {
    const size_t nw = (n + 63) / 64;
    const size_t b = h_steps.size();
    h_steps.resize(b + cnt);
    h_E.resize(b + cnt);
    h_words.resize((b + cnt) * nw);
    TAMC_CUDA(tamc::copy_async(h_steps.data() + b, gs_steps.p, cnt * 4, cudaMemcpyDeviceToHost, st));
    TAMC_CUDA(tamc::copy_async(h_E.data() + b, gs_E.p, cnt * 4, cudaMemcpyDeviceToHost, st));
    TAMC_CUDA(tamc::copy_async(h_words.data() + b * nw, gs_words.p, cnt * nw * 8, cudaMemcpyDeviceToHost, st));
    TAMC_CUDA(cudaMemsetAsync(gs_count.p, 0, 4, st));
    TAMC_CUDA(cudaStreamSynchronize(st));
  }
  pending = 0;
  dirty = false;
}

static void ref_create(tamc_pt* pt, Xo master) {
  const PtCfg& c = pt->cfg;
  tamc_inst* I = pt->inst;
  cudaStream_t st = pt->g->stream;
  const uint32_t n = I->n, R = c.C * c.nt;
  // generate_init_state (src/pt.rs:506-519): chains outer, temperatures inner,
  // n draws each from the master stream.
  std::vector<int8_t> h((size_t)R * n);
  for (uint32_t r = 0; r < R; ++r)
    for (uint32_t i = 0; i < n; ++i) h[(size_t)r * n + i] = (master.next_u32() >> 31) ? 1 : -1;
  std::vector<Xo> rv;
  if (c.threads > 1) {  // rng_vec[c][t]: clone, then jump (src/pt.rs:365-373)
    rv.resize(R);
    for (uint32_t k = 0; k < R; ++k) {
      rv[k] = master;
      xo_jump(master);
    }
  } else {
    rv.push_back(master);
  }
  pt->spins.alloc((size_t)R * n);
  pt->energy.alloc(R);
  pt->perm.alloc(R);
  pt->tags.alloc(R);
  pt->acc.alloc(R);
  pt->rtrips.alloc(c.C);
  pt->dhist.alloc((size_t)R * 2);
  pt->e_stale.alloc(R);
  pt->d_betas.alloc(c.nt);
  pt->d_dbeta.alloc(c.nt);
  pt->visited.alloc(std::max(n, I->g_nodes));
  pt->queue.alloc(std::max(n, I->g_nodes));
  pt->rows.alloc(n);
  pt->rng.alloc(rv.size());
  pt->err.alloc(1);
  std::vector<uint32_t> perm(R);
  std::vector<uint8_t> tags(R, 0);
  for (uint32_t k = 0; k < R; ++k) perm[k] = k;
  for (uint32_t ch = 0; ch < c.C; ++ch) {  // PTState::new (tamc-core/src/pt.rs:27-35)
    tags[(size_t)ch * c.nt] = 1;
    tags[(size_t)ch * c.nt + c.nt - 1] = 2;
  }
  std::vector<float> db(c.nt, 0.0f);
  for (uint32_t k = 0; k + 1 < c.nt; ++k) db[k] = c.betas[k + 1] - c.betas[k];
  TAMC_CUDA(tamc::copy_async(pt->spins.p, h.data(), h.size(), cudaMemcpyHostToDevice, st));
  TAMC_CUDA(tamc::copy_async(pt->perm.p, perm.data(), R * 4, cudaMemcpyHostToDevice, st));
  TAMC_CUDA(tamc::copy_async(pt->tags.p, tags.data(), R, cudaMemcpyHostToDevice, st));
  TAMC_CUDA(tamc::copy_async(pt->d_betas.p, c.betas.data(), c.nt * 4, cudaMemcpyHostToDevice, st));
  TAMC_CUDA(tamc::copy_async(pt->d_dbeta.p, db.data(), c.nt * 4, cudaMemcpyHostToDevice, st));
  TAMC_CUDA(tamc::copy_async(pt->rng.p, rv.data(), rv.size() * sizeof(Xo), cudaMemcpyHostToDevice, st));
  pt->acc.zero(st);
  pt->rtrips.zero(st);
  pt->dhist.zero(st);
  pt->err.zero(st);
  ref_energy_all(st, make_ref_inst(I), pt->spins.p, pt->energy.p, R);
  pt->g->count();
  TAMC_CUDA(cudaGetLastError());
}

static RefPt ref_view(tamc_pt* pt) {
  RefPt P;
  P.spins = pt->spins.p;
  P.energy = pt->energy.p;
  P.perm = pt->perm.p;
  P.tags = pt->tags.p;
  P.acc = pt->acc.p;
  P.rtrips = pt->rtrips.p;
  P.dhist = pt->dhist.p;
  P.e_stale = pt->e_stale.p;
  P.betas = pt->d_betas.p;
  P.dbeta = pt->d_dbeta.p;
  P.nt = pt->cfg.nt;
  P.C = pt->cfg.C;
  P.lo = pt->cfg.lo;
  P.visited = pt->visited.p;
  P.queue = pt->queue.p;
  P.rows = pt->rows.p;
  return P;
}

static void check_err(tamc_pt* pt) {
  if (!pt->err.p) return;
  int e = 0;
  TAMC_CUDA(tamc::copy_async(&e, pt->err.p, 4, cudaMemcpyDeviceToHost, pt->g->stream));
  TAMC_CUDA(cudaStreamSynchronize(pt->g->stream));
  if (e == TAMC_E_REFPANIC) fail(TAMC_E_REFPANIC, "ICM seed site outside the coupling graph (the reference panics)");
  if (e) fail(e, "device error");
}

static void ref_round(tamc_pt* pt, uint32_t i) {
  const PtCfg& c = pt->cfg;
  cudaStream_t st = pt->g->stream;
  const RefInst I = make_ref_inst(pt->inst);
  const RefPt P = ref_view(pt);
  const ExpTable& X = pt->g->exp;
  uint64_t k = 0;
  if (c.threads > 1) {  // parallel_pt_loop (src/pt.rs:446-450)
    if (c.icm) { ref_icm(st, I, P, X, pt->rng.p, pt->err.p); ++k; }
    ref_exchange_threaded(st, P, X, pt->rng.p);
    ref_sweep_threaded(st, I, P, X, pt->rng.p);
    k += 3;
  } else {  // pt_loop (src/pt.rs:493-497)
    if (c.icm) { ref_icm(st, I, P, X, pt->rng.p, pt->err.p); ++k; }
    ref_serial_round(st, I, P, X, pt->rng.p);
    ++k;
  }
  if (i >= c.meas_init) {
    const bool m = c.is_meas(i), s = c.is_snap(i);
    if (m || s) {
      ref_measure(st, I, P, pt->out.meas(c), pt->m_next, m, pt->s_next, s);
      ++k;
    }
    pt->m_next += m;
    pt->s_next += s;
    ref_gs_track(st, I, P, pt->out.log(), i);
    ++k;
  }
  pt->g->count(k);
  TAMC_CUDA(cudaGetLastError());
}

tamc_pt* pt_create_ref_stream(tamc_inst* inst, const tamc_pt_params* p, const Xo& master) {
  if (!inst || !p) fail(TAMC_E_INVAL, "null argument");
  TAMC_CUDA(cudaSetDevice(inst->g->device));
  auto* pt = new tamc_pt();
  tamc_inst_retain(inst);
  try {
    pt->inst = inst;
    pt->g = inst->g;
    pt->mode = TAMC_MODE_REF;
    pt->cfg = make_cfg(p);
    pt->out.init(pt->cfg, inst->n, inst->nchi, pt->g->stream);
    ref_create(pt, master);
    TAMC_CUDA(cudaStreamSynchronize(pt->g->stream));
  } catch (...) {
    delete pt;
    tamc_inst_release(inst);
    throw;
  }
  return pt;
}

}  // namespace tamc

using namespace tamc;

extern "C" {

int tamc_gpu_pt_create(tamc_inst* inst, const tamc_pt_params* p, uint64_t seed, int mode, tamc_pt** out) {
  TAMC_API_BEGIN
  if (!inst || !out) fail(TAMC_E_INVAL, "null argument");
  if (mode != TAMC_MODE_REF && mode != TAMC_MODE_FAST) fail(TAMC_E_INVAL, "unknown mode");
  TAMC_CUDA(cudaSetDevice(inst->g->device));
  auto* pt = new tamc_pt();
  tamc_inst_retain(inst);
  try {
    pt->inst = inst;
    pt->g = inst->g;
    pt->mode = mode;
    pt->cfg = make_cfg(p);
    pt->out.init(pt->cfg, inst->n, inst->nchi, pt->g->stream);
    if (mode == TAMC_MODE_REF) ref_create(pt, xo_seed_from_u64(seed));
    else fast_pt_create(pt, seed);
    // a batch run has launched nothing yet (its copies read pageable host
    // memory, which cudaMemcpyAsync stages before returning): no wait; the
    // batch's first chunk launch reports any error
    if (!pt->fast_deferred()) TAMC_CUDA(cudaStreamSynchronize(pt->g->stream));
  } catch (...) {
    if (pt->fast) fast_pt_destroy(pt);
    delete pt;
    tamc_inst_release(inst);
    throw;
  }
  *out = pt;
  TAMC_API_END
}

int tamc_gpu_pt_run(tamc_pt* pt, uint32_t sweep_end) {
  TraceRange tr("tamc pt run");
  TAMC_API_BEGIN
  if (!pt) fail(TAMC_E_INVAL, "null handle");
  TAMC_CUDA(cudaSetDevice(pt->g->device));
  const PtCfg& c = pt->cfg;
  sweep_end = std::min(sweep_end, c.num_sweeps);
  if (!pt->running) {
    pt->running = true;
    pt->t0 = std::chrono::steady_clock::now();
  }
  if (pt->mode == TAMC_MODE_REF) {
    for (uint32_t i = pt->next_sweep; i < sweep_end; ++i) {
      ref_round(pt, i);
      pt->out.dirty = true;
      pt->next_sweep = i + 1;
      if (i >= c.meas_init && ++pt->out.pending >= pt->out.cap) {
        check_err(pt);
        pt->out.drain(pt->g->stream);
      }
    }
  } else {
    fast_pt_run(pt, sweep_end);
  }
  TAMC_API_END
}

int tamc_gpu_pt_sync(tamc_pt* pt) {
  TAMC_API_BEGIN
  if (!pt) fail(TAMC_E_INVAL, "null handle");
  TAMC_CUDA(cudaSetDevice(pt->g->device));
  TAMC_CUDA(cudaStreamSynchronize(pt->g->stream));
  if (pt->mode == TAMC_MODE_REF) check_err(pt);
  pt->out.drain(pt->g->stream);
  if (pt->running) {
    pt->running = false;
    pt->timing_us += std::chrono::duration<double, std::micro>(std::chrono::steady_clock::now() - pt->t0).count();
  }
  TAMC_API_END
}

int tamc_gpu_pt_get_state(tamc_pt* pt, int8_t* spins, float* energies) {
  TAMC_API_BEGIN
  if (!pt) fail(TAMC_E_INVAL, "null handle");
  TAMC_CUDA(cudaSetDevice(pt->g->device));
  const PtCfg& c = pt->cfg;
  const uint32_t n = pt->inst->n, R = c.C * c.nt;
  if (pt->mode == TAMC_MODE_FAST) {
    fast_pt_get_state(pt, spins, energies);
    return TAMC_OK;
  }
  cudaStream_t st = pt->g->stream;
  std::vector<int8_t> h((size_t)R * n);
  std::vector<float> e(R);
  std::vector<uint32_t> perm(R);
  TAMC_CUDA(tamc::copy_async(h.data(), pt->spins.p, h.size(), cudaMemcpyDeviceToHost, st));
  TAMC_CUDA(tamc::copy_async(e.data(), pt->energy.p, R * 4, cudaMemcpyDeviceToHost, st));
  TAMC_CUDA(tamc::copy_async(perm.data(), pt->perm.p, R * 4, cudaMemcpyDeviceToHost, st));
  TAMC_CUDA(cudaStreamSynchronize(st));
  for (uint32_t k = 0; k < R; ++k) {
    if (spins) memcpy(spins + (size_t)k * n, h.data() + (size_t)perm[k] * n, n);
    if (energies) energies[k] = e[perm[k]];
  }
  TAMC_API_END
}

int tamc_gpu_pt_set_state(tamc_pt* pt, const int8_t* spins) {
  TAMC_API_BEGIN
  if (!pt || !spins) fail(TAMC_E_INVAL, "null argument");
  TAMC_CUDA(cudaSetDevice(pt->g->device));
  const PtCfg& c = pt->cfg;
  const uint32_t n = pt->inst->n, R = c.C * c.nt;
  for (size_t k = 0; k < (size_t)R * n; ++k)
    if (spins[k] != 1 && spins[k] != -1) fail(TAMC_E_INVAL, "spins must be +1 or -1");
  if (pt->mode == TAMC_MODE_FAST) {
    fast_pt_set_state(pt, spins);
    return TAMC_OK;
  }
  cudaStream_t st = pt->g->stream;
  std::vector<uint32_t> perm(R);
  TAMC_CUDA(tamc::copy_async(perm.data(), pt->perm.p, R * 4, cudaMemcpyDeviceToHost, st));
  TAMC_CUDA(cudaStreamSynchronize(st));
  std::vector<int8_t> h((size_t)R * n);
  for (uint32_t k = 0; k < R; ++k) memcpy(h.data() + (size_t)perm[k] * n, spins + (size_t)k * n, n);
  TAMC_CUDA(tamc::copy_async(pt->spins.p, h.data(), h.size(), cudaMemcpyHostToDevice, st));
  ref_energy_all(st, make_ref_inst(pt->inst), pt->spins.p, pt->energy.p, R);
  pt->g->count();
  TAMC_CUDA(cudaStreamSynchronize(st));
  TAMC_API_END
}

int tamc_gpu_pt_acceptance(tamc_pt* pt, uint32_t* counts) {
  TAMC_API_BEGIN
  if (!pt || !counts) fail(TAMC_E_INVAL, "null argument");
  TAMC_CUDA(cudaSetDevice(pt->g->device));
  const PtCfg& c = pt->cfg;
  std::vector<uint32_t> acc((size_t)c.C * c.nt);
  if (pt->mode == TAMC_MODE_FAST) {
    fast_pt_acceptance(pt, acc.data());
  } else {
    TAMC_CUDA(tamc::copy_async(acc.data(), pt->acc.p, acc.size() * 4, cudaMemcpyDeviceToHost, pt->g->stream));
    TAMC_CUDA(cudaStreamSynchronize(pt->g->stream));
  }
  for (uint32_t t = 0; t < c.nt; ++t) {
    uint32_t s = 0;
    for (uint32_t ch = 0; ch < c.C; ++ch) s += acc[(size_t)ch * c.nt + t];
    counts[t] = s;
  }
  TAMC_API_END
}

int tamc_gpu_pt_round_trips(tamc_pt* pt, uint8_t* tags, uint32_t* round_trips, uint32_t* diffusion_hist) {
  TAMC_API_BEGIN
  if (!pt) fail(TAMC_E_INVAL, "null handle");
  TAMC_CUDA(cudaSetDevice(pt->g->device));
  const PtCfg& c = pt->cfg;
  if (pt->mode == TAMC_MODE_FAST) {
    fast_pt_round_trips(pt, tags, round_trips, diffusion_hist);
    return TAMC_OK;
  }
  cudaStream_t st = pt->g->stream;
  if (tags) TAMC_CUDA(tamc::copy_async(tags, pt->tags.p, (size_t)c.C * c.nt, cudaMemcpyDeviceToHost, st));
  if (round_trips) TAMC_CUDA(tamc::copy_async(round_trips, pt->rtrips.p, c.C * 4, cudaMemcpyDeviceToHost, st));
  if (diffusion_hist)
    TAMC_CUDA(tamc::copy_async(diffusion_hist, pt->dhist.p, (size_t)c.C * c.nt * 8, cudaMemcpyDeviceToHost, st));
  TAMC_CUDA(cudaStreamSynchronize(st));
  TAMC_API_END
}

int tamc_gpu_pt_gs(tamc_pt* pt, uint32_t cap, uint32_t* count, uint32_t* steps, float* energies, uint64_t* states) {
  TAMC_API_BEGIN
  if (!pt || !count) fail(TAMC_E_INVAL, "null argument");
  TAMC_CUDA(cudaSetDevice(pt->g->device));
  pt->out.drain(pt->g->stream);
  const uint32_t cnt = (uint32_t)pt->out.h_steps.size();
  *count = cnt;
  const uint32_t k = std::min(cap, cnt);
  const size_t nw = (pt->inst->n + 63) / 64;
  if (steps) memcpy(steps, pt->out.h_steps.data(), k * 4);
  if (energies) memcpy(energies, pt->out.h_E.data(), k * 4);
  if (states) memcpy(states, pt->out.h_words.data(), k * nw * 8);
  TAMC_API_END
}

int tamc_gpu_pt_samples_dims(tamc_pt* pt, uint32_t* M, uint32_t* S, uint32_t* Z, uint32_t* nchi) {
  TAMC_API_BEGIN
  if (!pt) fail(TAMC_E_INVAL, "null handle");
  if (M) *M = pt->cfg.M;
  if (S) *S = pt->cfg.S;
  if (Z) *Z = pt->cfg.Z;
  if (nchi) *nchi = pt->inst->nchi;
  TAMC_API_END
}

int tamc_gpu_pt_samples(tamc_pt* pt, float* e, int32_t* q, float* suscept, uint8_t* samples) {
  TAMC_API_BEGIN
  if (!pt) fail(TAMC_E_INVAL, "null handle");
  TAMC_CUDA(cudaSetDevice(pt->g->device));
  cudaStream_t st = pt->g->stream;
  const PtOutputs& o = pt->out;
  if (e) TAMC_CUDA(tamc::copy_async(e, o.e.p, o.e.n * 4, cudaMemcpyDeviceToHost, st));
  if (q) TAMC_CUDA(tamc::copy_async(q, o.q.p, o.q.n * 4, cudaMemcpyDeviceToHost, st));
  if (suscept) TAMC_CUDA(tamc::copy_async(suscept, o.sus.p, o.sus.n * 4, cudaMemcpyDeviceToHost, st));
  if (samples) TAMC_CUDA(tamc::copy_async(samples, o.samp.p, o.samp.n, cudaMemcpyDeviceToHost, st));
  TAMC_CUDA(cudaStreamSynchronize(st));
  TAMC_API_END
}

int tamc_gpu_pt_phase_cycles(tamc_pt* pt, uint64_t* cycles) {
  TAMC_API_BEGIN
  if (!pt || !cycles) fail(TAMC_E_INVAL, "null argument");
  if (pt->mode != TAMC_MODE_FAST) fail(TAMC_E_INVAL, "phase accounting exists in fast mode only");
  fast_pt_phase_cycles(pt, cycles);
  TAMC_API_END
}

double tamc_gpu_pt_timing_us(tamc_pt* pt) { return pt ? pt->timing_us : 0.0; }

int tamc_gpu_pt_destroy(tamc_pt* pt) {
  TAMC_API_BEGIN
  if (!pt) return TAMC_OK;
  cudaSetDevice(pt->g->device);
  cudaStreamSynchronize(pt->g->stream);
  if (pt->fast) fast_pt_destroy(pt);
  tamc_inst* inst = pt->inst;
  delete pt;
  tamc_inst_release(inst);
  TAMC_API_END
}

}  // extern "C"
