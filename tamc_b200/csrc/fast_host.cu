// fast_host.cu -- host side of the colour-ordered PT-ICM path: the tamc_pt
// glue (one job), the batched runner (many jobs per launch, each chunk of
// rounds replayed from a captured CUDA graph) and the tile autotuner.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>
#include <tuple>

#include "fast_pt.cuh"

struct tamc_pt::FastState {
  tamc::PtJob job{};
  tamc::DBuf<uint32_t> W;
  tamc::DBuf<double> Ec, Er;
  tamc::DBuf<char> book;  // the block that betas, tags, acc, rtrips and dhist view
  tamc::DBuf<uint8_t> tags;
  tamc::DBuf<uint32_t> acc, rtrips, dhist;
  tamc::DBuf<float> betas;
  tamc::DBuf<tamc::PtJob> d_job;
  tamc::DBuf<uint32_t> ctr;
  uint32_t T = 512;
  size_t smem = 0;
  // fused runs added to a batch: the random initial replicas are drawn in the
  // batch's first chunk launch instead of a launch of their own at creation
  bool init_pending = false;
  // plain form (one instance over the whole GPU)
  bool plain = false;
  tamc::DBuf<tamc::PlainCtl> ctl;
  tamc::DBuf<long long> eacc;  // fixed-point sweep sums (2 x C x ntp)
  tamc::DBuf<long long> icm_dE;     // fixed-point ICM energy changes (C x ntp)
  tamc::DBuf<uint32_t> icm_valid;   // caches invalidated by ICM (C x ntp)
  tamc::DBuf<unsigned long long> dm;  // exchange: swapped slot pairs per chain
  size_t head_smem = 0;
  int head_stage = 0;  // the head kernel stages replica words for measurements
  uint32_t grid_cap = 0;
  std::map<uint32_t, cudaGraphExec_t> graphs;  // captured chunks of K rounds
  tamc::DBuf<unsigned long long> prof;          // per-phase cycles (TAMC_PHASE_PROF=1)
  ~FastState() {
    for (auto& kv : graphs) cudaGraphExecDestroy(kv.second);
  }
};

bool tamc_pt::fast_plain() const { return fast && fast->plain; }
bool tamc_pt::fast_deferred() const { return fast && fast->init_pending; }

namespace tamc {

// ------------------------------------------------------------ autotuner ----
// The fused kernel's free choices per job shape are the CTA size and whether
// the colour-ordered CSR is staged in shared memory.  Candidates are timed on a
// scratch copy of the job (a few rounds, CUDA events) the first time a shape
// is seen; the winner is cached per (device, n, nnz, nt, C) shape.
struct TileChoice {
  uint32_t T;
  bool csr;
};
static std::mutex g_tune_mu;
static std::map<std::tuple<int, uint32_t, uint32_t, uint32_t, uint32_t, int, int>, TileChoice> g_tune;

static bool fits(const tamc_gpu* g, const PtJob& j, uint32_t T, bool csr) {
  return fused_smem_bytes(j, T, csr) <= g->smem_optin;
}

// 512 threads with the instance in shared memory if that fits, else the
// largest CTA (512, 256, 128) whose shared memory fits without it.
static TileChoice heuristic_tile(const tamc_gpu* g, const PtJob& j) {
  if (fits(g, j, 512, true)) return TileChoice{512, true};
  for (uint32_t T : {512u, 256u, 128u})
    if (T >= j.qps && fits(g, j, T, false)) return TileChoice{T, false};
  return TileChoice{512, false};
}

// Kernel time of `rounds` rounds of the job with tile t, on scratch state: one
// launch of `rounds` rounds from random replicas (warm-up, and it moves the
// replicas off the random start, whose clusters are untypical), then two
// launches continuing from there; the faster of the two is returned.
static float time_tile(tamc_gpu* g, const PtJob& proto, TileChoice t, uint32_t rounds) {
  // scratch state so the real job is untouched
  PtJob j = proto;
  DBuf<uint32_t> W((size_t)j.n * j.nw);
  DBuf<double> Ec((size_t)j.C * j.ntp), Er((size_t)j.C * j.ntp);
  DBuf<uint8_t> tags((size_t)j.C * j.nt);
  DBuf<uint32_t> acc((size_t)j.C * j.nt), rt(j.C), dh((size_t)j.C * j.nt * 2);
  DBuf<PtJob> dj(1);
  DBuf<uint32_t> ctr(1);
  cudaStream_t st = g->stream;
  tags.zero(st);
  acc.zero(st);
  rt.zero(st);
  dh.zero(st);
  j.W = W.p;
  j.Ec = Ec.p;
  j.Er = Er.p;
  j.tags = tags.p;
  j.acc = acc.p;
  j.rtrips = rt.p;
  j.dhist = dh.p;
  j.meas_init = 0xffffffffu;  // no measurements while timing
  j.count_out = nullptr;
  j.csr_smem = t.csr;
  const size_t smem = fused_smem_bytes(j, t.T, t.csr);
  cudaEvent_t e0, e1;
  TAMC_CUDA(cudaEventCreate(&e0));
  TAMC_CUDA(cudaEventCreate(&e1));
  float best = 1e30f;
  for (uint32_t rep = 0; rep < 3; ++rep) {
    j.init = rep == 0 ? 1 : 0;
    j.sweep_begin = rep * rounds;
    j.sweep_end = (rep + 1) * rounds;
    TAMC_CUDA(tamc::copy_async(dj.p, &j, sizeof(PtJob), cudaMemcpyHostToDevice, st));
    ctr.zero(st);
    TAMC_CUDA(cudaEventRecord(e0, st));
    fused_launch(st, dj.p, 1, ctr.p, 1, t.T, smem);
    TAMC_CUDA(cudaEventRecord(e1, st));
    g->count();
    TAMC_CUDA(cudaEventSynchronize(e1));  // also keeps the host copy of j unchanged until it is read
    float ms = 0.0f;
    TAMC_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    if (rep > 0) best = std::min(best, ms);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return best;
}

// Set while a server creates runs: every request has its own shape, so the
// timing autotuner would run per request; the heuristic tile is used instead.
thread_local bool g_no_autotune = false;
// Set while a batch adds a run: its initial replicas wait for the first chunk.
thread_local bool g_defer_init = false;

static TileChoice tune_tile(tamc_gpu* g, const PtJob& j) {
  if (g_no_autotune) return heuristic_tile(g, j);
  const auto key = std::make_tuple(g->device, j.n, j.F.nnz, j.nt, j.C, (int)j.self_loops, (int)j.icm_uf);
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune.find(key);
    if (it != g_tune.end()) return it->second;
  }
  TileChoice best = heuristic_tile(g, j);
  const char* env = getenv("TAMC_AUTOTUNE");
  if (!env || env[0] != '0') {
    float best_ms = 1e30f;
    for (uint32_t T : {128u, 256u, 512u}) {
      if (T < j.qps) continue;
      for (bool csr : {true, false}) {
        if (!fits(g, j, T, csr)) continue;
        const float ms = time_tile(g, j, TileChoice{T, csr}, 16);
        if (ms < best_ms) {
          best_ms = ms;
          best = TileChoice{T, csr};
        }
      }
    }
  }
  if (getenv("TAMC_DEBUG"))
    fprintf(stderr, "[tamc] PT fused tile n=%u nt=%u C=%u: threads=%u csr_smem=%d\n", j.n, j.nt, j.C, best.T, (int)best.csr);
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune[key] = best;
  return best;
}

// ------------------------------------------------------------ one job ----
static void fill_job(tamc_pt* pt, uint64_t seed, tamc_pt::FastState* F) {
  const PtCfg& c = pt->cfg;
  const tamc_inst* I = pt->inst;
  if (c.nt > 64) fail(TAMC_E_UNSUPPORTED, "fast mode supports at most 64 temperatures per chain");
  PtJob& j = F->job;
  j.F = make_fast_inst(I);
  j.n = I->n;
  j.nt = c.nt;
  j.ntp = (c.nt + 3) & ~3u;
  j.C = c.C;
  j.wpc = (j.ntp + 31) / 32;
  j.nw = j.C * j.wpc;
  j.lo = c.lo;
  j.qpc = j.ntp / 4;
  j.qps = j.C * j.qpc;
  if (j.qps > 512) fail(TAMC_E_UNSUPPORTED, "fast mode supports at most 2048 replicas per run");
  j.icm = c.icm;
  j.threaded = c.threads > 1;
  j.self_loops = I->self_loops;
  j.key = philox_key(seed);
  // multi-spin-coded sweep for +-J instances (TAMC_MSC=0 keeps the per-quad update)
  j.msc = j.F.pmj && (j.nw == 1 || j.nw == 2 || j.nw == 4);
  if (const char* e = getenv("TAMC_MSC"))
    if (e[0] == '0') j.msc = 0;
  cudaStream_t st = pt->g->stream;
  F->W.alloc((size_t)j.n * j.nw);
  F->Ec.alloc((size_t)j.C * j.ntp);
  F->Er.alloc((size_t)j.C * j.ntp);
  F->d_job.alloc(1);
  F->ctr.alloc(1);
  // the ladder and the exchange bookkeeping in one block, set by one copy:
  // betas padded with beta = 0, round-trip tags (1 at the lowest slot, 2 at
  // the highest, per chain), zero acceptance counts, round trips and
  // diffusion histograms
  const size_t CT = (size_t)j.C * j.nt;
  auto a16 = [](size_t b) { return (b + 15) & ~(size_t)15; };
  const size_t o_acc = a16((size_t)j.ntp * 4), o_rt = o_acc + a16(CT * 4), o_dh = o_rt + a16((size_t)j.C * 4),
               o_tags = o_dh + a16(CT * 8), book_bytes = o_tags + a16(CT);
  std::vector<char> hb(book_bytes, 0);
  std::copy(c.betas.begin(), c.betas.end(), reinterpret_cast<float*>(hb.data()));
  for (uint32_t ch = 0; ch < j.C; ++ch) {
    hb[o_tags + (size_t)ch * j.nt] = 1;
    hb[o_tags + (size_t)ch * j.nt + j.nt - 1] = 2;
  }
  F->book.alloc(book_bytes);
  TAMC_CUDA(tamc::copy_async(F->book.p, hb.data(), book_bytes, cudaMemcpyHostToDevice, st));
  F->betas.view(F->book.p, j.ntp);
  F->acc.view(F->book.p + o_acc, CT);
  F->rtrips.view(F->book.p + o_rt, j.C);
  F->dhist.view(F->book.p + o_dh, CT * 2);
  F->tags.view(F->book.p + o_tags, CT);
  j.betas = F->betas.p;
  j.W = F->W.p;
  j.Ec = F->Ec.p;
  j.Er = F->Er.p;
  j.tags = F->tags.p;
  j.acc = F->acc.p;
  j.rtrips = F->rtrips.p;
  j.dhist = F->dhist.p;
  j.num_sweeps = c.num_sweeps;
  j.meas_init = c.meas_init;
  j.sample = c.sample;
  j.sample_states = c.sample_states;
  j.level = c.level;
  j.out = pt->out.meas(c);
  j.log = pt->out.log();
  j.count_out = nullptr;
  j.prof = nullptr;
  if (const char* e = getenv("TAMC_PHASE_PROF")) {
    if (e[0] == '1') {
      F->prof.alloc(PHASE_N);
      F->prof.zero(st);
      j.prof = F->prof.p;
    }
  }
  j.cost = (uint64_t)c.num_sweeps * j.n * j.C * j.ntp;
  // ICM slots labelled together: all active slots of a word if their label
  // arrays fit (aiming at <= 110 KB of shared memory so two CTAs can share an
  // SM), else fewer
  uint32_t active = 0;
  for (uint32_t w = 0; w < j.wpc; ++w) {
    uint32_t a = 0;
    for (uint32_t b = 0; b < 32; ++b) a += (32 * w + b >= j.lo && 32 * w + b < j.nt);
    active = std::max(active, a);
  }
  // cluster search: frontier BFS unless TAMC_ICM=uf asks for union-find
  // labelling (same clusters; BFS touches only the clusters)
  j.icm_uf = 0;
  if (const char* e = getenv("TAMC_ICM")) j.icm_uf = strcmp(e, "uf") == 0;
  const size_t budget = std::min<size_t>(pt->g->smem_optin, 110 * 1024);
  j.icm_group = std::max(1u, active);
  while (j.icm_group > 1 && fused_smem_bytes(j, 512, false) > budget) --j.icm_group;
}

static uint32_t count_sched(int64_t period, uint32_t meas_init, uint32_t num_sweeps, uint32_t a, uint32_t b) {
  uint32_t k = 0;
  for (uint32_t i = std::max(a, meas_init); i < b; ++i)
    k += period >= 0 && ((i - meas_init) % (uint32_t)period == 0 || i == num_sweeps - 1);
  return k;
}

static void launch_one(tamc_pt* pt, uint32_t begin, uint32_t end, int init) {
  auto* F = pt->fast;
  PtJob& j = F->job;
  cudaStream_t st = pt->g->stream;
  j.init = init;
  j.sweep_begin = begin;
  j.sweep_end = end;
  j.m_base = pt->m_next;
  j.s_base = pt->s_next;
  TAMC_CUDA(tamc::copy_async(F->d_job.p, &j, sizeof(PtJob), cudaMemcpyHostToDevice, st));
  F->ctr.zero(st);
  fused_launch(st, F->d_job.p, 1, F->ctr.p, 1, F->T, F->smem);
  pt->g->count();
  // the job struct is read by the kernel; keep the host copy alive until done
  TAMC_CUDA(cudaStreamSynchronize(st));
}

// ---- plain form: one launch per sweep phase over the whole GPU
// (the head launch of a round without measurements returns at once; leaving
// it out of the captured chunk measured slower on C4, so every round has one)
static void plain_enqueue_rounds(tamc_pt* pt, uint32_t K) {
  auto* F = pt->fast;
  const PtJob& j = F->job;
  cudaStream_t st = pt->g->stream;
  const auto& off = pt->inst->color_off;
  for (uint32_t r = 0; r < K; ++r) {
    plain_launch_head(st, F->d_job.p, F->ctl.p, F->eacc.p, 1, F->head_smem, F->head_stage);
    if (!plain_launch_icm(st, j, F->d_job.p, F->ctl.p, F->icm_dE.p, F->icm_valid.p, pt->g->smem_optin,
                          (uint32_t)pt->g->num_sms, F->dm.p))
      plain_launch_exch(st, j, F->d_job.p, F->ctl.p, F->icm_dE.p, F->icm_valid.p, F->dm.p);
    plain_launch_perm(st, j, F->d_job.p, F->dm.p, F->grid_cap);
    for (uint32_t c = 0; c + 1 < off.size(); ++c)
      plain_launch_sweep(st, j, F->d_job.p, F->ctl.p, c, (off[c + 1] - off[c]) * j.qps, F->eacc.p, F->grid_cap);
  }
  plain_launch_head(st, F->d_job.p, F->ctl.p, F->eacc.p, 1, F->head_smem, F->head_stage);  // close the last round
}

static void plain_run_chunk(tamc_pt* pt, uint32_t K) {
  TraceRange tr("tamc plain chunk");
  auto* F = pt->fast;
  cudaStream_t st = pt->g->stream;
  auto it = F->graphs.find(K);
  if (it == F->graphs.end()) {
    cudaGraph_t graph;
    TAMC_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    plain_enqueue_rounds(pt, K);
    TAMC_CUDA(cudaStreamEndCapture(st, &graph));
    cudaGraphExec_t exec;
    TAMC_CUDA(cudaGraphInstantiate(&exec, graph, 0));
    cudaGraphDestroy(graph);
    it = F->graphs.emplace(K, exec).first;
  }
  TAMC_CUDA(cudaGraphLaunch(it->second, st));
  pt->g->count((uint64_t)K * (3 + pt->inst->ncolors) + 1);
}

static void plain_setup(tamc_pt* pt) {
  auto* F = pt->fast;
  PtJob& j = F->job;
  cudaStream_t st = pt->g->stream;
  F->plain = true;
  F->head_stage = plain_head_bytes(j, true) <= pt->g->smem_optin;
  F->head_smem = plain_head_bytes(j, F->head_stage != 0);
  if (F->head_smem > pt->g->smem_optin) fail(TAMC_E_UNSUPPORTED, "instance too large for the plain PT head kernel");
  F->grid_cap = (uint32_t)pt->g->num_sms * 8;
  F->ctl.alloc(1);
  F->ctl.zero(st);
  F->eacc.alloc(2 * (size_t)j.C * j.ntp);
  F->eacc.zero(st);
  F->icm_dE.alloc((size_t)j.C * j.ntp);
  F->icm_valid.alloc((size_t)j.C * j.ntp);
  F->icm_valid.zero(st);
  F->dm.alloc(j.C);
  F->dm.zero(st);
  if (plain_icm_bytes(j) > pt->g->smem_optin) fail(TAMC_E_UNSUPPORTED, "instance too large for the plain ICM kernel");
  j.init = 0;
  j.count_out = nullptr;
  TAMC_CUDA(tamc::copy_async(F->d_job.p, &j, sizeof(PtJob), cudaMemcpyHostToDevice, st));
}

static void plain_init_energies(tamc_pt* pt, bool random) {
  auto* F = pt->fast;
  cudaStream_t st = pt->g->stream;
  F->eacc.zero(st);
  plain_launch_init(st, F->d_job.p, F->eacc.p, random ? 1 : 0, (uint32_t)pt->g->num_sms * 4);
  plain_launch_head(st, F->d_job.p, F->ctl.p, F->eacc.p, 2, F->head_smem, F->head_stage);
  pt->g->count(random ? 3 : 2);
  TAMC_CUDA(cudaStreamSynchronize(st));
}

// Which form runs a single instance: the fused kernel (one CTA, state in
// shared memory) or the plain form (all SMs, state in L2/HBM).  Both give the
// same results; the autotuner times a few rounds of each on this shape.
static std::map<std::tuple<int, uint32_t, uint32_t, uint32_t, uint32_t, int>, bool> g_form;

static bool choose_plain(tamc_pt* pt) {
  const char* f = getenv("TAMC_PT_FORM");
  if (f && !strcmp(f, "plain")) return true;
  if (f && !strcmp(f, "fused")) return false;
  if (g_no_autotune) return fused_smem_bytes(pt->fast->job, 128, false) > pt->g->smem_optin;
  const PtJob& j = pt->fast->job;
  const bool fused_fits = fused_smem_bytes(j, 128, false) <= pt->g->smem_optin;
  const bool plain_fits = plain_head_bytes(j, false) <= pt->g->smem_optin;
  if (!fused_fits || !plain_fits) return !fused_fits;
  const auto key = std::make_tuple(pt->g->device, j.n, j.F.nnz, j.nt, j.C, (int)j.icm_uf);
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_form.find(key);
    if (it != g_form.end()) return it->second;
  }
  // small runs cannot fill the GPU with the plain form
  bool plain = false;
  if ((uint64_t)j.n * j.qps >= 256ull * (uint64_t)pt->g->num_sms) {
    const TileChoice t = tune_tile(pt->g, j);
    const float ms_fused = time_tile(pt->g, j, t, 8);
    // time the plain form on a scratch copy
    tamc_pt scratch;
    scratch.inst = pt->inst;
    scratch.g = pt->g;
    scratch.cfg = pt->cfg;
    scratch.cfg.meas_init = 0xffffffffu;
    scratch.fast = new tamc_pt::FastState();
    float ms_plain = 1e30f;
    try {
      fill_job(&scratch, 1, scratch.fast);
      scratch.fast->job.meas_init = 0xffffffffu;
      plain_setup(&scratch);
      plain_init_energies(&scratch, true);
      cudaEvent_t e0, e1;
      TAMC_CUDA(cudaEventCreate(&e0));
      TAMC_CUDA(cudaEventCreate(&e1));
      plain_run_chunk(&scratch, 8);  // capture + warm up
      TAMC_CUDA(cudaEventRecord(e0, pt->g->stream));
      plain_run_chunk(&scratch, 8);
      TAMC_CUDA(cudaEventRecord(e1, pt->g->stream));
      TAMC_CUDA(cudaEventSynchronize(e1));
      TAMC_CUDA(cudaEventElapsedTime(&ms_plain, e0, e1));
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
    } catch (...) {
      delete scratch.fast;
      scratch.fast = nullptr;
      throw;
    }
    delete scratch.fast;
    scratch.fast = nullptr;
    plain = ms_plain < ms_fused;
  }
  if (getenv("TAMC_DEBUG")) fprintf(stderr, "[tamc] PT form n=%u nt=%u C=%u: %s\n", j.n, j.nt, j.C, plain ? "plain" : "fused");
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_form[key] = plain;
  return plain;
}

void fast_pt_create(tamc_pt* pt, uint64_t seed) {
  pt->fast = new tamc_pt::FastState();
  fill_job(pt, seed, pt->fast);
  if (choose_plain(pt)) {
    plain_setup(pt);
    plain_init_energies(pt, true);
    return;
  }
  const TileChoice t = tune_tile(pt->g, pt->fast->job);
  pt->fast->T = t.T;
  pt->fast->job.csr_smem = t.csr;
  pt->fast->smem = fused_smem_bytes(pt->fast->job, t.T, t.csr);
  if (pt->fast->smem > pt->g->smem_optin) fail(TAMC_E_UNSUPPORTED, "instance too large for the fused PT kernel");
  if (g_defer_init) {  // drawn by the batch's first chunk launch (same chain)
    pt->fast->init_pending = true;
    return;
  }
  launch_one(pt, 0, 0, 1);  // random initial replicas and their energies
}

// The deferred initial replicas of a batch run, when something reads or runs
// the run before the batch's first chunk.
static void ensure_init(tamc_pt* pt) {
  if (pt->fast && pt->fast->init_pending) {
    pt->fast->init_pending = false;
    launch_one(pt, pt->next_sweep, pt->next_sweep, 1);
  }
}

void fast_pt_run(tamc_pt* pt, uint32_t sweep_end) {
  ensure_init(pt);
  const PtCfg& c = pt->cfg;
  while (pt->next_sweep < sweep_end) {
    const uint32_t b = pt->next_sweep;
    const uint32_t e = std::min(sweep_end, b + pt->out.cap);
    if (pt->fast->plain) plain_run_chunk(pt, e - b);
    else launch_one(pt, b, e, 0);
    pt->out.dirty = true;
    pt->m_next += count_sched(c.sample, c.meas_init, c.num_sweeps, b, e);
    pt->s_next += count_sched(c.sample_states, c.meas_init, c.num_sweeps, b, e);
    pt->next_sweep = e;
    pt->out.drain(pt->g->stream);
  }
}

void fast_pt_get_state(tamc_pt* pt, int8_t* spins, float* energies) {
  ensure_init(pt);
  auto* F = pt->fast;
  const PtJob& j = F->job;
  cudaStream_t st = pt->g->stream;
  std::vector<uint32_t> W((size_t)j.n * j.nw);
  std::vector<double> Ec((size_t)j.C * j.ntp);
  TAMC_CUDA(tamc::copy_async(W.data(), F->W.p, W.size() * 4, cudaMemcpyDeviceToHost, st));
  TAMC_CUDA(tamc::copy_async(Ec.data(), F->Ec.p, Ec.size() * 8, cudaMemcpyDeviceToHost, st));
  TAMC_CUDA(cudaStreamSynchronize(st));
  const std::vector<uint32_t>& perm = pt->inst->h_perm;
  for (uint32_t ch = 0; ch < j.C; ++ch)
    for (uint32_t t = 0; t < j.nt; ++t) {
      if (energies) energies[(size_t)ch * j.nt + t] = (float)Ec[(size_t)ch * j.ntp + t];
      if (!spins) continue;
      int8_t* dst = spins + ((size_t)ch * j.nt + t) * j.n;
      const uint32_t o = ch * j.wpc + t / 32, b = t % 32;
      for (uint32_t s = 0; s < j.n; ++s) dst[perm[s]] = ((W[(size_t)s * j.nw + o] >> b) & 1u) ? -1 : 1;
    }
}

void fast_pt_set_state(tamc_pt* pt, const int8_t* spins) {
  auto* F = pt->fast;
  const PtJob& j = F->job;
  cudaStream_t st = pt->g->stream;
  std::vector<uint32_t> W((size_t)j.n * j.nw, 0);
  const std::vector<uint32_t>& perm = pt->inst->h_perm;
  for (uint32_t ch = 0; ch < j.C; ++ch)
    for (uint32_t t = 0; t < j.nt; ++t) {
      const int8_t* src = spins + ((size_t)ch * j.nt + t) * j.n;
      const uint32_t o = ch * j.wpc + t / 32, b = t % 32;
      for (uint32_t s = 0; s < j.n; ++s)
        if (src[perm[s]] < 0) W[(size_t)s * j.nw + o] |= 1u << b;
    }
  TAMC_CUDA(tamc::copy_async(F->W.p, W.data(), W.size() * 4, cudaMemcpyHostToDevice, st));
  F->init_pending = false;  // the set state replaces the initial replicas
  if (F->plain) plain_init_energies(pt, false);
  else launch_one(pt, pt->next_sweep, pt->next_sweep, 2);  // recompute energies
}

void fast_pt_acceptance(tamc_pt* pt, uint32_t* acc) {
  auto* F = pt->fast;
  TAMC_CUDA(tamc::copy_async(acc, F->acc.p, F->acc.n * 4, cudaMemcpyDeviceToHost, pt->g->stream));
  TAMC_CUDA(cudaStreamSynchronize(pt->g->stream));
}

void fast_pt_round_trips(tamc_pt* pt, uint8_t* tags, uint32_t* round_trips, uint32_t* dhist) {
  auto* F = pt->fast;
  cudaStream_t st = pt->g->stream;
  if (tags) TAMC_CUDA(tamc::copy_async(tags, F->tags.p, F->tags.n, cudaMemcpyDeviceToHost, st));
  if (round_trips) TAMC_CUDA(tamc::copy_async(round_trips, F->rtrips.p, F->rtrips.n * 4, cudaMemcpyDeviceToHost, st));
  if (dhist) TAMC_CUDA(tamc::copy_async(dhist, F->dhist.p, F->dhist.n * 4, cudaMemcpyDeviceToHost, st));
  TAMC_CUDA(cudaStreamSynchronize(st));
}

void fast_pt_phase_cycles(tamc_pt* pt, uint64_t* out) {
  auto* F = pt->fast;
  for (int k = 0; k < PHASE_N; ++k) out[k] = 0;
  if (!F || !F->prof.p) return;
  TAMC_CUDA(tamc::copy_async(out, F->prof.p, PHASE_N * 8, cudaMemcpyDeviceToHost, pt->g->stream));
  TAMC_CUDA(cudaStreamSynchronize(pt->g->stream));
}

void fast_pt_destroy(tamc_pt* pt) {
  delete pt->fast;
  pt->fast = nullptr;
}

}  // namespace tamc

// ================================================================ batch ====
namespace tamc {

// Runs one chunk of PT rounds for a set of fast-mode runs in a single fused
// launch (jobs ordered longest-remaining-first).  With `graph`, the
// upload -> reset -> kernel -> readback sequence is captured once per job
// count / tile and replayed for every later chunk.
// Ground-state logs of many runs read in one pass: their entry counts, then
// their entries packed into one staging buffer ([steps][energies][states] per
// run at 8-byte-aligned offsets), the counts reset.
struct LogRef {
  uint32_t* count;
  const uint32_t* steps;
  const float* E;
  const uint64_t* words;
  uint32_t nw;  // 64-bit words per logged state
  uint32_t pad;
};
__global__ void k_log_counts(const LogRef* __restrict__ r, uint32_t nj, uint32_t* __restrict__ out) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < nj) out[j] = *r[j].count;
}
__global__ void k_log_gather(const LogRef* __restrict__ r, const uint32_t* __restrict__ cnt,
                             const unsigned long long* __restrict__ off, char* __restrict__ stage) {
  const uint32_t j = blockIdx.x;
  const LogRef R = r[j];
  const uint32_t c = cnt[j];
  char* dst = stage + off[j];
  const size_t b4 = ((size_t)c * 4 + 7) & ~(size_t)7;
  for (uint32_t e = threadIdx.x; e < c; e += blockDim.x) {
    reinterpret_cast<uint32_t*>(dst)[e] = R.steps[e];
    reinterpret_cast<float*>(dst + b4)[e] = R.E[e];
  }
  uint64_t* w = reinterpret_cast<uint64_t*>(dst + 2 * b4);
  for (size_t x = threadIdx.x; x < (size_t)c * R.nw; x += blockDim.x) w[x] = R.words[x];
  if (threadIdx.x == 0) *R.count = 0;
}

struct ChunkRunner {
  DBuf<PtJob> d_jobs;
  DBuf<uint32_t> ctr;
  DBuf<uint32_t> counts;
  uint32_t cap_jobs = 0;
  // Two buffer sets, so that a batch can enqueue a chunk while the previous
  // one runs: each has its pinned job table and log counts, its captured
  // graph and its timing events, and remembers what its chunk advanced.
  struct Slot {
    PtJob* h_jobs = nullptr;
    uint32_t* h_counts = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    uint32_t key[8] = {};  // launch shape of the captured graph
    cudaEvent_t ev[2] = {nullptr, nullptr};
    bool busy = false;
    std::vector<tamc_pt*> act;
    uint32_t next = 0;  // the most rounds one run advances per chunk
    uint64_t seq = 0;   // enqueue order
  };
  Slot slots[2];
  uint64_t seq_next = 0;
  // second stream and fork/join events of the two-class launch
  cudaStream_t aux = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
  int prio_hi = 0, prio_lo = 0;
  // device time of the chunk launches (CUDA events around each one: the job
  // table upload, the fused kernels and the count readback) and their number
  double dev_ms = 0.0;
  uint64_t launches = 0;
  // pinned staging of drain_all
  char* pin = nullptr;
  size_t pin_bytes = 0;
  void pinned(size_t bytes) {
    if (bytes <= pin_bytes) return;
    if (pin) cudaFreeHost(pin);
    pin = nullptr;
    pin_bytes = 0;
    TAMC_CUDA(cudaMallocHost((void**)&pin, bytes));
    pin_bytes = bytes;
  }
  // The ground-state logs of every run that ran since its last drain, read in
  // one pass: a kernel gathers the entry counts (one copy, one
  // synchronisation), a second packs every log into one staging buffer and
  // resets the counts (one copy, one more), instead of two synchronous reads
  // per run.
  DBuf<LogRef> d_refs;
  DBuf<uint32_t> d_cnt;
  DBuf<unsigned long long> d_off;
  DBuf<char> d_stage;
  void drain_all(tamc_gpu* g, const std::vector<tamc_pt*>& jobs) {
    cudaStream_t st = g->stream;
    std::vector<tamc_pt*> d;
    for (auto* pt : jobs)
      if (pt->out.dirty) d.push_back(pt);
    if (d.empty()) return;
    const uint32_t nj = (uint32_t)d.size();
    std::vector<LogRef> refs(nj);
    for (uint32_t k = 0; k < nj; ++k) {
      const PtOutputs& o = d[k]->out;
      refs[k] = LogRef{o.gs_count.p, o.gs_steps.p, o.gs_E.p, o.gs_words.p, (o.n + 63) / 64, 0};
    }
    if (d_refs.n < nj) d_refs.alloc(nj);
    if (d_cnt.n < nj) d_cnt.alloc(nj);
    if (d_off.n < nj) d_off.alloc(nj);
    pinned((size_t)nj * 8 + nj * sizeof(LogRef));
    memcpy(pin, refs.data(), nj * sizeof(LogRef));
    TAMC_CUDA(tamc::copy_async(d_refs.p, pin, nj * sizeof(LogRef), cudaMemcpyHostToDevice, st));
    k_log_counts<<<(nj + 255) / 256, 256, 0, st>>>(d_refs.p, nj, d_cnt.p);
    TAMC_CUDA(cudaGetLastError());
    g->count();
    uint32_t* cnt_h = reinterpret_cast<uint32_t*>(pin + nj * sizeof(LogRef));
    TAMC_CUDA(tamc::copy_async(cnt_h, d_cnt.p, nj * 4, cudaMemcpyDeviceToHost, st));
    TAMC_CUDA(cudaStreamSynchronize(st));
    std::vector<uint32_t> cnt(cnt_h, cnt_h + nj);
    auto up8 = [](size_t x) { return (x + 7) & ~(size_t)7; };
    std::vector<unsigned long long> off(nj);
    size_t bytes = 0;
    for (uint32_t k = 0; k < nj; ++k) {
      if (cnt[k] > d[k]->out.cap) fail(TAMC_E_INVAL, "ground-state log overflow");
      off[k] = bytes;
      bytes += 2 * up8((size_t)cnt[k] * 4) + (size_t)cnt[k] * refs[k].nw * 8;
    }
    if (bytes) {
      if (d_stage.n < bytes) d_stage.alloc(bytes);
      pinned(std::max(bytes, (size_t)nj * 8));
      memcpy(pin, off.data(), nj * 8);
      TAMC_CUDA(tamc::copy_async(d_off.p, pin, nj * 8, cudaMemcpyHostToDevice, st));
      k_log_gather<<<nj, 128, 0, st>>>(d_refs.p, d_cnt.p, d_off.p, d_stage.p);
      TAMC_CUDA(cudaGetLastError());
      g->count();
      TAMC_CUDA(tamc::copy_async(pin, d_stage.p, bytes, cudaMemcpyDeviceToHost, st));
      TAMC_CUDA(cudaStreamSynchronize(st));
      for (uint32_t k = 0; k < nj; ++k) {
        if (!cnt[k]) continue;
        PtOutputs& out = d[k]->out;
        const size_t nw = refs[k].nw, b = out.h_steps.size();
        const char* src = pin + off[k];
        out.h_steps.resize(b + cnt[k]);
        out.h_E.resize(b + cnt[k]);
        out.h_words.resize((b + cnt[k]) * nw);
        memcpy(out.h_steps.data() + b, src, cnt[k] * 4);
        memcpy(out.h_E.data() + b, src + up8((size_t)cnt[k] * 4), cnt[k] * 4);
        memcpy(out.h_words.data() + b * nw, src + 2 * up8((size_t)cnt[k] * 4), cnt[k] * nw * 8);
      }
    }
    for (auto* pt : d) {
      pt->out.pending = 0;
      pt->out.dirty = false;
    }
  }
  ~ChunkRunner() {
    reset();
    if (pin) cudaFreeHost(pin);
    for (auto& sl : slots)
      for (auto e : sl.ev)
        if (e) cudaEventDestroy(e);
    if (fork) cudaEventDestroy(fork);
    if (join) cudaEventDestroy(join);
    if (aux) cudaStreamDestroy(aux);
  }
  void reset() {
    for (auto& sl : slots) {
      if (sl.exec) cudaGraphExecDestroy(sl.exec);
      if (sl.graph) cudaGraphDestroy(sl.graph);
      sl.exec = nullptr;
      sl.graph = nullptr;
      if (sl.h_jobs) cudaFreeHost(sl.h_jobs);
      if (sl.h_counts) cudaFreeHost(sl.h_counts);
      sl.h_jobs = nullptr;
      sl.h_counts = nullptr;
      sl.busy = false;
    }
    cap_jobs = 0;
  }
  void reserve(uint32_t n) {
    if (n <= cap_jobs) return;
    reset();
    cap_jobs = std::max(n, 16u);
    for (auto& sl : slots) {
      for (auto& e : sl.ev)
        if (!e) TAMC_CUDA(cudaEventCreate(&e));
      TAMC_CUDA(cudaMallocHost((void**)&sl.h_jobs, cap_jobs * sizeof(PtJob)));
      TAMC_CUDA(cudaMallocHost((void**)&sl.h_counts, cap_jobs * sizeof(uint32_t)));
    }
    d_jobs.alloc(cap_jobs);
    ctr.alloc(2);
    counts.alloc(cap_jobs);
  }
  // The CTA size, shared memory and grid of one persistent launch over `grp`:
  // T0 raised to 512 where a run's quads need it, halved while the largest
  // run's shared memory does not fit (TAMC_PT_CSR=0 keeps every CSR in HBM).
  struct Launch {
    uint32_t T = 0, grid = 0;
    size_t smem = 0;
    int per_sm = 0;
  };
  static Launch shape(tamc_gpu* g, std::vector<tamc_pt*>& grp, uint32_t T) {
    const char* csr_env = getenv("TAMC_PT_CSR");
    uint32_t qps_max = 0;
    for (auto* pt : grp) {
      if (T < pt->fast->job.qps) T = 512;
      qps_max = std::max(qps_max, pt->fast->job.qps);
    }
    size_t smem = 0;
    for (;;) {  // the largest run decides: smaller CTAs leave more shared memory
      smem = 0;
      for (auto* pt : grp) {
        PtJob& j = pt->fast->job;
        if (csr_env && csr_env[0] == '0') j.csr_smem = 0;
        if (fused_smem_bytes(j, T, j.csr_smem) > g->smem_optin) j.csr_smem = 0;
        smem = std::max(smem, fused_smem_bytes(j, T, j.csr_smem));
      }
      if (smem <= g->smem_optin || T / 2 < std::max(128u, qps_max)) break;
      T /= 2;
    }
    if (smem > g->smem_optin) fail(TAMC_E_UNSUPPORTED, "a run is too large for the fused PT kernel");
    Launch L;
    L.T = T;
    L.smem = smem;
    L.per_sm = fused_blocks_per_sm(T, smem);
    L.grid = std::min<uint32_t>((uint32_t)grp.size(), (uint32_t)(g->num_sms * std::max(L.per_sm, 1)));
    return L;
  }

  // Advances every run in `act` by up to `chunk` rounds.  With `balance`, a run
  // whose rounds cost less than the costliest run's gets proportionally more
  // rounds (up to 8x), so that every run does about the same work per launch
  // and small runs are not held back by large ones (the serving loop).
  // With `lazy_logs` the ground-state logs stay on the device until they could
  // overflow in the next chunk (at most one entry per round) or are read
  // (tamc_gpu_pt_gs drains them), instead of one readback per job and chunk.
  // Runs autotuned to 512 threads and runs autotuned to fewer go to two
  // persistent launches that share the GPU (two streams, forked and joined by
  // events, in one graph): the large runs' launch at the higher launch
  // priority, one CTA per SM, and the small runs' launch beside it with two or
  // more CTAs per SM, so that small runs no longer hold a whole SM each after
  // the large ones have taken theirs (TAMC_PT_SPLIT=0: one launch).
  // Enqueues one chunk into slot `sl` (which must not be busy) and returns
  // without waiting; the runs' host-side progress is advanced at once.
  // Returns false when no run has rounds left.
  bool enqueue(tamc_gpu* g, Slot& sl, std::vector<tamc_pt*> act, uint32_t chunk, bool use_graph, bool balance,
               bool by_size = false) {
    cudaStream_t st = g->stream;
    act.erase(std::remove_if(act.begin(), act.end(),
                             [](tamc_pt* p) { return p->next_sweep >= p->cfg.num_sweeps; }),
              act.end());
    if (act.empty()) return false;
    auto remaining = [](const tamc_pt* p) {
      return (uint64_t)(p->cfg.num_sweeps - p->next_sweep) * (p->fast->job.cost / std::max(1u, p->cfg.num_sweeps));
    };
    std::stable_sort(act.begin(), act.end(), [&](tamc_pt* x, tamc_pt* y) { return remaining(x) > remaining(y); });
    const char* t_env = getenv("TAMC_PT_T");
    const char* split_env = getenv("TAMC_PT_SPLIT");
    Launch A, B;
    bool split = false;
    uint32_t nb = (uint32_t)act.size();
    if (!t_env && !(split_env && split_env[0] == '0')) {
      // the small class runs at 128 threads (four CTAs per SM by registers):
      // on C3 that measured 27.6 ms per 1000 sweeps against 35.0 ms at the
      // small runs' own autotuned 256 threads (two per SM), which time one
      // run alone on an otherwise idle SM
      std::vector<tamc_pt*> big, small;
      uint32_t Ts = 128;
      // (`by_size`: runs of at most 512 sites also go to the small class
      // whatever their tile, so that a batch built with heuristic tiles, all
      // of 512 threads, still splits)
      for (auto* pt : act)
        (pt->fast->T >= 512 && !(by_size && pt->fast->job.n <= 512) ? big : small).push_back(pt);
      if (const char* e = getenv("TAMC_PT_TSMALL")) {  // the small class's CTA size, for measurements
        const int t = atoi(e);
        if (t == 128 || t == 256) Ts = (uint32_t)t;
      }
      if (!big.empty() && !small.empty()) {
        A = shape(g, big, 512);
        B = shape(g, small, Ts);
        split = B.per_sm >= 2 && B.T < A.T;
        if (split) {
          nb = (uint32_t)big.size();
          act = big;
          act.insert(act.end(), small.begin(), small.end());
        }
      }
    }
    if (!split) {
      // one CTA size per launch: the autotuned size of the costliest run
      // (TAMC_PT_T overrides it for measurements)
      uint32_t T = act[0]->fast->T;
      if (t_env) {
        const int t = atoi(t_env);
        if (t == 128 || t == 256 || t == 512) T = (uint32_t)t;
      }
      A = shape(g, act, T);
    }
    const uint32_t na = (uint32_t)act.size();
    if (na > cap_jobs) {  // growing the buffers: nothing may be in flight
      finish_all(g, false);
      reserve(na);
    }
    PtJob* const h_jobs = sl.h_jobs;
    std::vector<uint32_t> ends(na);
    double c_max = 1.0;  // the largest cost of one round among the runs
    for (auto* pt : act) c_max = std::max(c_max, (double)pt->fast->job.cost / std::max(1u, pt->cfg.num_sweeps));
    for (uint32_t x = 0; x < na; ++x) {
      tamc_pt* pt = act[x];
      PtJob j = pt->fast->job;
      j.init = pt->fast->init_pending ? 1 : 0;  // a batch run's deferred initial replicas
      j.sweep_begin = pt->next_sweep;
      uint32_t rounds = chunk;
      if (balance) {
        const double c_x = (double)pt->fast->job.cost / std::max(1u, pt->cfg.num_sweeps);
        rounds = (uint32_t)std::min<double>(8.0 * chunk, chunk * std::max(1.0, c_max / std::max(c_x, 1.0)));
      }
      ends[x] = std::min(pt->cfg.num_sweeps, pt->next_sweep + std::min(rounds, pt->out.cap));
      j.sweep_end = ends[x];
      j.m_base = pt->m_next;
      j.s_base = pt->s_next;
      j.count_out = counts.p + x;
      h_jobs[x] = j;
    }
    sl.next = balance ? 8 * chunk : chunk;
    if (split && !aux) {
      int least = 0, greatest = 0;
      TAMC_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
      prio_hi = greatest;
      prio_lo = least;
      TAMC_CUDA(cudaStreamCreateWithPriority(&aux, cudaStreamNonBlocking, least));
      TAMC_CUDA(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
      TAMC_CUDA(cudaEventCreateWithFlags(&join, cudaEventDisableTiming));
    }
    // the kernel launches of one chunk (both classes, or one launch)
    auto launch_all = [&]() {
      if (!split) {
        fused_launch(st, d_jobs.p, na, ctr.p, A.grid, A.T, A.smem);
        return;
      }
      fused_smem_limit(std::max(A.smem, B.smem));
      TAMC_CUDA(cudaEventRecord(fork, st));
      TAMC_CUDA(cudaStreamWaitEvent(aux, fork, 0));
      fused_launch_prio(st, d_jobs.p, nb, ctr.p, A.grid, A.T, A.smem, prio_hi);
      fused_launch_prio(aux, d_jobs.p + nb, na - nb, ctr.p + 1, B.grid, B.T, B.smem, prio_lo);
      TAMC_CUDA(cudaEventRecord(join, aux));
      TAMC_CUDA(cudaStreamWaitEvent(st, join, 0));
    };
    if (use_graph) {
      const uint32_t key[8] = {na, nb, A.grid, A.T, (uint32_t)A.smem, B.grid, B.T, (uint32_t)B.smem};
      if (!sl.exec || memcmp(key, sl.key, sizeof(key)) != 0) {
        if (sl.exec) cudaGraphExecDestroy(sl.exec);
        if (sl.graph) cudaGraphDestroy(sl.graph);
        sl.exec = nullptr;
        sl.graph = nullptr;
        TAMC_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        // the graph's two copies are counted at every replay below
        cudaMemcpyAsync(d_jobs.p, h_jobs, na * sizeof(PtJob), cudaMemcpyHostToDevice, st);
        cudaMemsetAsync(ctr.p, 0, 8, st);
        launch_all();
        cudaMemcpyAsync(sl.h_counts, counts.p, na * 4, cudaMemcpyDeviceToHost, st);
        TAMC_CUDA(cudaStreamEndCapture(st, &sl.graph));
        TAMC_CUDA(cudaGraphInstantiate(&sl.exec, sl.graph, 0));
        memcpy(sl.key, key, sizeof(key));
      }
      TAMC_CUDA(cudaEventRecord(sl.ev[0], st));
      TAMC_CUDA(cudaGraphLaunch(sl.exec, st));
      TAMC_CUDA(cudaEventRecord(sl.ev[1], st));
      count_copy(na * sizeof(PtJob), cudaMemcpyHostToDevice);
      count_copy(na * 4, cudaMemcpyDeviceToHost);
    } else {
      TAMC_CUDA(cudaEventRecord(sl.ev[0], st));
      TAMC_CUDA(tamc::copy_async(d_jobs.p, h_jobs, na * sizeof(PtJob), cudaMemcpyHostToDevice, st));
      TAMC_CUDA(cudaMemsetAsync(ctr.p, 0, 8, st));
      launch_all();
      TAMC_CUDA(tamc::copy_async(sl.h_counts, counts.p, na * 4, cudaMemcpyDeviceToHost, st));
      TAMC_CUDA(cudaEventRecord(sl.ev[1], st));
    }
    g->count(split ? 2 : 1);
    for (uint32_t x = 0; x < na; ++x) {
      tamc_pt* pt = act[x];
      const PtCfg& c = pt->cfg;
      pt->fast->init_pending = false;
      pt->out.dirty = true;
      pt->m_next += count_sched(c.sample, c.meas_init, c.num_sweeps, pt->next_sweep, ends[x]);
      pt->s_next += count_sched(c.sample_states, c.meas_init, c.num_sweeps, pt->next_sweep, ends[x]);
      pt->next_sweep = ends[x];
    }
    sl.act = std::move(act);
    sl.busy = true;
    sl.seq = seq_next++;
    return true;
  }

  // Waits for slot `sl`'s chunk, adds its device time and reads its log
  // counts.  `lazy`: a log is drained only when the entries it may hold after
  // the next `ahead` chunks (at most `next` rounds each, one entry per round)
  // could exceed its capacity; otherwise every non-empty log is drained.
  void finish(tamc_gpu* g, Slot& sl, bool lazy, uint32_t ahead) {
    if (!sl.busy) return;
    sl.busy = false;
    TAMC_CUDA(cudaEventSynchronize(sl.ev[1]));
    float ms = 0.0f;
    TAMC_CUDA(cudaEventElapsedTime(&ms, sl.ev[0], sl.ev[1]));
    dev_ms += ms;
    ++launches;
    for (size_t x = 0; x < sl.act.size(); ++x) {
      tamc_pt* pt = sl.act[x];
      const uint32_t cnt = sl.h_counts[x];
      const uint64_t next = std::min<uint64_t>(pt->out.cap, sl.next);
      if (cnt && (!lazy || cnt + ahead * next > pt->out.cap)) pt->out.drain(g->stream);
      else if (!cnt) pt->out.pending = 0;
    }
  }
  void finish_all(tamc_gpu* g, bool lazy) {
    Slot* a = &slots[0];
    Slot* b = &slots[1];
    if (b->busy && (!a->busy || b->seq < a->seq)) std::swap(a, b);  // the older chunk first
    finish(g, *a, lazy, 1);
    finish(g, *b, lazy, 1);
  }

  // Advances every run in `act` by up to `chunk` rounds (one chunk) and waits.
  void run(tamc_gpu* g, std::vector<tamc_pt*> act, uint32_t chunk, bool use_graph, bool balance = false,
           bool lazy_logs = false) {
    if (enqueue(g, slots[0], std::move(act), chunk, use_graph, balance)) finish(g, slots[0], lazy_logs, 1);
  }

  // Runs every run in `jobs` to its end, chunk after chunk, with the next
  // chunk enqueued before the previous one has finished (two buffer sets, so
  // no host gap between chunks); the logs are drained lazily, looking two
  // chunks ahead, and once at the end.
  void run_all(tamc_gpu* g, const std::vector<tamc_pt*>& jobs, uint32_t chunk) {
    uint32_t k = 0;
    for (;; k ^= 1) {
      TraceRange tr("tamc batch chunk");
      Slot& sl = slots[k];
      finish(g, sl, true, 2);  // the chunk that used these buffers two chunks ago
      if (!enqueue(g, sl, jobs, chunk, true, false, true)) break;
    }
    finish_all(g, true);
  }
};

void chunk_run(ChunkRunner* r, tamc_gpu* g, std::vector<tamc_pt*>& act, uint32_t chunk) {
  r->run(g, act, chunk, false, true);
}
ChunkRunner* chunk_runner_new() { return new ChunkRunner(); }
void chunk_runner_free(ChunkRunner* r) { delete r; }

}  // namespace tamc

using namespace tamc;

namespace tamc {
// Chunk runners kept per context after their batch is destroyed, with their
// buffers and captured graphs, so that the next batch of the same shape
// replays them instead of capturing anew.
static std::mutex g_pool_mu;
static std::map<tamc_gpu*, std::vector<ChunkRunner*>> g_pool;
static ChunkRunner* runner_take(tamc_gpu* g) {
  std::lock_guard<std::mutex> lk(g_pool_mu);
  auto& v = g_pool[g];
  if (v.empty()) return new ChunkRunner();
  ChunkRunner* r = v.back();
  v.pop_back();
  return r;
}
static void runner_give(tamc_gpu* g, ChunkRunner* r) {
  for (auto& sl : r->slots) sl.busy = false;
  r->dev_ms = 0.0;
  r->launches = 0;
  std::lock_guard<std::mutex> lk(g_pool_mu);
  auto& v = g_pool[g];
  if (v.size() >= 4) delete r;
  else v.push_back(r);
}
void runner_pool_release(tamc_gpu* g) {
  std::vector<ChunkRunner*> v;
  {
    std::lock_guard<std::mutex> lk(g_pool_mu);
    auto it = g_pool.find(g);
    if (it == g_pool.end()) return;
    v.swap(it->second);
    g_pool.erase(it);
  }
  for (auto* r : v) delete r;
}
}  // namespace tamc

struct tamc_batch {
  tamc_gpu* g = nullptr;
  std::vector<tamc_pt*> jobs;
  ChunkRunner* runner = nullptr;
  uint32_t chunk = 256;
  bool logs_pending = false;  // the last run's ground-state logs are still on the device
  // acceptance counts of every run, read in one pass on the first request
  // after a run (asynchronous copies into pinned memory, one synchronisation)
  bool acc_pending = true;
  std::vector<std::vector<uint32_t>> acc;
  uint32_t* acc_pin = nullptr;
  size_t acc_pin_n = 0;
  ~tamc_batch() {
    for (auto* p : jobs) tamc_gpu_pt_destroy(p);
    if (runner) runner_give(g, runner);
    if (acc_pin) cudaFreeHost(acc_pin);
  }
  void read_acceptance() {
    size_t total = 0;
    for (auto* pt : jobs) total += pt->fast->acc.n;
    if (total > acc_pin_n) {
      if (acc_pin) cudaFreeHost(acc_pin);
      acc_pin = nullptr;
      acc_pin_n = 0;
      TAMC_CUDA(cudaMallocHost((void**)&acc_pin, std::max<size_t>(total, 1) * 4));
      acc_pin_n = total;
    }
    size_t o = 0;
    for (auto* pt : jobs) {
      TAMC_CUDA(tamc::copy_async(acc_pin + o, pt->fast->acc.p, pt->fast->acc.n * 4, cudaMemcpyDeviceToHost,
                                 g->stream));
      o += pt->fast->acc.n;
    }
    TAMC_CUDA(cudaStreamSynchronize(g->stream));
    acc.resize(jobs.size());
    o = 0;
    for (size_t k = 0; k < jobs.size(); ++k) {
      acc[k].assign(acc_pin + o, acc_pin + o + jobs[k]->fast->acc.n);
      o += jobs[k]->fast->acc.n;
    }
    acc_pending = false;
  }
};

extern "C" {

int tamc_gpu_batch_create(tamc_gpu* g, tamc_batch** out) {
  TAMC_API_BEGIN
  if (!g || !out) fail(TAMC_E_INVAL, "null argument");
  auto* b = new tamc_batch();
  b->g = g;
  if (const char* e = getenv("TAMC_BATCH_CHUNK"))  // rounds per chunk launch (1..1024)
    b->chunk = std::min(1024u, std::max(1u, (uint32_t)strtoul(e, nullptr, 10)));
  b->runner = runner_take(g);
  tamc_gpu_retain(g);
  *out = b;
  TAMC_API_END
}

int tamc_gpu_batch_add(tamc_batch* b, tamc_inst* inst, const tamc_pt_params* p, uint64_t seed, uint32_t* job) {
  TAMC_API_BEGIN
  if (!b || !inst) fail(TAMC_E_INVAL, "null argument");
  tamc_pt* pt = nullptr;
  g_defer_init = true;
  const int rc = tamc_gpu_pt_create(inst, p, seed, TAMC_MODE_FAST, &pt);
  g_defer_init = false;
  if (rc != TAMC_OK) return rc;
  b->jobs.push_back(pt);
  b->acc_pending = true;
  if (job) *job = (uint32_t)(b->jobs.size() - 1);
  TAMC_API_END
}

int tamc_gpu_batch_run(tamc_batch* b) {
  TAMC_API_BEGIN
  TraceRange tr("tamc batch run");
  if (!b) fail(TAMC_E_INVAL, "null batch");
  TAMC_CUDA(cudaSetDevice(b->g->device));
  b->runner->run_all(b->g, b->jobs, b->chunk);
  b->logs_pending = true;  // drained, all runs at once, by the first log read
  b->acc_pending = true;
  TAMC_API_END
}

int tamc_gpu_batch_sync(tamc_batch* b) {
  TAMC_API_BEGIN
  if (!b) fail(TAMC_E_INVAL, "null batch");
  TAMC_CUDA(cudaStreamSynchronize(b->g->stream));
  TAMC_API_END
}

static tamc_pt* job_of(tamc_batch* b, uint32_t job) {
  if (!b || job >= b->jobs.size()) fail(TAMC_E_INVAL, "no such job");
  return b->jobs[job];
}

int tamc_gpu_batch_get_state(tamc_batch* b, uint32_t job, int8_t* spins, float* energies) {
  TAMC_API_BEGIN
  return tamc_gpu_pt_get_state(job_of(b, job), spins, energies);
  TAMC_API_END
}
int tamc_gpu_batch_set_state(tamc_batch* b, uint32_t job, const int8_t* spins) {
  TAMC_API_BEGIN
  return tamc_gpu_pt_set_state(job_of(b, job), spins);
  TAMC_API_END
}
int tamc_gpu_batch_round_trips(tamc_batch* b, uint32_t job, uint8_t* tags, uint32_t* round_trips,
                               uint32_t* diffusion_hist) {
  TAMC_API_BEGIN
  return tamc_gpu_pt_round_trips(job_of(b, job), tags, round_trips, diffusion_hist);
  TAMC_API_END
}
int tamc_gpu_batch_acceptance(tamc_batch* b, uint32_t job, uint32_t* counts) {
  TAMC_API_BEGIN
  tamc_pt* pt = job_of(b, job);
  if (!counts) fail(TAMC_E_INVAL, "null argument");
  if (!pt->fast || pt->fast->plain) return tamc_gpu_pt_acceptance(pt, counts);
  TAMC_CUDA(cudaSetDevice(b->g->device));
  if (b->acc_pending) b->read_acceptance();
  const PtCfg& c = pt->cfg;
  const std::vector<uint32_t>& a = b->acc[job];  // [C][nt]
  for (uint32_t t = 0; t < c.nt; ++t) {
    uint32_t s = 0;
    for (uint32_t ch = 0; ch < c.C; ++ch) s += a[(size_t)ch * c.nt + t];
    counts[t] = s;
  }
  TAMC_API_END
}
int tamc_gpu_batch_gs(tamc_batch* b, uint32_t job, uint32_t cap, uint32_t* count, uint32_t* steps, float* energies,
                      uint64_t* states) {
  TAMC_API_BEGIN
  tamc_pt* pt = job_of(b, job);
  if (b->logs_pending) {
    TAMC_CUDA(cudaSetDevice(b->g->device));
    b->runner->drain_all(b->g, b->jobs);
    b->logs_pending = false;
  }
  return tamc_gpu_pt_gs(pt, cap, count, steps, energies, states);
  TAMC_API_END
}
int tamc_gpu_batch_gs_all(tamc_batch* b, uint64_t cap_entries, uint64_t cap_words, uint32_t* counts,
                          uint32_t* steps, float* energies, uint64_t* states) {
  TAMC_API_BEGIN
  if (!b || !counts) fail(TAMC_E_INVAL, "null argument");
  const uint32_t nj = (uint32_t)b->jobs.size();
  uint64_t entries = 0, words = 0;
  for (uint32_t j = 0; j < nj; ++j) {
    const int rc = tamc_gpu_batch_gs(b, j, 0, &counts[j], nullptr, nullptr, nullptr);
    if (rc != TAMC_OK) return rc;
    entries += counts[j];
    words += (uint64_t)counts[j] * ((b->jobs[j]->inst->n + 63) / 64);
  }
  if (!steps && !energies && !states) return TAMC_OK;
  if (!steps || !energies || !states) fail(TAMC_E_INVAL, "steps, energies and states go together");
  if (entries > cap_entries || words > cap_words)
    fail(TAMC_E_INVAL, "output capacity below the logs' " + std::to_string(entries) + " entries / " +
                           std::to_string(words) + " state words");
  uint64_t eo = 0, wo = 0;
  for (uint32_t j = 0; j < nj; ++j) {
    uint32_t c = counts[j];
    const int rc = tamc_gpu_pt_gs(b->jobs[j], c, &c, steps + eo, energies + eo, states + wo);
    if (rc != TAMC_OK) return rc;
    eo += counts[j];
    wo += (uint64_t)counts[j] * ((b->jobs[j]->inst->n + 63) / 64);
  }
  TAMC_API_END
}
int tamc_gpu_batch_acceptance_all(tamc_batch* b, uint64_t cap, uint32_t* counts) {
  TAMC_API_BEGIN
  if (!b || !counts) fail(TAMC_E_INVAL, "null argument");
  uint64_t need = 0;
  for (tamc_pt* pt : b->jobs) need += pt->cfg.nt;
  if (need > cap) fail(TAMC_E_INVAL, "output capacity below the " + std::to_string(need) + " counts of the batch");
  uint64_t o = 0;
  for (uint32_t j = 0; j < (uint32_t)b->jobs.size(); ++j) {
    const int rc = tamc_gpu_batch_acceptance(b, j, counts + o);
    if (rc != TAMC_OK) return rc;
    o += b->jobs[j]->cfg.nt;
  }
  TAMC_API_END
}
int tamc_gpu_batch_samples_dims(tamc_batch* b, uint32_t job, uint32_t* M, uint32_t* S, uint32_t* Z, uint32_t* nchi) {
  TAMC_API_BEGIN
  return tamc_gpu_pt_samples_dims(job_of(b, job), M, S, Z, nchi);
  TAMC_API_END
}
int tamc_gpu_batch_samples(tamc_batch* b, uint32_t job, float* e, int32_t* q, float* suscept, uint8_t* samples) {
  TAMC_API_BEGIN
  return tamc_gpu_pt_samples(job_of(b, job), e, q, suscept, samples);
  TAMC_API_END
}
int tamc_gpu_batch_device_time(tamc_batch* b, double* ms, uint64_t* launches) {
  TAMC_API_BEGIN
  if (!b) fail(TAMC_E_INVAL, "null batch");
  if (ms) *ms = b->runner->dev_ms;
  if (launches) *launches = b->runner->launches;
  TAMC_API_END
}
int tamc_gpu_batch_tile(tamc_batch* b, uint32_t job, uint32_t* cta_threads, uint32_t* slots_per_task, int32_t* csr_in_smem) {
  TAMC_API_BEGIN
  tamc_pt* pt = job_of(b, job);
  if (cta_threads) *cta_threads = pt->fast->T;
  if (slots_per_task) *slots_per_task = 4;
  if (csr_in_smem) *csr_in_smem = pt->fast->job.csr_smem;
  TAMC_API_END
}
int tamc_gpu_batch_destroy(tamc_batch* b) {
  TAMC_API_BEGIN
  if (!b) return TAMC_OK;
  tamc_gpu* g = b->g;
  cudaSetDevice(g->device);
  cudaStreamSynchronize(g->stream);
  delete b;
  tamc_gpu_release(g);
  TAMC_API_END
}

}  // extern "C"
