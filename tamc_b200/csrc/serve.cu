// serve.cu -- continuous-batching solve server.
//
// Requests (instance + PT-ICM method) arrive at any time.  A scheduling step
// admits queued requests while the number of active requests stays under
// `max_active` and their estimated HBM footprint stays under the budget, runs
// one chunk of PT rounds for every active request in a single fused launch
// (each request's replica state stays on the device between steps), and
// retires requests that reached their sweep budget or their target energy.
// Every request runs exactly the Markov chain it would run alone: its Philox
// streams depend only on its own seed and sweep index, and its state is only
// touched by the CTA that owns it during a launch.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <deque>
#include <map>
#include <string>

#include "fast_pt.cuh"

namespace tamc {
extern thread_local bool g_no_autotune;
struct ChunkRunner;
void chunk_run(ChunkRunner* r, tamc_gpu* g, std::vector<tamc_pt*>& act, uint32_t chunk);
ChunkRunner* chunk_runner_new();
void chunk_runner_free(ChunkRunner* r);
}  // namespace tamc

using namespace tamc;
using Clock = std::chrono::steady_clock;

namespace {
struct Request {
  uint64_t id = 0;
  tamc_host_instance* h = nullptr;
  tamc_pt_params p{};
  std::vector<float> betas;
  uint64_t seed = 0;
  float target = NAN;
  uint64_t footprint = 0;
  tamc_inst* dinst = nullptr;
  tamc_pt* pt = nullptr;
  int state = 0;  // TAMC_REQ_QUEUED / _ACTIVE / _DONE / _CANCELLED / _FAILED
  std::string error;  // why admission failed
  Clock::time_point t_submit, t_done;
  float best = INFINITY;
  uint32_t sweeps = 0;
  std::vector<int8_t> final_spins;
  std::vector<float> final_energies;
};

uint64_t footprint_bytes(const HostInstance& h, const tamc_pt_params& p) {
  const uint64_t n = h.n, nnz = h.col.size(), nchi = h.suscept.size();
  const uint64_t nt = p.num_beta, ntp = (nt + 3) & ~3ull, C = p.num_replica_chains;
  const uint64_t wpc = (ntp + 31) / 32;
  uint64_t b = 0;
  b += (n + 1) * 4 * 3 + nnz * (4 + 4 + 8) + n * 4 * 6 + nchi * n * 16;  // instance (both orders)
  b += n * C * wpc * 4 + C * ntp * 16 + C * nt * 13 + ntp * 4;             // replica state
  const uint64_t M = p.sample > 0 ? p.num_sweeps / (uint64_t)p.sample + 2 : 0;
  const uint64_t S = p.sample_states > 0 ? p.num_sweeps / (uint64_t)p.sample_states + 2 : 0;
  b += nt * M * C * 4 + nt * M * (C / 2) * 4 * (1 + nchi) + nt * S * C * ((n + 7) / 8);
  b += 1024ull * (8 + ((n + 63) / 64) * 8);  // ground-state log
  return b;
}
}  // namespace

struct tamc_server {
  tamc_gpu* g = nullptr;
  uint64_t budget = 0, used = 0;
  uint32_t max_active = 0, chunk = 0;
  uint64_t next_id = 1;
  std::deque<Request*> queue;
  std::vector<Request*> active;
  std::map<uint64_t, Request*> all;
  ChunkRunner* runner = nullptr;
  ~tamc_server() {
    for (auto& kv : all) {
      Request* r = kv.second;
      if (r->pt) tamc_gpu_pt_destroy(r->pt);
      if (r->dinst) tamc_gpu_instance_destroy(r->dinst);
      if (r->h) tamc_instance_free(r->h);
      delete r;
    }
    if (runner) chunk_runner_free(runner);
  }
};

// Ends an active request: its final replicas and energies are copied out,
// its device state freed and its HBM budget returned.  `state` is
// TAMC_REQ_DONE, or TAMC_REQ_CANCELLED for a request stopped between steps.
static void retire(tamc_server* s, Request* r, int state = TAMC_REQ_DONE) {
  const uint32_t n = r->h->h.n;
  const size_t R = (size_t)r->p.num_replica_chains * r->p.num_beta;
  r->final_spins.resize(R * n);
  r->final_energies.resize(R);
  if (tamc_gpu_pt_get_state(r->pt, r->final_spins.data(), r->final_energies.data()) != TAMC_OK)
    fail(TAMC_E_CUDA, tamc_last_error());
  r->sweeps = r->pt->next_sweep;
  tamc_gpu_pt_destroy(r->pt);
  tamc_gpu_instance_destroy(r->dinst);
  r->pt = nullptr;
  r->dinst = nullptr;
  r->state = state;
  r->t_done = Clock::now();
  s->used -= r->footprint;
}

extern "C" {

int tamc_serve_create(tamc_gpu* g, uint64_t hbm_budget_bytes, uint32_t max_active, uint32_t chunk_sweeps,
                      tamc_server** out) {
  TAMC_API_BEGIN
  if (!g || !out) fail(TAMC_E_INVAL, "null argument");
  if (!max_active || !chunk_sweeps) fail(TAMC_E_INVAL, "max_active and chunk_sweeps must be > 0");
  auto* s = new tamc_server();
  s->g = g;
  tamc_gpu_retain(g);
  s->budget = hbm_budget_bytes;
  s->max_active = max_active;
  s->chunk = std::min(chunk_sweeps, 1024u);
  s->runner = chunk_runner_new();
  *out = s;
  TAMC_API_END
}

int tamc_serve_submit(tamc_server* s, const tamc_host_instance* inst, const tamc_pt_params* p, uint64_t seed,
                      float target_energy, uint64_t* request_id) {
  TAMC_API_BEGIN
  if (!s || !inst || !p || !p->betas) fail(TAMC_E_INVAL, "null argument");
  (void)make_cfg(p);  // validates like tamc_gpu_pt_create
  if (p->num_beta > 64) fail(TAMC_E_UNSUPPORTED, "fast mode supports at most 64 temperatures per chain");
  auto* r = new Request();
  r->h = new tamc_host_instance(*inst);
  r->p = *p;
  r->betas.assign(p->betas, p->betas + p->num_beta);
  r->p.betas = r->betas.data();
  r->seed = seed;
  r->target = target_energy;
  r->footprint = footprint_bytes(inst->h, *p);
  if (r->footprint > s->budget) {
    delete r->h;
    delete r;
    fail(TAMC_E_ADMISSION, "request footprint exceeds the server's HBM budget");
  }
  r->id = s->next_id++;
  r->t_submit = Clock::now();
  s->queue.push_back(r);
  s->all[r->id] = r;
  if (request_id) *request_id = r->id;
  TAMC_API_END
}

int tamc_serve_step(tamc_server* s, uint32_t* active, uint32_t* queued) {
  TAMC_API_BEGIN
  TraceRange tr("tamc serve step");
  if (!s) fail(TAMC_E_INVAL, "null server");
  TAMC_CUDA(cudaSetDevice(s->g->device));
  // admission: FIFO while slots and HBM budget allow
  // A request that cannot be set up (its instance or run is refused) fails
  // alone: it is marked TAMC_REQ_FAILED with the reason and the others go on.
  while (!s->queue.empty() && s->active.size() < s->max_active && s->used + s->queue.front()->footprint <= s->budget) {
    Request* r = s->queue.front();
    s->queue.pop_front();
    int rc = tamc_gpu_instance_upload(s->g, r->h, &r->dinst);
    if (rc == TAMC_OK) {
      g_no_autotune = true;
      rc = tamc_gpu_pt_create(r->dinst, &r->p, r->seed, TAMC_MODE_FAST, &r->pt);
      g_no_autotune = false;
    }
    if (rc == TAMC_OK && r->pt->fast && r->pt->fast_plain()) {
      rc = TAMC_E_UNSUPPORTED;
      set_error("request too large for the fused PT kernel");
    }
    if (rc != TAMC_OK) {
      r->error = tamc_last_error();
      if (r->pt) tamc_gpu_pt_destroy(r->pt);
      if (r->dinst) tamc_gpu_instance_destroy(r->dinst);
      r->pt = nullptr;
      r->dinst = nullptr;
      r->state = TAMC_REQ_FAILED;
      r->t_done = Clock::now();
      continue;
    }
    r->state = TAMC_REQ_ACTIVE;
    s->used += r->footprint;
    s->active.push_back(r);
  }
  if (!s->active.empty()) {
    std::vector<tamc_pt*> pts;
    for (auto* r : s->active) pts.push_back(r->pt);
    chunk_run(s->runner, s->g, pts, s->chunk);
    std::vector<Request*> keep;
    for (auto* r : s->active) {
      const auto& E = r->pt->out.h_E;
      if (!E.empty()) r->best = E.back();
      const bool hit = !std::isnan(r->target) && r->best <= r->target;
      if (r->pt->next_sweep >= r->pt->cfg.num_sweeps || hit) retire(s, r, TAMC_REQ_DONE);
      else keep.push_back(r);
    }
    s->active.swap(keep);
  }
  if (active) *active = (uint32_t)s->active.size();
  if (queued) *queued = (uint32_t)s->queue.size();
  TAMC_API_END
}

int tamc_serve_result(tamc_server* s, uint64_t request_id, int32_t* done, float* best_energy, uint32_t* sweeps,
                      double* latency_s) {
  TAMC_API_BEGIN
  if (!s) fail(TAMC_E_INVAL, "null server");
  auto it = s->all.find(request_id);
  if (it == s->all.end()) fail(TAMC_E_INVAL, "no such request");
  Request* r = it->second;
  const bool ended = r->state >= TAMC_REQ_DONE;
  if (done) *done = ended;
  if (best_energy) *best_energy = r->best;
  if (sweeps) *sweeps = ended ? r->sweeps : (r->pt ? r->pt->next_sweep : 0);
  if (latency_s) *latency_s = ended ? std::chrono::duration<double>(r->t_done - r->t_submit).count() : -1.0;
  TAMC_API_END
}

int tamc_serve_status(tamc_server* s, uint64_t request_id, int32_t* status, const char** error) {
  TAMC_API_BEGIN
  if (!s) fail(TAMC_E_INVAL, "null server");
  auto it = s->all.find(request_id);
  if (it == s->all.end()) fail(TAMC_E_INVAL, "no such request");
  if (status) *status = it->second->state;
  if (error) *error = it->second->error.c_str();
  TAMC_API_END
}

int tamc_serve_cancel(tamc_server* s, uint64_t request_id) {
  TAMC_API_BEGIN
  if (!s) fail(TAMC_E_INVAL, "null server");
  auto it = s->all.find(request_id);
  if (it == s->all.end()) fail(TAMC_E_INVAL, "no such request");
  Request* r = it->second;
  if (r->state == TAMC_REQ_QUEUED) {
    s->queue.erase(std::find(s->queue.begin(), s->queue.end(), r));
    r->state = TAMC_REQ_CANCELLED;
    r->t_done = Clock::now();
  } else if (r->state == TAMC_REQ_ACTIVE) {
    // steps run synchronously: between calls no launch of this request is in flight
    TAMC_CUDA(cudaSetDevice(s->g->device));
    s->active.erase(std::find(s->active.begin(), s->active.end(), r));
    retire(s, r, TAMC_REQ_CANCELLED);
  } else {
    fail(TAMC_E_INVAL, "request already ended");
  }
  TAMC_API_END
}

int tamc_serve_state(tamc_server* s, uint64_t request_id, int8_t* spins, float* energies) {
  TAMC_API_BEGIN
  if (!s) fail(TAMC_E_INVAL, "null server");
  auto it = s->all.find(request_id);
  if (it == s->all.end()) fail(TAMC_E_INVAL, "no such request");
  Request* r = it->second;
  if (r->state != TAMC_REQ_DONE && r->state != TAMC_REQ_CANCELLED) fail(TAMC_E_INVAL, "request not retired yet");
  if (r->final_spins.empty()) fail(TAMC_E_INVAL, "request ended before it ran (cancelled in the queue or failed)");
  if (spins) memcpy(spins, r->final_spins.data(), r->final_spins.size());
  if (energies) memcpy(energies, r->final_energies.data(), r->final_energies.size() * 4);
  TAMC_API_END
}

int tamc_serve_destroy(tamc_server* s) {
  TAMC_API_BEGIN
  if (!s) return TAMC_OK;
  tamc_gpu* g = s->g;
  cudaSetDevice(g->device);
  cudaStreamSynchronize(g->stream);
  delete s;
  tamc_gpu_release(g);
  TAMC_API_END
}

}  // extern "C"
