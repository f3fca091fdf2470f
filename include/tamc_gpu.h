/* tamc_gpu.h -- C ABI of the B200 (sm_100a) Monte-Carlo backend for tamc's
 * parallel-tempering + Houdayer-ICM (PT-ICM) and simulated-annealing (SA)
 * runners.
 *
 * Every function returns an int status (TAMC_OK = 0, negative on error) unless
 * stated otherwise; tamc_last_error() returns a thread-local message for the
 * last failure.  No C++ exception crosses this boundary.  The caller owns all
 * host buffers passed in or out (inputs are copied, outputs are written);
 * handles own their device memory and are released by their *_destroy call.
 * A handle is bound to one CUDA stream and is not re-entrant; distinct handles
 * may be used from different threads.
 *
 * Citations name the reference interface each entry point replaces
 * (path:line within USCqserver/tamc).
 */
#ifndef TAMC_GPU_H
#define TAMC_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TAMC_OK 0
#define TAMC_E_INVAL (-1)       /* bad argument / parameter combination      */
#define TAMC_E_NOMEM (-2)       /* host or device allocation failed          */
#define TAMC_E_CUDA (-3)        /* CUDA runtime error                        */
#define TAMC_E_TIMEOUT (-4)     /* a bounded device wait expired             */
#define TAMC_E_PARSE (-5)       /* instance / method / vector file syntax    */
#define TAMC_E_IO (-6)          /* file could not be opened / written        */
#define TAMC_E_UNSUPPORTED (-7) /* shape outside what a mode supports        */
#define TAMC_E_REFPANIC (-8)    /* input on which the reference aborts       */
#define TAMC_E_ADMISSION (-9)   /* server: request does not fit the budget   */

/* Run modes.
 * TAMC_MODE_REF  : reference-order replay.  Sequential site order per replica,
 *                  Xoshiro256++ streams seeded and jumped as the reference does
 *                  (src/pt.rs:354-373, src/sa.rs:136-146), glibc-identical
 *                  expf.  Spin states, ICM choices and exchange decisions are
 *                  bit-exact with the reference for a given seed.  `threads`
 *                  selects run (<=1, one stream) or run_parallel (>1).
 * TAMC_MODE_FAST : colour-ordered parallel update with per-replica Philox-4x32-10
 *                  streams; statistically equivalent, not bit-exact.        */
#define TAMC_MODE_REF 0
#define TAMC_MODE_FAST 1

const char* tamc_last_error(void);
const char* tamc_version(void);
/* The glibc-identical expf used by TAMC_MODE_REF (host evaluation of the same
 * code the device runs; f32::exp in tamc-core/src/metropolis.rs:50). */
float tamc_ref_expf(float x);

/* ------------------------------------------------------------------------
 * Host-side instance (no GPU needed).
 * Mirrors BqmIsingInstance::from_instance_file (src/ising.rs:286-324) over
 * read_adjacency_list (src/util.rs:76-109): `i j K` lines, fixed-point K only
 * (no exponent, no '+'; trailing text ignored), symmetrised, later duplicates
 * overwrite, rows sorted by j; --qubo conversion including the diagonal
 * self-coupling the reference stores (src/ising.rs:308-310).
 * ---------------------------------------------------------------------- */
typedef struct tamc_host_instance tamc_host_instance;

int tamc_instance_parse(const char* text, uint64_t len, int qubo, tamc_host_instance** out);
int tamc_instance_read(const char* path, int qubo, tamc_host_instance** out);
/* Same CSR as coupling_vecs: row_ptr[n+1], col/J[nnz] (self-loops kept), bias[n]. */
int tamc_instance_from_csr(uint32_t n, const uint32_t* row_ptr, const uint32_t* col, const float* J,
                           const float* bias, float offset, tamc_host_instance** out);
/* BqmIsingInstance::with_suscept (src/ising.rs:388-403) / read_txt_vec (src/util.rs:112-139).
 * A length mismatch is rejected with TAMC_E_INVAL (the reference warns, then panics later). */
int tamc_instance_add_suscept_file(tamc_host_instance* inst, const char* path);
int tamc_instance_add_suscept(tamc_host_instance* inst, const double* w, uint32_t n);
int tamc_instance_dims(const tamc_host_instance* inst, uint32_t* n, uint64_t* nnz, float* offset,
                       uint32_t* nchi);
int tamc_instance_csr(const tamc_host_instance* inst, uint32_t* row_ptr, uint32_t* col, float* J,
                      float* bias);
/* Number of nodes of the ICM graph (petgraph Csr::from_sorted_edges, src/pt.rs:344-346):
 * largest endpoint of an off-diagonal coupling + 1 (may be < n). */
uint32_t tamc_instance_graph_nodes(const tamc_host_instance* inst);
/* Graph colouring used by TAMC_MODE_FAST: ncolors and colour of each site. */
int tamc_instance_coloring(const tamc_host_instance* inst, uint32_t* ncolors, uint32_t* color);
/* energy_ref (src/ising.rs:438-454), f32 in the reference's summation order. */
float tamc_instance_energy_ref(const tamc_host_instance* inst, const int8_t* spins);
void tamc_instance_free(tamc_host_instance* inst);

/* ------------------------------------------------------------------------
 * Method files (YAML, `PT:` / `SA:` / `GLA:` externally tagged; src/lib.rs:80-113).
 * ---------------------------------------------------------------------- */
#define TAMC_METHOD_PT 1
#define TAMC_METHOD_SA 2
#define TAMC_METHOD_GLA 3

/* PtIcmParams (src/pt.rs:259-272) with the beta ladder resolved to f32
 * (BetaOptions::get_beta_arr, src/pt.rs:246-256) and lo_beta_idx resolved
 * (src/pt.rs:316-341).  Optional fields use -1 for None. */
typedef struct {
  uint32_t num_sweeps;
  double warmup_fraction;
  uint32_t num_beta;
  const float* betas;          /* num_beta entries, non-decreasing */
  uint32_t lo_beta_idx;
  int32_t icm;
  uint32_t num_replica_chains;
  uint32_t threads;            /* <=1: serial exchange semantics; >1: threaded */
  int64_t sample;              /* measurement period, -1 = None */
  int64_t sample_states;       /* state-sample period, -1 = None */
  uint32_t sample_limiting;    /* compression level 0 / 1 / >=2 */
} tamc_pt_params;

typedef struct tamc_method tamc_method;
int tamc_method_parse(const char* yaml, uint64_t len, tamc_method** out);
int tamc_method_read(const char* path, tamc_method** out);
int tamc_method_kind(const tamc_method* m);
/* PT: fills *p; p->betas points into the method object (valid until free).
 * Also reports whether lo_beta / lo_num_beta were given. */
int tamc_method_pt(const tamc_method* m, tamc_pt_params* p);
/* SA (SaParams, src/sa.rs:21-26): beta array (points into m), replicas, threads. */
int tamc_method_sa(const tamc_method* m, const float** betas, uint32_t* nbeta, uint32_t* num_replicas,
                   uint32_t* threads);
/* GLA (GlaParams, src/gla.rs:28-33): num_threads, the partition file path
 * (points into m), and the sub-solver's PtIcmParams (`pt_params`) as
 * tamc_method_pt reports them; any output pointer may be NULL. */
int tamc_method_gla(const tamc_method* m, uint32_t* num_threads, const char** partition_file, tamc_pt_params* p);
void tamc_method_free(tamc_method* m);
/* geometric_beta_schedule (tamc-core/src/sa.rs:13-22) cast to f32. */
int tamc_geometric_betas(float beta_min, float beta_max, uint32_t n, float* out);

/* ------------------------------------------------------------------------
 * Device context and device-resident instances.
 * ---------------------------------------------------------------------- */
typedef struct tamc_gpu tamc_gpu;
typedef struct tamc_inst tamc_inst;

int tamc_gpu_open(int device, tamc_gpu** out);
int tamc_gpu_close(tamc_gpu* g);
int tamc_gpu_sync(tamc_gpu* g);
/* The CUDA stream (cudaStream_t) the context launches on. */
void* tamc_gpu_stream(tamc_gpu* g);
/* Number of kernels this context launched so far (for accounting). */
uint64_t tamc_gpu_launch_count(tamc_gpu* g);
/* Bytes the library has copied host->device and device->host since it was
 * loaded, over all contexts (for end-to-end accounting). */
void tamc_copy_bytes(uint64_t* h2d, uint64_t* d2h);

/* Uploads the instance: reference-order CSR, ICM graph, colour-sorted CSR for
 * the fast mode and the susceptibility weights.  An instance with no sites is
 * refused with TAMC_E_INVAL. */
int tamc_gpu_instance_upload(tamc_gpu* g, const tamc_host_instance* h, tamc_inst** out);
/* Uploads `count` instances at once, as `count` calls of
 * tamc_gpu_instance_upload would (outs[k] for his[k]), with the host-side
 * preparation (colouring, re-layouts) spread over up to 16 threads and the
 * copies staged through a pinned block of the context in rounds of at most
 * 256 MiB (TAMC_UPLOAD_STAGE_BYTES; an instance larger than that goes alone).  For
 * callers that upload many instances together, such as the instances of one
 * batch or GLA's sub-instances, which the reference builds all before it runs
 * them (src/gla.rs:137-153).  All or nothing: on an error no instance is
 * returned; a null or empty instance is refused with TAMC_E_INVAL naming its
 * index. */
int tamc_gpu_instance_upload_many(tamc_gpu* g, uint32_t count, const tamc_host_instance* const* his,
                                  tamc_inst** outs);
int tamc_gpu_instance_destroy(tamc_inst* d);

/* ------------------------------------------------------------------------
 * PT-ICM, plain form: one instance, one launch per sweep phase.
 * Replaces PtIcmRunner::{run, run_parallel, pt_loop, parallel_pt_loop}
 * (src/pt.rs:354-504) below run_parallel_tempering (src/pt.rs:609-655).
 * ---------------------------------------------------------------------- */
typedef struct tamc_pt tamc_pt;

int tamc_gpu_pt_create(tamc_inst* inst, const tamc_pt_params* p, uint64_t seed, int mode, tamc_pt** out);
/* Advances to sweep index `sweep_end` (exclusive), asynchronously. */
int tamc_gpu_pt_run(tamc_pt* pt, uint32_t sweep_end);
int tamc_gpu_pt_sync(tamc_pt* pt);
/* Slot-ordered states [chain][temperature][n] (int8 +-1) and cached f32 energies [chain][temperature]. */
int tamc_gpu_pt_get_state(tamc_pt* pt, int8_t* spins, float* energies);
/* Replaces all states (e.g. to resume, PtIcmRunner::run(Some(states)), src/pt.rs:397-407). */
int tamc_gpu_pt_set_state(tamc_pt* pt, const int8_t* spins);
/* acceptance_counts (count_acc, src/pt.rs:585-591): [num_beta], summed over chains. */
int tamc_gpu_pt_acceptance(tamc_pt* pt, uint32_t* counts);
/* Round-trip bookkeeping (tamc-core/src/pt.rs:54-84), per chain:
 * tags [C][nt] (0 none,1 min,2 max,3 min-reflected,4 max-reflected),
 * round_trips [C], diffusion_hist [C][nt][2]. */
int tamc_gpu_pt_round_trips(tamc_pt* pt, uint8_t* tags, uint32_t* round_trips, uint32_t* diffusion_hist);
/* Ground-state trajectory (MinResults gs_*; src/pt.rs:576-581).  Returns the
 * entry count in *count; copies at most `cap` entries (states as u64 words,
 * ceil(n/64) per entry, as IsingState::as_u64_vec). */
int tamc_gpu_pt_gs(tamc_pt* pt, uint32_t cap, uint32_t* count, uint32_t* steps, float* energies,
                   uint64_t* states);
/* PtIcmThermalSamples (src/pt.rs:117-125) sizes: measurements M, state
 * snapshots S, sample slots Z (nt / nt/2 / 1 by compression level). */
int tamc_gpu_pt_samples_dims(tamc_pt* pt, uint32_t* M, uint32_t* S, uint32_t* Z, uint32_t* nchi);
/* e [nt][M*C], q [nt][M*C/2], suscept [nt][nchi][M*C/2], samples [Z][S*C][ceil(n/8)];
 * any pointer may be NULL to skip it. */
int tamc_gpu_pt_samples(tamc_pt* pt, float* e, int32_t* q, float* suscept, uint8_t* samples);
/* Fast mode with TAMC_PHASE_PROF=1 in the environment at creation: SM cycles
 * spent per round phase (ICM: seed scan, union-find label init, pointer
 * jumping, cluster growth (BFS levels or union-find hooking), cluster marking,
 * energy change and flip; exchange, sweep, measurement, other), summed over
 * rounds, then four parts of the multi-spin-coded sweep of +-J instances summed
 * over the CTA's warps (loads and bond levels, flip decisions, energy sums and
 * stores, barrier waits); zeros otherwise.  cycles[14]. */
int tamc_gpu_pt_phase_cycles(tamc_pt* pt, uint64_t* cycles);
/* Wall time of the sweep loop in microseconds (the reference's `timing`). */
double tamc_gpu_pt_timing_us(tamc_pt* pt);
int tamc_gpu_pt_destroy(tamc_pt* pt);

/* ------------------------------------------------------------------------
 * Simulated annealing.  Replaces SaRunner::{run, run_parallel, sa_loop}
 * (src/sa.rs:110-199).  Host buffers; returns the replica count actually
 * simulated (threads * (num_replicas / threads), src/sa.rs:147,161) in *r_eff.
 * energies_out[r_eff] = energy_ref per replica; packed_out[r_eff][ceil(n/8)]
 * bit-packed states (IsingState::write_to_bytes, src/ising.rs:102-115).
 * ---------------------------------------------------------------------- */
int tamc_gpu_sa_run(tamc_inst* inst, const float* betas, uint32_t nbeta, uint32_t num_replicas,
                    uint32_t threads, uint64_t seed, int mode, float* energies_out, uint8_t* packed_out,
                    uint32_t* r_eff);
/* Device-resident variant (TAMC_MODE_FAST): d_betas, d_energies (float[R]) and
 * d_words are device pointers; the state layout is [R/32 words][n] u32 with bit
 * r%32 = 1 for spin -1.  Launches on `stream` (NULL = the context stream). */
int tamc_gpu_sa_run_device(tamc_inst* inst, const float* d_betas, uint32_t nbeta, uint32_t num_replicas,
                           uint64_t seed, float* d_energies, uint32_t* d_words, void* stream);
/* Bytes of device scratch tamc_gpu_sa_run_device needs beyond its arguments. */
uint64_t tamc_gpu_sa_scratch_bytes(tamc_inst* inst, uint32_t num_replicas);

/* Largest replica-word scratch tamc_gpu_sa_run_noalloc accepts:
 * ceil(num_replicas / 32) * n * 4 bytes must not exceed it (4 MiB: e.g. 1024
 * replicas of up to 32768 spins). */
#define TAMC_SA_NOALLOC_SCRATCH_BYTES (4u << 20)
/* Simulated annealing in TAMC_MODE_FAST that allocates no device memory.
 * No reference counterpart: it returns what tamc_gpu_sa_run (TAMC_MODE_FAST)
 * returns -- energies_out as d_energies (float[num_replicas]) and packed_out as
 * d_packed ([num_replicas][ceil(n/8)] bytes, the AnnealState layout) -- but
 * into caller-owned device buffers, with d_betas (float[nbeta]) on the device.
 *
 * For callers that cannot allocate device memory mid-run: a serving loop
 * that admits work against a fixed HBM budget (an allocation outside the
 * budget defeats the admission), and host code on a latency path that must
 * not meet the device-wide synchronisation cudaMalloc/cudaFree can cause.
 * tamc_gpu_sa_run allocates its replica words on first use; this entry point
 * uses a file-scope device array of TAMC_SA_NOALLOC_SCRATCH_BYTES instead and
 * fails with TAMC_E_INVAL for larger num_replicas x n.
 *
 * First call on a device: resolves the array's address on that device
 * (cudaGetSymbolAddress, with the context's device made current); make one
 * call per device before any stream capture begins.  Each call clears the
 * words it uses (cudaMemsetAsync on `stream`) before the anneal, so nothing
 * has to be zero beforehand.  All calls on one device share the one array:
 * calls whose work overlaps on the device (different streams, or threads
 * that do not wait for each other) race on it; order them on one stream or
 * synchronise between them.  Launches on `stream` (NULL = the context
 * stream) and returns without waiting. */
int tamc_gpu_sa_run_noalloc(tamc_inst* inst, const float* d_betas, uint32_t nbeta, uint32_t num_replicas,
                            uint64_t seed, float* d_energies, uint8_t* d_packed, void* stream);

/* ------------------------------------------------------------------------
 * Batched PT-ICM (TAMC_MODE_FAST): many instances of uneven N, ladder length
 * and chain count in one persistent kernel that pulls instance tiles from a
 * device work queue; chunks of whole PT rounds are captured in CUDA graphs.
 * GLA (src/gla.rs:364-374) and tamc-pt-opt (src/bin/tamc-pt-opt.rs:242-243)
 * call PtIcmRunner per sub-instance in exactly this shape.
 * ---------------------------------------------------------------------- */
typedef struct tamc_batch tamc_batch;

int tamc_gpu_batch_create(tamc_gpu* g, tamc_batch** out);
/* Adds a job; *job receives its index.  The instance must outlive the batch. */
int tamc_gpu_batch_add(tamc_batch* b, tamc_inst* inst, const tamc_pt_params* p, uint64_t seed, uint32_t* job);
/* Runs every job to its num_sweeps. */
int tamc_gpu_batch_run(tamc_batch* b);
int tamc_gpu_batch_sync(tamc_batch* b);
/* Per-job results, same layouts as the tamc_gpu_pt_* getters. */
int tamc_gpu_batch_get_state(tamc_batch* b, uint32_t job, int8_t* spins, float* energies);
int tamc_gpu_batch_acceptance(tamc_batch* b, uint32_t job, uint32_t* counts);
/* Replaces a job's replicas before its run (PtIcmRunner::run(Some(states)), src/pt.rs:397-407). */
int tamc_gpu_batch_set_state(tamc_batch* b, uint32_t job, const int8_t* spins);
int tamc_gpu_batch_round_trips(tamc_batch* b, uint32_t job, uint8_t* tags, uint32_t* round_trips,
                               uint32_t* diffusion_hist);
int tamc_gpu_batch_gs(tamc_batch* b, uint32_t job, uint32_t cap, uint32_t* count, uint32_t* steps,
                      float* energies, uint64_t* states);
/* Every job's ground-state log in one call: counts[njobs] = entries per job
 * (always written); with steps/energies/states given, the logs job after job
 * (entries in job order, each job's states as ceil(n/64) words per entry),
 * which must fit cap_entries / cap_words.  Same values as tamc_gpu_batch_gs
 * per job; for callers that read a whole batch (no reference counterpart:
 * the reference returns each run's PtIcmMinResults, src/pt.rs:97-103,
 * 397-412). */
int tamc_gpu_batch_gs_all(tamc_batch* b, uint64_t cap_entries, uint64_t cap_words, uint32_t* counts,
                          uint32_t* steps, float* energies, uint64_t* states);
/* Every job's acceptance counts, job after job (nt per job), within cap. */
int tamc_gpu_batch_acceptance_all(tamc_batch* b, uint64_t cap, uint32_t* counts);
int tamc_gpu_batch_samples_dims(tamc_batch* b, uint32_t job, uint32_t* M, uint32_t* S, uint32_t* Z,
                                uint32_t* nchi);
int tamc_gpu_batch_samples(tamc_batch* b, uint32_t job, float* e, int32_t* q, float* suscept,
                           uint8_t* samples);
/* Device time of the batch's kernel launches so far: the sum of CUDA-event
 * times around each chunk launch (job-table upload, the persistent kernel,
 * count readback), and the number of such launches. */
int tamc_gpu_batch_device_time(tamc_batch* b, double* ms, uint64_t* launches);
/* Autotuner choice for a job: threads per CTA, slots per task, smem residency. */
int tamc_gpu_batch_tile(tamc_batch* b, uint32_t job, uint32_t* cta_threads, uint32_t* slots_per_task,
                        int32_t* csr_in_smem);
int tamc_gpu_batch_destroy(tamc_batch* b);

/* ------------------------------------------------------------------------
 * GLA partitioned solve.  Replaces run_gla (src/gla.rs:121-195): the instance
 * is split into the sub-instances induced by a partition of its sites
 * (induced_subgraph_instance_sorted, src/ising.rs:327-355), each is solved by
 * PT-ICM with PtIcmRunner::pt_loop semantics (single stream, serial
 * exchange, whatever pt_params.threads says), and the last ground state of
 * every sub-run is joined with the couplings that cross partitions.
 * TAMC_MODE_FAST runs all sub-instances as one batch; TAMC_MODE_REF runs one
 * reference-order replay per sub-instance on the Xoshiro256++ stream
 * seed_from_u64(seed) cloned and jumped once per sub-instance (the
 * reference draws that master stream's seed from OS entropy). */
typedef struct tamc_partition tamc_partition;
typedef struct tamc_gla tamc_gla;

/* GlaParams::read_graph_partition (src/gla.rs:37-58) over read_u32_lines
 * (src/util.rs:142-172): one partition per line of whitespace-separated site
 * indices (lines without a leading index are skipped, text after the last
 * index is ignored); an index >= n or listed twice is TAMC_E_INVAL. */
int tamc_partition_parse(const char* text, uint64_t len, uint32_t n, tamc_partition** out);
int tamc_partition_read(const char* path, uint32_t n, tamc_partition** out);
int tamc_partition_dims(const tamc_partition* p, uint32_t* num_parts, uint64_t* num_sites);
/* part_ptr[num_parts + 1] offsets into sites[num_sites], partitions in file order. */
int tamc_partition_get(const tamc_partition* p, uint32_t* part_ptr, uint32_t* sites);
void tamc_partition_free(tamc_partition* p);

/* Runs the solve.  Inputs on which the reference panics (a site in no
 * partition, a last site without couplings, a sub-run without a recorded
 * ground state) return TAMC_E_REFPANIC. */
int tamc_gla_run(tamc_gpu* g, const tamc_host_instance* inst, const tamc_partition* part, const tamc_pt_params* p,
                 uint64_t seed, int mode, tamc_gla** out);
/* GlaResults (src/gla.rs:61-69) sizes and fields: partition_energies[num_partitions],
 * boundary_energies as (bnd_src, bnd_dst, bnd_energies)[num_boundaries], total_energy. */
int tamc_gla_dims(const tamc_gla* r, uint32_t* instance_size, uint32_t* num_partitions, uint32_t* num_boundaries);
int tamc_gla_results(const tamc_gla* r, float* partition_energies, uint32_t* bnd_src, uint32_t* bnd_dst,
                     float* bnd_energies, float* total_energy);
/* The partitions' ground states joined into one state of the whole instance
 * (int8 +-1, n entries).  The reference leaves GlaResults.final_state empty. */
int tamc_gla_state(const tamc_gla* r, int8_t* spins);
/* write_data (src/util.rs:26-36): pickle for a `.pkl` path, else bincode. */
int tamc_gla_write(const tamc_gla* r, const char* path);
void tamc_gla_free(tamc_gla* r);

/* ------------------------------------------------------------------------
 * Temperature-ladder optimisation (tamc-pt-opt).  One update of
 * pt_optimize_beta (src/bin/tamc-pt-opt.rs:59-181) from the statistics that
 * PT runs at the current ladder recorded: round_trips[num_instances] and
 * diffusion_hist[num_instances][nt][2], each summed over the instance's
 * chains (tamc_gpu_pt_round_trips / tamc_gpu_batch_round_trips).  betas[nt]
 * is replaced by the next ladder and momentum[nt] (the first ladder on the
 * first call) updated; tau[num_instances] receives the round-trip times in
 * sweeps and *err the mean |log10| change of the interior betas.  f32
 * arithmetic in the reference's order.  Returns TAMC_OK; 1 when the runs saw
 * too few round trips ("Insufficient round trips for eta CDF": betas and
 * momentum unchanged, tau still written); TAMC_E_REFPANIC where the
 * reference's bisection panics. */
int tamc_pt_opt_step(uint32_t nt, float* betas, float* momentum, uint32_t num_instances,
                     const uint32_t* round_trips, const uint32_t* diffusion_hist, uint32_t num_sweeps,
                     uint32_t num_chains, float alpha, float m, float* tau, float* err);

/* ------------------------------------------------------------------------
 * Serving: continuous batching of solve requests.  Requests arriving while
 * others run are admitted as slots and HBM budget free up; each request keeps
 * its replica state on the device between rounds and retires on its sweep
 * budget or when its best energy reaches target_energy.
 * ---------------------------------------------------------------------- */
typedef struct tamc_server tamc_server;

int tamc_serve_create(tamc_gpu* g, uint64_t hbm_budget_bytes, uint32_t max_active, uint32_t chunk_sweeps,
                      tamc_server** out);
/* Submits a request (host instance is copied).  target_energy = NaN: none. */
int tamc_serve_submit(tamc_server* s, const tamc_host_instance* inst, const tamc_pt_params* p, uint64_t seed,
                      float target_energy, uint64_t* request_id);
/* One scheduling step: admit, run one chunk of rounds for all active requests,
 * retire finished ones.  *active / *queued report the counts afterwards. */
int tamc_serve_step(tamc_server* s, uint32_t* active, uint32_t* queued);
/* Result of a request: done flag (it has ended: finished, cancelled or
 * failed), best energy so far, sweeps run, latency from submit to its end
 * in seconds (-1 while it has not ended). */
int tamc_serve_result(tamc_server* s, uint64_t request_id, int32_t* done, float* best_energy,
                      uint32_t* sweeps, double* latency_s);
/* Final slot-ordered state of a request that ran and ended (finished, or
 * cancelled while active), as tamc_gpu_pt_get_state. */
int tamc_serve_state(tamc_server* s, uint64_t request_id, int8_t* spins, float* energies);
/* Request states reported by tamc_serve_status. */
#define TAMC_REQ_QUEUED 0
#define TAMC_REQ_ACTIVE 1
#define TAMC_REQ_DONE 2      /* sweep budget or target energy reached */
#define TAMC_REQ_CANCELLED 3 /* tamc_serve_cancel */
#define TAMC_REQ_FAILED 4    /* refused at admission; *error says why */
/* State of a request, and for a failed one the reason (valid until the
 * server is destroyed). */
int tamc_serve_status(tamc_server* s, uint64_t request_id, int32_t* status, const char** error);
/* Cancels a queued request (it never runs) or an active one (stopped between
 * steps: its replicas so far are kept as its final state, its device memory
 * and HBM budget are released at once).  Other requests are unaffected.
 * TAMC_E_INVAL for a request that has already ended. */
int tamc_serve_cancel(tamc_server* s, uint64_t request_id);
int tamc_serve_destroy(tamc_server* s);

#ifdef __cplusplus
}
#endif
#endif /* TAMC_GPU_H */
