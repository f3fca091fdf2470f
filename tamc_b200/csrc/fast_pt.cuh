// fast_pt.cuh -- colour-ordered PT-ICM (TAMC_MODE_FAST): job description of the
// fused round kernel and the glue used by the tamc_pt / tamc_batch handles.
#pragma once
#include "fast_common.cuh"
#include "pt.cuh"

namespace tamc {

// One PT-ICM run as the fused kernel sees it.  Spins are stored slot-major:
// W[s * nw + c * wpc + w] holds, in bit b, the spin of the replica currently at
// temperature slot 32*w + b of chain c (1 = spin -1), sites in colour order.
struct PtJob {
  FastInst F;
  uint32_t n, nt, ntp, C, wpc, nw, lo, qpc, qps;
  int32_t icm, threaded, self_loops, csr_smem;
  int32_t init;        // 0: load state, 1: random spins + energies, 2: load spins + energies
  uint32_t icm_group;  // ICM slots labelled together (label arrays in shared memory)
  int32_t icm_uf;      // cluster search: 0 = frontier BFS from the seeds, 1 = union-find labelling
  const float* betas;  // [ntp], padding slots have beta = 0
  uint2 key;
  uint32_t* W;         // [n][nw]
  double* Ec;          // [C][ntp] cached energy as the reference keeps it
  double* Er;          // [C][ntp] energy_ref of the current spins
  uint8_t* tags;       // [C][nt]
  uint32_t* acc;       // [C][nt]
  uint32_t* rtrips;    // [C]
  uint32_t* dhist;     // [C][nt][2]
  uint32_t sweep_begin, sweep_end, num_sweeps, meas_init;
  int64_t sample, sample_states;
  uint32_t level, m_base, s_base;
  MeasOut out;
  GsLog log;
  uint32_t* count_out; // if set: receives the log count when the job's range is done
  unsigned long long* prof;  // if set: per-phase clock64 cycles (PHASE_* order), off otherwise
  uint64_t cost;       // sweeps * n * R, for longest-first ordering
  int32_t msc;         // multi-spin-coded sweep (+-J instance, nw in {1, 2, 4})
  int32_t pad_;
};

enum { PHASE_ICM_SCAN, PHASE_ICM_INIT, PHASE_ICM_JUMP, PHASE_ICM_GROW, PHASE_ICM_MARK, PHASE_ICM_APPLY, PHASE_EXCH,
       PHASE_SWEEP, PHASE_MEASURE, PHASE_OTHER,
       // multi-spin-coded sweep, per warp (summed over warps): loads and bond
       // levels, flip decisions, energy sums and stores, barrier waits
       PHASE_SW_LEVELS, PHASE_SW_FLIP, PHASE_SW_ENERGY, PHASE_SW_WAIT, PHASE_N };

// Shared-memory bytes the fused kernel needs for a job with T threads.
size_t fused_smem_bytes(const PtJob& j, uint32_t T, bool csr_smem);
// Resident CTAs per SM for the fused kernel at this size.
int fused_blocks_per_sm(uint32_t T, size_t smem);
// Launch over `njobs` jobs already on the device; `ctr` is a zeroed counter.
void fused_launch(cudaStream_t st, const PtJob* d_jobs, uint32_t njobs, uint32_t* ctr, uint32_t grid,
                  uint32_t T, size_t smem);
// A fused launch with a launch priority (cudaLaunchAttributePriority; lower
// numbers run first); the shared-memory attribute must already cover `smem`
// (fused_smem_limit).
void fused_launch_prio(cudaStream_t st, const PtJob* d_jobs, uint32_t njobs, uint32_t* ctr, uint32_t grid, uint32_t T,
                       size_t smem, int priority);
void fused_smem_limit(size_t smem);

// Plain form (one instance over the whole GPU, one launch per sweep phase).
struct PlainCtl {
  uint32_t i;        // next round to start
  uint32_t m_cur;    // next measurement index
  uint32_t s_cur;    // next state-snapshot index
  uint32_t pending;  // the sweeps of round i-1 ran; their sums and measurements are pending
  uint32_t icm_done; // Houdayer CTAs of the current round that finished (reset by the last)
  uint32_t sweep_done; // CTAs of the round's last sweep launch that finished (reset by the last)
};
// with stage: room to hold the replica words and weights of a measured round
size_t plain_head_bytes(const PtJob& j, bool stage);
// mode 1: close the previous round (sweep sums, measurements); 2: set initial energies
void plain_launch_head(cudaStream_t st, const PtJob* d_job, PlainCtl* ctl, long long* acc, int mode, size_t smem,
                       int stage);
size_t plain_icm_bytes(const PtJob& j);
// Houdayer moves of round ctl->i, one CTA (or cluster) per (chain pair, slot
// >= lo); the last CTA also runs the exchange decisions (writing dm).  Returns
// false, and launches nothing, when the round has no Houdayer move.
// With rows of 4 or 6 entries, each (pair, slot) runs on a cluster of 2 or 4
// CTAs over distributed shared memory (TAMC_PLAIN_CLUSTER=0 keeps one CTA).
bool plain_launch_icm(cudaStream_t st, const PtJob& j, const PtJob* d_job, PlainCtl* ctl, long long* icm_dE,
                      uint32_t* icm_valid, size_t smem_limit, uint32_t num_sms, unsigned long long* dm);
// energies after ICM and the exchange decisions; advances ctl->i
void plain_launch_exch(cudaStream_t st, const PtJob& j, const PtJob* d_job, PlainCtl* ctl, const long long* icm_dE,
                       uint32_t* icm_valid, unsigned long long* dm);
// the exchange's spin permutation over all site words
void plain_launch_perm(cudaStream_t st, const PtJob& j, const PtJob* d_job, const unsigned long long* dm,
                       uint32_t grid_cap);
// one launch per colour class; the last class's launch also closes the round
// when it takes no measurement (energies, ground-state tracking)
void plain_launch_sweep(cudaStream_t st, const PtJob& j, const PtJob* d_job, PlainCtl* ctl, uint32_t color,
                        uint32_t ntask, long long* acc, uint32_t grid_cap);
void plain_launch_init(cudaStream_t st, const PtJob* d_job, long long* acc, int random, uint32_t grid);

// tamc_pt glue (single-instance handle in fast mode)
void fast_pt_create(tamc_pt* pt, uint64_t seed);
void fast_pt_run(tamc_pt* pt, uint32_t sweep_end);
void fast_pt_get_state(tamc_pt* pt, int8_t* spins, float* energies);
void fast_pt_set_state(tamc_pt* pt, const int8_t* spins);
void fast_pt_acceptance(tamc_pt* pt, uint32_t* acc);
void fast_pt_round_trips(tamc_pt* pt, uint8_t* tags, uint32_t* round_trips, uint32_t* dhist);
void fast_pt_phase_cycles(tamc_pt* pt, uint64_t* out);
void fast_pt_destroy(tamc_pt* pt);

}  // namespace tamc
