// pt.cuh -- the PT-ICM run handle shared by the reference-order and fast paths.
#pragma once
#include <chrono>
#include <memory>

#include "fast_common.cuh"
#include "ref_kernels.cuh"

namespace tamc {

template <class T>
struct DBuf {  // owning device buffer, or a view into another buffer's block
  T* p = nullptr;
  size_t n = 0;
  bool own = true;
  DBuf() = default;
  explicit DBuf(size_t count) { alloc(count); }
  void release() {
    if (p && own) dev_free(p, std::max<size_t>(n, 1) * sizeof(T));
    p = nullptr;
  }
  void alloc(size_t count) {
    release();
    own = true;
    n = count;
    p = static_cast<T*>(dev_alloc(std::max<size_t>(count, 1) * sizeof(T)));
  }
  // `count` elements at `q`, inside a block that another DBuf owns and frees
  void view(void* q, size_t count) {
    release();
    own = false;
    n = count;
    p = static_cast<T*>(q);
  }
  void zero(cudaStream_t st) { TAMC_CUDA(cudaMemsetAsync(p, 0, std::max<size_t>(n, 1) * sizeof(T), st)); }
  ~DBuf() { release(); }
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
};

// Resolved run configuration (PtIcmParams + PtIcmRunner::new, src/pt.rs:307-351).
struct PtCfg {
  uint32_t num_sweeps = 0;
  double warmup = 0;
  std::vector<float> betas;
  uint32_t nt = 0, C = 0, lo = 0;
  bool icm = false;
  uint32_t threads = 1;
  int64_t sample = -1, sample_states = -1;
  uint32_t level = 0;
  uint32_t meas_init = 0;
  uint32_t M = 0, S = 0, Z = 0;  // measurements, state snapshots, sample slots
  bool is_meas(uint32_t i) const {
    return sample >= 0 && i >= meas_init && ((i - meas_init) % (uint32_t)sample == 0 || i == num_sweeps - 1);
  }
  bool is_snap(uint32_t i) const {
    return sample_states >= 0 && i >= meas_init &&
           ((i - meas_init) % (uint32_t)sample_states == 0 || i == num_sweeps - 1);
  }
};
PtCfg make_cfg(const tamc_pt_params* p);

// Device output buffers and the host-side ground-state trajectory.
struct PtOutputs {
  uint32_t n = 0, nchi = 0;
  DBuf<float> e;
  DBuf<int32_t> q;
  DBuf<float> sus;
  DBuf<uint8_t> samp;
  DBuf<char> gs_cells;  // one block holding the three cells below
  DBuf<uint32_t> gs_count;
  DBuf<int> gs_have;
  DBuf<float> gs_min;
  DBuf<uint32_t> gs_steps;
  DBuf<float> gs_E;
  DBuf<uint64_t> gs_words;
  uint32_t cap = 0;
  uint32_t pending = 0;  // tracked sweeps since the last drain
  bool dirty = true;     // rounds may have logged entries since the last drain
  std::vector<uint32_t> h_steps;
  std::vector<float> h_E;
  std::vector<uint64_t> h_words;  // concatenated
  void init(const PtCfg& c, uint32_t n_, uint32_t nchi_, cudaStream_t st);
  MeasOut meas(const PtCfg& c) const;
  GsLog log() const;
  void drain(cudaStream_t st);  // synchronous
};

}  // namespace tamc

namespace tamc {
// A reference-order run whose initial replicas and serial loop draw from the
// Xoshiro256++ state `master` (p->threads should be <= 1: the single-stream
// pt_loop), as GLA's sub-solvers run (src/gla.rs:148-166).
tamc_pt* pt_create_ref_stream(tamc_inst* inst, const tamc_pt_params* p, const Xo& master);
}  // namespace tamc

struct tamc_pt {
  tamc_inst* inst = nullptr;
  tamc_gpu* g = nullptr;
  int mode = 0;
  tamc::PtCfg cfg;
  uint32_t next_sweep = 0;
  uint32_t m_next = 0, s_next = 0;  // next measurement / snapshot index
  double timing_us = 0;
  bool running = false;
  std::chrono::steady_clock::time_point t0;
  tamc::PtOutputs out;
  // reference-order state
  tamc::DBuf<int8_t> spins;
  tamc::DBuf<float> energy;
  tamc::DBuf<uint32_t> perm;
  tamc::DBuf<uint8_t> tags;
  tamc::DBuf<uint32_t> acc;
  tamc::DBuf<uint32_t> rtrips;
  tamc::DBuf<uint32_t> dhist;
  tamc::DBuf<float> e_stale;
  tamc::DBuf<float> d_betas;
  tamc::DBuf<float> d_dbeta;
  tamc::DBuf<uint32_t> visited;
  tamc::DBuf<uint32_t> queue;
  tamc::DBuf<float> rows;
  tamc::DBuf<tamc::Xo> rng;
  tamc::DBuf<int> err;
  // fast-mode state lives behind an opaque pointer (fast_pt.cu)
  struct FastState;
  FastState* fast = nullptr;
  bool fast_plain() const;  // the run uses the all-SM plain form
  bool fast_deferred() const;  // a batch run whose initial replicas wait for the batch's first chunk
};
