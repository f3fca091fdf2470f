// internal.h -- shared host-side declarations of libtamc_b200.
#pragma once
#include <stdint.h>

#include <cmath>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/tamc_gpu.h"

namespace tamc {

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void set_error(const std::string& msg);
[[noreturn]] inline void fail(int code, const std::string& msg) { throw Error(code, msg); }

#define TAMC_API_BEGIN try {
#define TAMC_API_END                                                   \
  }                                                                    \
  catch (const tamc::Error& e) {                                       \
    tamc::set_error(e.what());                                         \
    return e.code;                                                     \
  }                                                                    \
  catch (const std::bad_alloc&) {                                      \
    tamc::set_error("host allocation failed");                         \
    return TAMC_E_NOMEM;                                               \
  }                                                                    \
  catch (const std::exception& e) {                                    \
    tamc::set_error(e.what());                                         \
    return TAMC_E_INVAL;                                               \
  }                                                                    \
  return TAMC_OK;

// A parsed instance: coupling_vecs as CSR (rows sorted by column, QUBO
// self-loops kept), bias, offset, susceptibility weights.
struct HostInstance {
  uint32_t n = 0;
  float offset = 0.0f;
  std::vector<uint32_t> row_ptr{0};
  std::vector<uint32_t> col;
  std::vector<float> J;
  std::vector<float> bias;
  std::vector<std::vector<double>> suscept;

  // The ICM graph's node range also counts self-couplings.  Set on the
  // sub-instances of a GLA split: their `coupling` matrix is built from every
  // row entry, the diagonal included (src/ising.rs:327-355).
  bool diag_in_graph = false;

  uint32_t graph_nodes() const;   // petgraph node count of the ICM graph
  bool has_self_loops() const;
  // Colouring of the off-diagonal graph: bipartite 2-colouring when possible,
  // else largest-first greedy followed by an equitable rebalancing pass.
  void coloring(uint32_t& ncolors, std::vector<uint32_t>& color) const;
  float energy_ref(const int8_t* s) const;
};

void parse_instance_text(const char* text, size_t len, bool qubo, HostInstance& out);
// induced_subgraph_instance_sorted (src/ising.rs:327-355): the sub-instance on
// the sorted site list `nodes`, offset 0, rows keep the entries whose column is
// in `nodes` (renumbered by position), susceptibility weights restricted.
HostInstance induced_sorted(const HostInstance& h, const std::vector<uint32_t>& nodes);
std::vector<double> read_txt_vec_file(const std::string& path);

// Method file
struct BetaSpec {
  bool geometric = true;
  float beta_min = 0, beta_max = 0;
  uint32_t num_beta = 0;
  std::vector<float> arr;
  std::vector<float> resolve() const;
};
struct PtParamsHost {
  uint32_t num_sweeps = 0;
  double warmup_fraction = 0;
  BetaSpec beta;
  bool has_lo_beta = false;
  float lo_beta = 0;
  bool has_lo_num_beta = false;
  uint32_t lo_num_beta = 0;
  bool icm = false;
  uint32_t num_replica_chains = 0;
  uint32_t threads = 0;
  bool has_sample = false, has_sample_states = false, has_sample_limiting = false;
  uint32_t sample = 0, sample_states = 0;
  uint8_t sample_limiting = 0;
};
struct SaParamsHost {
  BetaSpec beta;
  uint32_t num_replicas = 0;
  uint32_t threads = 0;
};
struct GlaParamsHost {
  uint32_t num_threads = 0;
  std::string partition_file;
};
struct Method {
  int kind = 0;
  PtParamsHost pt;  // PT, or GLA's pt_params
  GlaParamsHost gla;
  SaParamsHost sa;
  std::vector<float> betas;  // resolved
  uint32_t lo_beta_idx = 0;
};
void parse_method_yaml(const std::string& text, Method& m);
std::vector<float> geometric_betas(float bmin, float bmax, uint32_t n);
uint32_t resolve_lo_beta_idx(const PtParamsHost& p, const std::vector<float>& betas, bool* warn);

// Output writers (formats of the reference's result files)
struct PtMinResultsOut {
  const PtParamsHost* params;
  double timing_us;
  std::vector<uint32_t> gs_time_steps;
  std::vector<float> gs_energies;
  std::vector<std::vector<uint64_t>> gs_states;
  uint32_t instance_size;
  std::vector<uint32_t> acceptance_counts;
};
struct ThermalSamplesOut {
  uint8_t compression_level;
  uint64_t instance_size;
  std::vector<float> beta_arr;
  std::vector<std::vector<std::vector<uint8_t>>> samples;
  std::vector<std::vector<float>> e;
  std::vector<std::vector<int32_t>> q;
  std::vector<std::vector<std::vector<float>>> suscept;
};
struct AnnealMinResultsOut {
  const SaParamsHost* params;
  uint32_t num_replicas_eff;
  double timing_us;
  float min_energy;
  std::vector<float> energies;
};
std::string yaml_pt_min_results(const PtMinResultsOut& r);
// serde_yaml of Method::PT(params) (src/lib.rs:80-85), as tamc-pt-opt writes it
std::string yaml_pt_method(const PtParamsHost& p);
std::string fmt_f32_display(float v);
std::string yaml_anneal_min_results(const AnnealMinResultsOut& r);
std::string bincode_thermal_samples(const ThermalSamplesOut& t);
std::string bincode_anneal_state(uint32_t instance_size, uint32_t num_replicas, const std::vector<uint8_t>& bytes);
std::string pickle_thermal_samples(const ThermalSamplesOut& t);
std::string pickle_anneal_min_results(const AnnealMinResultsOut& r);
std::string pickle_anneal_state(uint32_t instance_size, uint32_t num_replicas, const std::vector<uint8_t>& bytes);
// GlaResults (src/gla.rs:61-69)
struct GlaResultsOut {
  uint32_t instance_size = 0;
  uint32_t num_partitions = 0;
  std::vector<float> partition_energies;
  std::vector<uint32_t> bnd_src, bnd_dst;
  std::vector<float> bnd_energies;
  float total_energy = 0.0f;
};
std::string bincode_gla_results(const GlaResultsOut& r);
std::string pickle_gla_results(const GlaResultsOut& r);
// read_u32_lines (src/util.rs:142-172) checked as GlaParams::read_graph_partition
// (src/gla.rs:37-58) for an instance of n sites.
void parse_partition(const char* text, size_t len, uint32_t n, std::vector<std::vector<uint32_t>>& parts);
std::string fmt_f32(float v);
std::string fmt_f64(double v);

}  // namespace tamc

struct tamc_host_instance {
  tamc::HostInstance h;
};
struct tamc_method {
  tamc::Method m;
};
