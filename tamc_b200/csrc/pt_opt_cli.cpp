// pt_opt_cli.cpp -- `tamc_b200_pt_opt`, a drop-in for the reference's
// `tamc-pt-opt` binary (src/bin/tamc-pt-opt.rs): optimises the temperature
// ladder of a PT method over a set of instances.  Same arguments
// (--max-iters, --step-size, --momentum, --tolerance, --opt-params,
// --tau-hist, <params> <instances>...) and outputs (the optimised method as
// YAML, with num_sweeps doubled; the round-trip times of every iteration as
// CSV rows).  Each iteration runs every instance at the current ladder --
// all of them as one batch on the GPU, continuing from the previous
// iteration's replicas -- and feeds the round trips and diffusion histograms
// to tamc_pt_opt_step.  Added flags: --seed S (the reference seeds every run
// from OS entropy; here run k of iteration i takes the (i * instances + k)-th
// SplitMix64 output of S), --device D.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <random>
#include <string>
#include <vector>

#include "internal.h"

using namespace tamc;

namespace {

[[noreturn]] void die(const std::string& m) {
  fprintf(stderr, "tamc-pt-opt terminated with an error:\n%s\n", m.c_str());
  exit(1);
}
void check(int rc) {
  if (rc != TAMC_OK) die(tamc_last_error());
}

uint64_t splitmix_next(uint64_t& st) {
  st += 0x9e3779b97f4a7c15ULL;
  uint64_t z = st;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

struct Args {
  uint32_t max_iters = 1000;
  float step_size = 0.2f, momentum = 0.85f, tolerance = 0.02f;
  std::string opt_params = "opt_params.yml", tau_hist = "tau_hist.csv";
  std::string params;
  std::vector<std::string> instances;
  uint64_t seed = 0;
  bool has_seed = false;
  int device = 0;
};

void usage() {
  printf(
      "pt-opt 0.1.0\nOptimize the PT temperature set over a set of instances.\n\n"
      "USAGE:\n    tamc_b200_pt_opt [OPTIONS] <params> [instances]...\n\n"
      "OPTIONS:\n        --max-iters <max-iters>       [default: 1000]\n"
      "        --momentum <momentum>         [default: 0.85]\n"
      "        --opt-params <opt-params>    Destination for optimized parameters [default: opt_params.yml]\n"
      "        --step-size <step-size>       [default: 0.2]\n"
      "        --tau-hist <tau-hist>         [default: tau_hist.csv]\n"
      "        --tolerance <tolerance>      Covergence tolerance criterion (MAE of log-betas) [default: 0.02]\n"
      "        --seed <seed>                fixed seed (default: OS entropy)\n"
      "        --device <device>            CUDA device (default 0)\n");
}

Args parse(int argc, char** argv) {
  Args a;
  std::vector<std::string> pos;
  for (int i = 1; i < argc; ++i) {
    std::string s = argv[i];
    auto val = [&](const char* name) -> std::string {
      const size_t eq = s.find('=');
      if (eq != std::string::npos) return s.substr(eq + 1);
      if (i + 1 >= argc) die(std::string("The argument '") + name + "' requires a value");
      return argv[++i];
    };
    auto starts = [&](const char* f) { return s == f || s.rfind(std::string(f) + "=", 0) == 0; };
    if (s == "-h" || s == "--help") { usage(); exit(0); }
    if (starts("--max-iters")) { a.max_iters = (uint32_t)strtoul(val("--max-iters").c_str(), nullptr, 10); continue; }
    if (starts("--step-size")) { a.step_size = strtof(val("--step-size").c_str(), nullptr); continue; }
    if (starts("--momentum")) { a.momentum = strtof(val("--momentum").c_str(), nullptr); continue; }
    if (starts("--tolerance")) { a.tolerance = strtof(val("--tolerance").c_str(), nullptr); continue; }
    if (starts("--opt-params")) { a.opt_params = val("--opt-params"); continue; }
    if (starts("--tau-hist")) { a.tau_hist = val("--tau-hist"); continue; }
    if (starts("--seed")) { a.seed = strtoull(val("--seed").c_str(), nullptr, 0); a.has_seed = true; continue; }
    if (starts("--device")) { a.device = atoi(val("--device").c_str()); continue; }
    if (s.size() > 1 && s[0] == '-') die("Found argument '" + s + "' which wasn't expected");
    pos.push_back(s);
  }
  if (pos.empty()) die("The following required arguments were not provided:\n    <params>");
  a.params = pos[0];
  a.instances.assign(pos.begin() + 1, pos.end());
  if (!a.has_seed) a.seed = ((uint64_t)std::random_device{}() << 32) ^ std::random_device{}();
  return a;
}

std::string row(const std::vector<float>& v, int width, int prec) {
  std::string o;
  char b[64];
  for (float x : v) {
    snprintf(b, sizeof b, " %*.*f ", width, prec, (double)x);
    o += b;
  }
  return o;
}

}  // namespace

int main(int argc, char** argv) {
  const Args a = parse(argc, argv);
  tamc_method* m = nullptr;
  if (tamc_method_read(a.params.c_str(), &m) != TAMC_OK) die(tamc_last_error());
  if (tamc_method_kind(m) != TAMC_METHOD_PT) {
    fprintf(stderr, "WARN  Must input a PT method for tamc-pt-opt\n");
    tamc_method_free(m);
    return 0;
  }
  PtParamsHost ph = m->m.pt;
  std::vector<float> betas = m->m.betas;
  const uint32_t nt = (uint32_t)betas.size();
  const uint32_t C = ph.num_replica_chains;
  if (nt < 3) die("tamc-pt-opt needs at least 3 temperatures");
  // instances read without the QUBO conversion (src/bin/tamc-pt-opt.rs:204-205)
  tamc_gpu* g = nullptr;
  check(tamc_gpu_open(a.device, &g));
  std::vector<tamc_host_instance*> hosts;
  std::vector<tamc_inst*> dinst;
  std::vector<uint32_t> ns;
  for (const auto& f : a.instances) {
    tamc_host_instance* h = nullptr;
    check(tamc_instance_read(f.c_str(), 0, &h));
    tamc_inst* d = nullptr;
    check(tamc_gpu_instance_upload(g, h, &d));
    uint32_t n = 0;
    check(tamc_instance_dims(h, &n, nullptr, nullptr, nullptr));
    hosts.push_back(h);
    dinst.push_back(d);
    ns.push_back(n);
  }
  const uint32_t I = (uint32_t)dinst.size();
  if (!I) die("no instance files given");
  std::vector<float> mom(betas);
  std::vector<std::vector<float>> tau_hist;
  std::vector<std::vector<int8_t>> init;  // previous iteration's replicas, per instance
  uint64_t seeds = a.seed;
  for (uint32_t it = 0; it < a.max_iters; ++it) {
    printf("* Iteration %u.\n* Step Size: %s\n", it, fmt_f32_display(a.step_size).c_str());
    // PtIcmRunner::new(instance, params) at the current ladder; run() is the
    // single-stream loop whatever `threads` says
    ph.beta.geometric = false;
    ph.beta.arr = betas;
    tamc_pt_params p;
    p.num_sweeps = ph.num_sweeps;
    p.warmup_fraction = ph.warmup_fraction;
    p.num_beta = nt;
    p.betas = betas.data();
    try {
      p.lo_beta_idx = resolve_lo_beta_idx(ph, betas, nullptr);
    } catch (const std::exception& e) {
      die(e.what());
    }
    p.icm = ph.icm;
    p.num_replica_chains = C;
    p.threads = 1;
    p.sample = ph.has_sample ? (int64_t)ph.sample : -1;
    p.sample_states = ph.has_sample_states ? (int64_t)ph.sample_states : -1;
    p.sample_limiting = ph.has_sample_limiting ? ph.sample_limiting : 0;
    tamc_batch* b = nullptr;
    check(tamc_gpu_batch_create(g, &b));
    for (uint32_t k = 0; k < I; ++k) {
      check(tamc_gpu_batch_add(b, dinst[k], &p, splitmix_next(seeds), nullptr));
      if (!init.empty()) check(tamc_gpu_batch_set_state(b, k, init[k].data()));
    }
    check(tamc_gpu_batch_run(b));
    check(tamc_gpu_batch_sync(b));
    std::vector<uint32_t> rts(I, 0), dh((size_t)I * nt * 2, 0);
    std::vector<std::vector<int8_t>> fin(I);
    for (uint32_t k = 0; k < I; ++k) {
      std::vector<uint32_t> r(C), d((size_t)C * nt * 2);
      check(tamc_gpu_batch_round_trips(b, k, nullptr, r.data(), d.data()));
      for (uint32_t c = 0; c < C; ++c) {
        rts[k] += r[c];
        for (uint32_t x = 0; x < nt * 2; ++x) dh[(size_t)k * nt * 2 + x] += d[(size_t)c * nt * 2 + x];
      }
      fin[k].resize((size_t)C * nt * ns[k]);
      check(tamc_gpu_batch_get_state(b, k, fin[k].data(), nullptr));
    }
    check(tamc_gpu_batch_destroy(b));
    const std::vector<float> prev(betas);
    std::vector<float> tau(I);
    float err = 0.0f;
    const int rc = tamc_pt_opt_step(nt, betas.data(), mom.data(), I, rts.data(), dh.data(), ph.num_sweeps, C,
                                    a.step_size, a.momentum, tau.data(), &err);
    if (rc < 0) die(tamc_last_error());
    printf("Round-trip times (sweeps):\n[%s]\n", row(tau, 0, 1).c_str());
    tau_hist.push_back(tau);
    if (rc == 1) {
      fprintf(stderr, "WARN   ** Insufficient round trips for eta CDF\n");
      continue;
    }
    printf("%9s%9s%9s\n", "beta", "betaM", "beta'");
    printf("--------------------------\n");
    for (uint32_t t = 0; t < nt; ++t) printf(" %7.4f  %7.4f  %7.4f \n", prev[t], mom[t], betas[t]);
    printf("Mean abs log rel_err: %s\n", fmt_f32_display(err).c_str());
    init = std::move(fin);  // the replicas continue, their tags reset (PTState::reset_tags)
    if (err < a.tolerance) {
      printf(" ** Relative Error converged\n");
      break;
    }
  }
  printf("Final temperature array:\n[%s]\n", row(betas, 0, 5).c_str());
  ph.beta.geometric = false;
  ph.beta.arr = betas;
  ph.num_sweeps *= 2;  // double the number of sweeps
  const std::string y = yaml_pt_method(ph);
  printf("%s\n", y.c_str());
  printf("\n\n ** Writing to %s **\n", a.opt_params.c_str());
  {
    std::ofstream f(a.opt_params, std::ios::binary);
    if (!f) die("could not write " + a.opt_params);
    f << y;
  }
  {
    std::ofstream f(a.tau_hist, std::ios::binary);
    if (!f) die("could not write " + a.tau_hist);
    for (const auto& r : tau_hist) {
      for (float x : r) f << fmt_f32_display(x) << ",";
      f << "\n";
    }
  }
  for (auto* d : dinst) tamc_gpu_instance_destroy(d);
  for (auto* h : hosts) tamc_instance_free(h);
  tamc_method_free(m);
  tamc_gpu_close(g);
  return 0;
}
