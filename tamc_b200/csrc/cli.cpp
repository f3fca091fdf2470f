// cli.cpp -- `tamc_b200`, a drop-in for the reference's `tamc` binary
// (src/main.rs:7-18, src/lib.rs:87-131): same positional arguments
// (method file, instance file, output file), same flags (--qubo,
// --suscepts <files>..., --sample-output <file>), same result files
// (PtIcmMinResults YAML + PtIcmThermalSamples bincode/pickle for PT,
// AnnealMinResults YAML/pickle + AnnealState bincode/pickle for SA,
// GlaResults bincode/pickle for GLA).
// Added flags: --seed S (the reference seeds from OS entropy), --mode
// ref|fast, --device D.
#include <chrono>
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

struct Args {
  std::string method, instance, output;
  std::vector<std::string> suscepts;
  std::string sample_output;
  bool has_sample_output = false;
  bool qubo = false;
  bool has_seed = false;
  uint64_t seed = 0;
  int mode = TAMC_MODE_FAST;
  int device = 0;
};

void usage() {
  printf(
      "tamc_b200 (B200 backend of tamc)\n\n"
      "USAGE:\n    tamc_b200 [FLAGS] [OPTIONS] <method-file> <instance-file> <output-file>\n\n"
      "FLAGS:\n    -h, --help       Prints help information\n        --qubo       \n"
      "    -V, --version    Prints version information\n\n"
      "OPTIONS:\n        --sample-output <sample-output>    \n        --suscepts <suscepts>...           \n"
      "        --seed <seed>                      fixed seed (default: OS entropy)\n"
      "        --mode <ref|fast>                  reference-order replay or colour-ordered (default fast)\n"
      "        --device <device>                  CUDA device (default 0)\n");
}

[[noreturn]] void die(const std::string& m) {
  fprintf(stderr, "tamc terminated with an error:\n%s\n * * * * * * \n", m.c_str());
  exit(1);
}

Args parse(int argc, char** argv) {
  Args a;
  std::vector<std::string> pos;
  for (int i = 1; i < argc; ++i) {
    std::string s = argv[i];
    auto val = [&](const char* name) -> std::string {
      const size_t eq = s.find('=');
      if (eq != std::string::npos) return s.substr(eq + 1);
      if (i + 1 >= argc) die(std::string("The argument '") + name + " <" + (name + 2) + ">' requires a value");
      return argv[++i];
    };
    if (s == "-h" || s == "--help") { usage(); exit(0); }
    if (s == "-V" || s == "--version") { printf("tamc_b200 %s\n", tamc_version()); exit(0); }
    if (s == "--qubo") { a.qubo = true; continue; }
    if (s.rfind("--sample-output", 0) == 0) { a.sample_output = val("--sample-output"); a.has_sample_output = true; continue; }
    if (s.rfind("--seed", 0) == 0) { a.seed = strtoull(val("--seed").c_str(), nullptr, 0); a.has_seed = true; continue; }
    if (s.rfind("--device", 0) == 0) { a.device = atoi(val("--device").c_str()); continue; }
    if (s.rfind("--mode", 0) == 0) {
      const std::string m = val("--mode");
      if (m == "ref") a.mode = TAMC_MODE_REF;
      else if (m == "fast") a.mode = TAMC_MODE_FAST;
      else die("--mode must be `ref` or `fast`");
      continue;
    }
    if (s.rfind("--suscepts", 0) == 0) {
      const size_t eq = s.find('=');
      if (eq != std::string::npos) { a.suscepts.push_back(s.substr(eq + 1)); continue; }
      while (i + 1 < argc && argv[i + 1][0] != '-') a.suscepts.push_back(argv[++i]);
      continue;
    }
    if (s.size() > 1 && s[0] == '-') die("Found argument '" + s + "' which wasn't expected");
    pos.push_back(s);
  }
  if (pos.size() != 3) { usage(); die("expected <method-file> <instance-file> <output-file>"); }
  a.method = pos[0];
  a.instance = pos[1];
  a.output = pos[2];
  if (!a.has_seed) a.seed = ((uint64_t)std::random_device{}() << 32) ^ std::random_device{}();
  return a;
}

void check(int rc) {
  if (rc != TAMC_OK) die(tamc_last_error());
}

bool ends_with(const std::string& s, const std::string& e) {
  return s.size() >= e.size() && s.compare(s.size() - e.size(), e.size(), e) == 0;
}
std::string ext_of(const std::string& path) {
  const size_t slash = path.find_last_of('/');
  const std::string base = slash == std::string::npos ? path : path.substr(slash + 1);
  const size_t dot = base.find_last_of('.');
  if (dot == std::string::npos || dot == 0) return "";
  return base.substr(dot + 1);
}
void write_file(const std::string& path, const std::string& data) {
  std::ofstream f(path, std::ios::binary);
  if (!f) die("Failed to create output file '" + path + "'");
  f.write(data.data(), (std::streamsize)data.size());
}

int run_pt(const Args& a, tamc_method* m, tamc_host_instance* hi) {
  tamc_pt_params p;
  check(tamc_method_pt(m, &p));
  const PtParamsHost& ph = m->m.pt;
  printf(" ** Parallel Tempering - ICM **\n");
  fprintf(stderr, "INFO  Number of sweeps: %u\n", p.num_sweeps);
  fprintf(stderr, p.icm ? "INFO  Using ICM\n" : "INFO  ICM Disabled\n");
  tamc_gpu* g = nullptr;
  check(tamc_gpu_open(a.device, &g));
  tamc_inst* d = nullptr;
  check(tamc_gpu_instance_upload(g, hi, &d));
  tamc_pt* pt = nullptr;
  check(tamc_gpu_pt_create(d, &p, a.seed, a.mode, &pt));
  check(tamc_gpu_pt_run(pt, p.num_sweeps));
  check(tamc_gpu_pt_sync(pt));
  uint32_t n = 0, nchi = 0;
  check(tamc_instance_dims(hi, &n, nullptr, nullptr, &nchi));
  PtMinResultsOut r;
  r.params = &ph;
  r.timing_us = tamc_gpu_pt_timing_us(pt);
  r.instance_size = n;
  uint32_t cnt = 0;
  check(tamc_gpu_pt_gs(pt, 0, &cnt, nullptr, nullptr, nullptr));
  const size_t nw = (n + 63) / 64;
  std::vector<uint64_t> words(cnt * nw);
  r.gs_time_steps.resize(cnt);
  r.gs_energies.resize(cnt);
  check(tamc_gpu_pt_gs(pt, cnt, &cnt, r.gs_time_steps.data(), r.gs_energies.data(), words.data()));
  for (uint32_t k = 0; k < cnt; ++k) r.gs_states.emplace_back(words.begin() + k * nw, words.begin() + (k + 1) * nw);
  r.acceptance_counts.resize(p.num_beta);
  check(tamc_gpu_pt_acceptance(pt, r.acceptance_counts.data()));
  printf("PT-ICM Done.\n** Ground state energy **\n");
  if (cnt) {
    printf("  e = %s\n", fmt_f32(r.gs_energies.back()).c_str());
    const uint32_t nsw = r.gs_time_steps.back();
    printf("  nsw = %u\n", nsw);
    printf("  %% remaining = %.3f%%\n", 100.0 * (double)(p.num_sweeps - nsw) / (double)p.num_sweeps);
  }
  write_file(a.output, yaml_pt_min_results(r));
  // PtIcmThermalSamples
  uint32_t M, S, Z;
  check(tamc_gpu_pt_samples_dims(pt, &M, &S, &Z, &nchi));
  const uint32_t nt = p.num_beta, C = p.num_replica_chains, P = C / 2, nb = (n + 7) / 8;
  std::vector<float> e((size_t)nt * M * C), sus((size_t)nt * nchi * M * P);
  std::vector<int32_t> q((size_t)nt * M * P);
  std::vector<uint8_t> smp((size_t)Z * S * C * nb);
  check(tamc_gpu_pt_samples(pt, e.data(), q.data(), sus.data(), smp.data()));
  ThermalSamplesOut t;
  t.compression_level = (uint8_t)p.sample_limiting;
  t.instance_size = n;
  t.beta_arr.assign(p.betas, p.betas + nt);
  t.e.resize(nt);
  t.q.resize(nt);
  t.suscept.resize(nt);
  for (uint32_t k = 0; k < nt; ++k) {
    t.e[k].assign(e.begin() + (size_t)k * M * C, e.begin() + (size_t)(k + 1) * M * C);
    t.q[k].assign(q.begin() + (size_t)k * M * P, q.begin() + (size_t)(k + 1) * M * P);
    t.suscept[k].resize(nchi);
    for (uint32_t c = 0; c < nchi; ++c) {
      const size_t o = ((size_t)k * nchi + c) * M * P;
      t.suscept[k][c].assign(sus.begin() + o, sus.begin() + o + (size_t)M * P);
    }
  }
  t.samples.resize(Z);
  for (uint32_t z = 0; z < Z; ++z)
    for (uint32_t k = 0; k < S * C; ++k) {
      const size_t o = ((size_t)z * S * C + k) * nb;
      t.samples[z].emplace_back(smp.begin() + o, smp.begin() + o + nb);
    }
  const std::string so = a.has_sample_output ? a.sample_output : "samples.bin";
  write_file(so, ext_of(so) == "pkl" ? pickle_thermal_samples(t) : bincode_thermal_samples(t));
  tamc_gpu_pt_destroy(pt);
  tamc_gpu_instance_destroy(d);
  tamc_gpu_close(g);
  return 0;
}

int run_sa(const Args& a, tamc_method* m, tamc_host_instance* hi) {
  const float* betas = nullptr;
  uint32_t nb = 0, R = 0, threads = 0;
  check(tamc_method_sa(m, &betas, &nb, &R, &threads));
  fprintf(stderr, "INFO   ** Simulated Annealing **\n");
  tamc_gpu* g = nullptr;
  check(tamc_gpu_open(a.device, &g));
  tamc_inst* d = nullptr;
  check(tamc_gpu_instance_upload(g, hi, &d));
  uint32_t n = 0;
  check(tamc_instance_dims(hi, &n, nullptr, nullptr, nullptr));
  const uint32_t parts = R > 1 ? threads : 1;
  const uint32_t per = R > 1 && threads ? R / threads : 1;
  const uint32_t Rmax = parts * per;
  const uint32_t nbytes = (n + 7) / 8;
  std::vector<float> e(Rmax);
  std::vector<uint8_t> packed((size_t)Rmax * nbytes);
  uint32_t r_eff = 0;
  const auto t0 = std::chrono::steady_clock::now();
  check(tamc_gpu_sa_run(d, betas, nb, R, threads, a.seed, a.mode, e.data(), packed.data(), &r_eff));
  const double us = std::chrono::duration<double, std::micro>(std::chrono::steady_clock::now() - t0).count();
  AnnealMinResultsOut res;
  res.params = &m->m.sa;
  res.num_replicas_eff = r_eff;
  res.timing_us = us;
  res.energies.assign(e.begin(), e.begin() + r_eff);
  res.min_energy = r_eff ? res.energies[0] : 0.0f;
  for (float v : res.energies) res.min_energy = std::min(res.min_energy, v);
  uint32_t ngs = 0;
  for (float v : res.energies) ngs += v <= res.min_energy;
  const double pgs = r_eff ? (double)ngs / (double)r_eff : 0.0;
  const double tts = (us / 1e6 / (double)R) * (std::log10(0.01) / std::log10(1.0 - pgs));
  fprintf(stderr, "INFO  \n** Ground state energy **\n  e = %s\n** GS Probability  **\n  p_gs = %.4e\n** Time-to-solution **\n  tts = %g s\n",
          fmt_f32(res.min_energy).c_str(), pgs, tts);
  const std::string ext = ext_of(a.output);
  if (ext == "pkl") write_file(a.output, pickle_anneal_min_results(res));
  else if (ext == "yml") write_file(a.output, yaml_anneal_min_results(res));
  std::vector<uint8_t> gsb;
  uint32_t ngs_states = 0;
  for (uint32_t r = 0; r < r_eff; ++r)
    if (res.energies[r] <= res.min_energy + 1.0e-8f) {
      gsb.insert(gsb.end(), packed.begin() + (size_t)r * nbytes, packed.begin() + (size_t)(r + 1) * nbytes);
      ++ngs_states;
    }
  const std::string so = a.has_sample_output ? a.sample_output : "samples.bin";
  write_file(so, ext_of(so) == "pkl" ? pickle_anneal_state(n, ngs_states, gsb) : bincode_anneal_state(n, ngs_states, gsb));
  tamc_gpu_instance_destroy(d);
  tamc_gpu_close(g);
  return 0;
}

// run_gla (src/gla.rs:121-195): the partition file named by the method,
// PT-ICM on every induced sub-instance, GlaResults to the output file
// (pickle for .pkl, else bincode).
int run_gla(const Args& a, tamc_method* m, tamc_host_instance* hi) {
  tamc_pt_params p;
  const char* pfile = nullptr;
  check(tamc_method_gla(m, nullptr, &pfile, &p));
  uint32_t n = 0;
  check(tamc_instance_dims(hi, &n, nullptr, nullptr, nullptr));
  tamc_partition* part = nullptr;
  check(tamc_partition_read(pfile, n, &part));
  uint32_t np = 0;
  check(tamc_partition_dims(part, &np, nullptr));
  fprintf(stderr, "INFO   ** Running GLA with PT-ICM sub-solvers ... (%u partitions)\n", np);
  tamc_gpu* g = nullptr;
  check(tamc_gpu_open(a.device, &g));
  tamc_gla* r = nullptr;
  check(tamc_gla_run(g, hi, part, &p, a.seed, a.mode, &r));
  uint32_t nb = 0;
  check(tamc_gla_dims(r, nullptr, &np, &nb));
  std::vector<float> pe(np), be(nb);
  std::vector<uint32_t> bs(nb), bd(nb);
  float total = 0.0f;
  check(tamc_gla_results(r, pe.data(), bs.data(), bd.data(), be.data(), &total));
  float bulk = 0.0f, bnd = 0.0f;
  for (float e : pe) bulk += e;
  for (float e : be) bnd += e;
  fprintf(stderr, "INFO  Bulk energy: %s\nINFO  Boundary energy: %s\nINFO  Total energy: %s\n",
          fmt_f32(bulk).c_str(), fmt_f32(bnd).c_str(), fmt_f32(total).c_str());
  check(tamc_gla_write(r, a.output.c_str()));
  tamc_gla_free(r);
  tamc_partition_free(part);
  tamc_gpu_close(g);
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  const Args a = parse(argc, argv);
  tamc_method* m = nullptr;
  int rc = tamc_method_read(a.method.c_str(), &m);
  if (rc != TAMC_OK) die(std::string("Failed to parse '") + a.method + "' as valid input\n" + tamc_last_error());
  tamc_host_instance* hi = nullptr;
  check(tamc_instance_read(a.instance.c_str(), a.qubo, &hi));
  for (const auto& f : a.suscepts) check(tamc_instance_add_suscept_file(hi, f.c_str()));
  const int kind = tamc_method_kind(m);
  if (kind == TAMC_METHOD_PT) run_pt(a, m, hi);
  else if (kind == TAMC_METHOD_SA) run_sa(a, m, hi);
  else run_gla(a, m, hi);
  tamc_instance_free(hi);
  tamc_method_free(m);
  printf("tamc finished successfully\n");
  fprintf(stderr, " * * * * * * \n");
  return 0;
}
