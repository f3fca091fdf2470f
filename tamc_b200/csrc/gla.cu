// gla.cu -- GLA partitioned solves (run_gla, src/gla.rs:121-195) on the PT-ICM
// runs: the instance is split into the sub-instances induced by a partition of
// its sites, each sub-instance is solved by PT-ICM -- all of them in one batch
// (persistent kernel over a job per sub-instance) in colour-ordered mode, or
// one reference-order run each on its own jumped Xoshiro256++ stream -- and
// the sub-solutions' last ground states are joined across the partition with
// the couplings that cross it (boundary energies).
#include <algorithm>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>

#include "pt.cuh"

struct tamc_partition {
  uint32_t n = 0;                            // instance size the partition was checked against
  std::vector<std::vector<uint32_t>> parts;  // site lists in file order, as read
};

struct tamc_gla {
  tamc::GlaResultsOut r;
  std::vector<int8_t> joined;  // the partitions' ground states on the whole instance
};

namespace tamc {
namespace {

inline uint64_t splitmix_next(uint64_t& st) {
  st += 0x9e3779b97f4a7c15ULL;
  uint64_t z = st;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

void check_rc(int rc) {
  if (rc != TAMC_OK) fail(rc, tamc_last_error());
}

struct Edge {
  uint32_t i, j;
  float K;
};

// The last ground-state entry of a finished run: energy and +-1 spins.
void last_ground_state(tamc_pt* pt, uint32_t n, float& e, std::vector<int8_t>& s) {
  uint32_t cnt = 0;
  check_rc(tamc_gpu_pt_gs(pt, 0, &cnt, nullptr, nullptr, nullptr));
  // gs_states.last().unwrap() (src/gla.rs:169-171)
  if (!cnt) fail(TAMC_E_REFPANIC, "a sub-instance run recorded no ground state (the reference panics)");
  const uint32_t nw = (n + 63) / 64;
  std::vector<uint32_t> steps(cnt);
  std::vector<float> en(cnt);
  std::vector<uint64_t> words((size_t)cnt * nw);
  check_rc(tamc_gpu_pt_gs(pt, cnt, &cnt, steps.data(), en.data(), words.data()));
  e = en[cnt - 1];
  // IsingState::from_u64_vec (src/ising.rs:139-155): bit set = spin -1
  s.assign(n, 1);
  const uint64_t* w = words.data() + (size_t)(cnt - 1) * nw;
  for (uint32_t i = 0; i < n; ++i) s[i] = ((w[i / 64] >> (i % 64)) & 1u) ? -1 : 1;
}

}  // namespace
}  // namespace tamc

using namespace tamc;

extern "C" {

int tamc_partition_parse(const char* text, uint64_t len, uint32_t n, tamc_partition** out) {
  TAMC_API_BEGIN
  if (!out || (!text && len)) fail(TAMC_E_INVAL, "null argument");
  auto* p = new tamc_partition();
  try {
    p->n = n;
    parse_partition(text, (size_t)len, n, p->parts);
  } catch (...) {
    delete p;
    throw;
  }
  *out = p;
  TAMC_API_END
}

int tamc_partition_read(const char* path, uint32_t n, tamc_partition** out) {
  TAMC_API_BEGIN
  if (!path) fail(TAMC_E_INVAL, "null path");
  std::ifstream f(path, std::ios::binary);
  if (!f) fail(TAMC_E_IO, std::string("Could not open partition file '") + path + "'");
  std::stringstream ss;
  ss << f.rdbuf();
  const std::string s = ss.str();
  return tamc_partition_parse(s.data(), s.size(), n, out);
  TAMC_API_END
}

int tamc_partition_dims(const tamc_partition* p, uint32_t* num_parts, uint64_t* num_sites) {
  TAMC_API_BEGIN
  if (!p) fail(TAMC_E_INVAL, "null partition");
  uint64_t total = 0;
  for (const auto& v : p->parts) total += v.size();
  if (num_parts) *num_parts = (uint32_t)p->parts.size();
  if (num_sites) *num_sites = total;
  TAMC_API_END
}

int tamc_partition_get(const tamc_partition* p, uint32_t* part_ptr, uint32_t* sites) {
  TAMC_API_BEGIN
  if (!p) fail(TAMC_E_INVAL, "null partition");
  uint32_t o = 0;
  for (size_t k = 0; k < p->parts.size(); ++k) {
    if (part_ptr) part_ptr[k] = o;
    if (sites) std::copy(p->parts[k].begin(), p->parts[k].end(), sites + o);
    o += (uint32_t)p->parts[k].size();
  }
  if (part_ptr) part_ptr[p->parts.size()] = o;
  TAMC_API_END
}

void tamc_partition_free(tamc_partition* p) { delete p; }

int tamc_gla_run(tamc_gpu* g, const tamc_host_instance* hi, const tamc_partition* part, const tamc_pt_params* p,
                 uint64_t seed, int mode, tamc_gla** out) {
  TAMC_API_BEGIN
  if (!g || !hi || !part || !p || !out) fail(TAMC_E_INVAL, "null argument");
  if (mode != TAMC_MODE_REF && mode != TAMC_MODE_FAST) fail(TAMC_E_INVAL, "unknown mode");
  const HostInstance& h = hi->h;
  const uint32_t n = h.n;
  if (part->n != n)
    fail(TAMC_E_INVAL, "the partition was checked against an instance of " + std::to_string(part->n) +
                           " sites, not " + std::to_string(n));
  // to_energy_graph (src/ising.rs:414-425): the coupling matrix's entries with
  // i < j in row order; its nodes run to the largest endpoint, and setting
  // the bias of a site beyond them panics in the reference
  std::vector<Edge> edges;
  uint32_t gn = 0;
  for (uint32_t i = 0; i < n; ++i)
    for (uint32_t e = h.row_ptr[i]; e < h.row_ptr[i + 1]; ++e)
      if (h.col[e] > i) {
        edges.push_back(Edge{i, h.col[e], h.J[e]});
        gn = std::max(gn, h.col[e] + 1);
      }
  if (gn < n)
    fail(TAMC_E_REFPANIC, "site " + std::to_string(n - 1) +
                              " couples to no other site; the reference's energy graph has fewer nodes and it panics");
  const uint32_t np = (uint32_t)part->parts.size();
  std::vector<uint32_t> pid(n, 0xffffffffu);
  for (uint32_t k = 0; k < np; ++k)
    for (uint32_t i : part->parts[k]) pid[i] = k;
  for (uint32_t i = 0; i < n; ++i)  // partition_mapping[&i] (src/gla.rs:92-95)
    if (pid[i] == 0xffffffffu)
      fail(TAMC_E_REFPANIC, "site " + std::to_string(i) + " is in no partition (the reference panics)");
  // partition graph (instance_partition, src/gla.rs:78-117): partitions as
  // sorted site lists; one directed edge per ordered pair (partition of i,
  // partition of j), in order of first appearance, holding its (i, j, K)
  std::vector<std::vector<uint32_t>> sorted(part->parts);
  for (auto& v : sorted) std::sort(v.begin(), v.end());
  std::map<uint64_t, uint32_t> bindex;
  std::vector<std::pair<uint32_t, uint32_t>> bkeys;
  std::vector<std::vector<Edge>> bedges;
  for (const Edge& e : edges) {
    const uint32_t a = pid[e.i], b = pid[e.j];
    if (a == b) continue;
    const uint64_t key = ((uint64_t)a << 32) | b;
    auto it = bindex.find(key);
    if (it == bindex.end()) {
      it = bindex.emplace(key, (uint32_t)bkeys.size()).first;
      bkeys.emplace_back(a, b);
      bedges.emplace_back();
    }
    bedges[it->second].push_back(e);
  }
  // sub-solvers: PtIcmRunner::pt_loop, the single-stream loop, whatever
  // pt_params.threads says (src/gla.rs:161-164)
  tamc_pt_params q = *p;
  q.threads = 1;
  std::vector<float> part_e(np);
  std::vector<std::vector<int8_t>> part_s(np);
  std::vector<tamc_inst*> dinst(np, nullptr);
  auto release = [&]() {
    for (tamc_inst* d : dinst)
      if (d) tamc_gpu_instance_destroy(d);
  };
  try {
    // the sub-instances (induced_subgraph_instance_sorted, src/gla.rs:137-139),
    // uploaded together
    std::vector<tamc_host_instance> subs(np);
    std::vector<const tamc_host_instance*> subp(np);
    for (uint32_t k = 0; k < np; ++k) {
      subs[k].h = induced_sorted(h, sorted[k]);
      subp[k] = &subs[k];
    }
    check_rc(tamc_gpu_instance_upload_many(g, np, subp.data(), dinst.data()));
    if (mode == TAMC_MODE_REF) {
      // one master stream, cloned then jumped per sub-instance (src/gla.rs:144-151);
      // each clone draws its initial replicas, then runs the loop
      Xo master = xo_seed_from_u64(seed);
      for (uint32_t k = 0; k < np; ++k) {
        const Xo rk = master;
        xo_jump(master);
        tamc_pt* pt = pt_create_ref_stream(dinst[k], &q, rk);
        try {
          check_rc(tamc_gpu_pt_run(pt, q.num_sweeps));
          check_rc(tamc_gpu_pt_sync(pt));
          last_ground_state(pt, (uint32_t)sorted[k].size(), part_e[k], part_s[k]);
        } catch (...) {
          tamc_gpu_pt_destroy(pt);
          throw;
        }
        tamc_gpu_pt_destroy(pt);
      }
    } else {
      // colour order: every sub-instance is a job of one batch
      tamc_batch* b = nullptr;
      check_rc(tamc_gpu_batch_create(g, &b));
      try {
        uint64_t st = seed;
        for (uint32_t k = 0; k < np; ++k) check_rc(tamc_gpu_batch_add(b, dinst[k], &q, splitmix_next(st), nullptr));
        check_rc(tamc_gpu_batch_run(b));
        check_rc(tamc_gpu_batch_sync(b));
        for (uint32_t k = 0; k < np; ++k) {
          uint32_t cnt = 0;
          check_rc(tamc_gpu_batch_gs(b, k, 0, &cnt, nullptr, nullptr, nullptr));
          if (!cnt) fail(TAMC_E_REFPANIC, "a sub-instance run recorded no ground state (the reference panics)");
          const uint32_t nk = (uint32_t)sorted[k].size(), nw = (nk + 63) / 64;
          std::vector<uint32_t> steps(cnt);
          std::vector<float> en(cnt);
          std::vector<uint64_t> words((size_t)cnt * nw);
          check_rc(tamc_gpu_batch_gs(b, k, cnt, &cnt, steps.data(), en.data(), words.data()));
          part_e[k] = en[cnt - 1];
          part_s[k].assign(nk, 1);
          const uint64_t* w = words.data() + (size_t)(cnt - 1) * nw;
          for (uint32_t i = 0; i < nk; ++i) part_s[k][i] = ((w[i / 64] >> (i % 64)) & 1u) ? -1 : 1;
        }
      } catch (...) {
        tamc_gpu_batch_destroy(b);
        throw;
      }
      tamc_gpu_batch_destroy(b);
    }
  } catch (...) {
    release();
    throw;
  }
  release();
  // join (src/gla.rs:167-188): bulk = sum of the partitions' energies, each
  // boundary edge group sums K * (s_i * s_j) in f32 in its edge order
  auto* r = new tamc_gla();
  r->r.instance_size = n;
  r->r.num_partitions = np;
  r->r.partition_energies = part_e;
  float bulk = 0.0f;
  for (float e : part_e) bulk += e;
  float total_bnd = 0.0f;
  for (size_t x = 0; x < bkeys.size(); ++x) {
    const uint32_t a = bkeys[x].first, b = bkeys[x].second;
    float bnd = 0.0f;
    for (const Edge& e : bedges[x]) {
      const size_t is = std::lower_bound(sorted[a].begin(), sorted[a].end(), e.i) - sorted[a].begin();
      const size_t js = std::lower_bound(sorted[b].begin(), sorted[b].end(), e.j) - sorted[b].begin();
      const float prod = (float)(int)(part_s[a][is] * part_s[b][js]);
      bnd += e.K * prod;
    }
    total_bnd += bnd;
    r->r.bnd_src.push_back(a);
    r->r.bnd_dst.push_back(b);
    r->r.bnd_energies.push_back(bnd);
  }
  r->r.total_energy = bulk + total_bnd;
  r->joined.assign(n, 1);
  for (uint32_t k = 0; k < np; ++k)
    for (size_t x = 0; x < sorted[k].size(); ++x) r->joined[sorted[k][x]] = part_s[k][x];
  *out = r;
  TAMC_API_END
}

int tamc_gla_dims(const tamc_gla* r, uint32_t* instance_size, uint32_t* num_partitions, uint32_t* num_boundaries) {
  TAMC_API_BEGIN
  if (!r) fail(TAMC_E_INVAL, "null result");
  if (instance_size) *instance_size = r->r.instance_size;
  if (num_partitions) *num_partitions = r->r.num_partitions;
  if (num_boundaries) *num_boundaries = (uint32_t)r->r.bnd_energies.size();
  TAMC_API_END
}

int tamc_gla_results(const tamc_gla* r, float* partition_energies, uint32_t* bnd_src, uint32_t* bnd_dst,
                     float* bnd_energies, float* total_energy) {
  TAMC_API_BEGIN
  if (!r) fail(TAMC_E_INVAL, "null result");
  const auto& x = r->r;
  if (partition_energies) std::copy(x.partition_energies.begin(), x.partition_energies.end(), partition_energies);
  if (bnd_src) std::copy(x.bnd_src.begin(), x.bnd_src.end(), bnd_src);
  if (bnd_dst) std::copy(x.bnd_dst.begin(), x.bnd_dst.end(), bnd_dst);
  if (bnd_energies) std::copy(x.bnd_energies.begin(), x.bnd_energies.end(), bnd_energies);
  if (total_energy) *total_energy = x.total_energy;
  TAMC_API_END
}

int tamc_gla_state(const tamc_gla* r, int8_t* spins) {
  TAMC_API_BEGIN
  if (!r || !spins) fail(TAMC_E_INVAL, "null argument");
  std::copy(r->joined.begin(), r->joined.end(), spins);
  TAMC_API_END
}

int tamc_gla_write(const tamc_gla* r, const char* path) {
  TAMC_API_BEGIN
  if (!r || !path) fail(TAMC_E_INVAL, "null argument");
  // write_data (src/util.rs:26-36): pickle for a .pkl extension, else bincode
  const std::string ps(path);
  const size_t slash = ps.find_last_of('/');
  const std::string base = slash == std::string::npos ? ps : ps.substr(slash + 1);
  const size_t dot = base.find_last_of('.');
  const bool pkl = dot != std::string::npos && dot != 0 && base.substr(dot + 1) == "pkl";
  const std::string data = pkl ? pickle_gla_results(r->r) : bincode_gla_results(r->r);
  std::ofstream f(path, std::ios::binary);
  if (!f) fail(TAMC_E_IO, "Failed to write GLA data to " + ps);
  f.write(data.data(), (std::streamsize)data.size());
  if (!f) fail(TAMC_E_IO, "Failed to write GLA data to " + ps);
  TAMC_API_END
}

void tamc_gla_free(tamc_gla* r) { delete r; }

}  // extern "C"
