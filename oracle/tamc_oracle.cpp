// tamc_oracle.cpp -- TEST INFRASTRUCTURE ONLY (the checker, never the product).
//
// A plain C++ CPU restatement of the reference's Monte-Carlo hot path
// (USCqserver/tamc), used by the tests as the parity oracle and by bench.py as
// the timed CPU baseline ("CPU restatement of reference").  Nothing in the
// product library links, loads or calls this file.
//
// PARITY UNPINNED: the reference is Rust and cannot be compiled in this
// environment (no cargo/rustc, crates not vendored), and its own tests assert
// nothing (no golden vectors, no fixtures).  This restatement therefore follows
// the reference source line by line (citations below) and the published
// algorithms of the third-party crates it calls:
//   * rand_xoshiro 0.6  Xoshiro256PlusPlus (Blackman & Vigna 2018): next(),
//     jump() with the published 2^128 jump polynomial, seed_from_u64 via a
//     SplitMix64 fill of the 32-byte seed (little-endian words);
//   * rand 0.8  next_u32 = upper 32 bits of next_u64; Standard f32 =
//     (next_u32 >> 8) * 2^-24; Uniform::new_inclusive(0i8, 1) = top bit of
//     next_u32; SliceRandom::choose = gen_range(0..len as u32) by widening
//     multiply with rejection zone (len << lz(len)) - 1;
//   * glibc 2.39 expf / exp / log (Rust's f32::exp and f64::exp/ln call libm);
//   * petgraph 0.6 Csr::from_sorted_edges + Bfs over NodeFiltered (only the
//     discovered set is used, so BFS order does not matter).
//
// Reference files cited as path:line within the reference project.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace orc {

// ---------------------------------------------------------------- RNG ----
// SplitMix64 (Steele, Lea, Flood 2014; Vigna's public-domain form).
static inline uint64_t splitmix64_next(uint64_t& st) {
  st += 0x9e3779b97f4a7c15ULL;
  uint64_t z = st;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

static inline uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

struct Xoshiro {
  uint64_t s[4];
  // Xoshiro256++ next (Blackman & Vigna 2018).
  inline uint64_t next() {
    const uint64_t result = rotl(s[0] + s[3], 23) + s[0];
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl(s[3], 45);
    return result;
  }
  inline uint32_t next_u32() { return (uint32_t)(next() >> 32); }
  // 2^128 jump (published polynomial).
  void jump() {
    static const uint64_t J[4] = {0x180ec6d33cfd0abaULL, 0xd5a61266f0c9392cULL,
                                  0xa9582618e03fc9aaULL, 0x39abdc4529b1661cULL};
    uint64_t t0 = 0, t1 = 0, t2 = 0, t3 = 0;
    for (int i = 0; i < 4; ++i)
      for (int b = 0; b < 64; ++b) {
        if (J[i] & (1ULL << b)) { t0 ^= s[0]; t1 ^= s[1]; t2 ^= s[2]; t3 ^= s[3]; }
        next();
      }
    s[0] = t0; s[1] = t1; s[2] = t2; s[3] = t3;
  }
};

// Xoshiro256PlusPlus::seed_from_u64 (rand_xoshiro: SplitMix64 fills the seed).
static Xoshiro seed_from_u64(uint64_t seed) {
  Xoshiro x;
  uint64_t st = seed;
  for (int i = 0; i < 4; ++i) x.s[i] = splitmix64_next(st);
  if (!(x.s[0] | x.s[1] | x.s[2] | x.s[3])) return seed_from_u64(0);
  return x;
}

// rand 0.8 Standard for f32: 24 random bits scaled by 2^-24.
static inline float std_f32(Xoshiro& r) {
  return (float)(r.next_u32() >> 8) * (1.0f / 16777216.0f);
}
// 2*Uniform::new_inclusive(0i8,1) - 1   (reference src/ising.rs:172)
static inline int8_t rand_spin(Xoshiro& r) { return (r.next_u32() >> 31) ? 1 : -1; }
// gen_range(0..range) for u32, range > 0 (rand 0.8 UniformInt::sample_single).
static inline uint32_t gen_range_u32(Xoshiro& r, uint32_t range) {
  const uint32_t zone = (range << __builtin_clz(range)) - 1u;
  for (;;) {
    const uint32_t v = r.next_u32();
    const uint64_t m = (uint64_t)v * (uint64_t)range;
    if ((uint32_t)m <= zone) return (uint32_t)(m >> 32);
  }
}

// ----------------------------------------------------------- instance ----
struct Instance {
  uint32_t n = 0;
  float offset = 0.0f;
  std::vector<float> bias;
  // coupling_vecs as CSR rows in BTreeMap (sorted j) order, incl. the QUBO
  // self-loop quirk (reference src/ising.rs:286-324).
  std::vector<uint32_t> row_ptr, col;
  std::vector<float> K;
  // ICM graph: the off-diagonal pattern of the sprs `coupling` matrix, as
  // petgraph Csr::from_sorted_edges builds it (src/pt.rs:343-346).  Its node
  // count is (largest endpoint + 1), which can be smaller than n.
  uint32_t g_nodes = 0;
  std::vector<uint32_t> g_row_ptr, g_col;
  std::vector<std::vector<double>> suscept;  // src/ising.rs:388-403
};

// diag: the sprs `coupling` matrix also holds the diagonal entries, as in the
// sub-instances GLA builds (src/ising.rs:327-355: every kept row entry goes
// into the triplet matrix); self-loops only extend the node range.
static void build_icm_graph(Instance& I, bool diag = false) {
  uint32_t maxn = 0;
  bool any = false;
  for (uint32_t i = 0; i < I.n; ++i)
    for (uint32_t e = I.row_ptr[i]; e < I.row_ptr[i + 1]; ++e)
      if (I.col[e] != i || diag) { any = true; maxn = std::max(maxn, std::max(i, I.col[e])); }
  I.g_nodes = any ? maxn + 1 : 0;
  I.g_row_ptr.assign(I.g_nodes + 1, 0);
  I.g_col.clear();
  for (uint32_t i = 0; i < I.g_nodes; ++i) {
    for (uint32_t e = I.row_ptr[i]; e < I.row_ptr[i + 1]; ++e)
      if (I.col[e] != i) I.g_col.push_back(I.col[e]);
    I.g_row_ptr[i + 1] = (uint32_t)I.g_col.size();
  }
}

// nom parser of one `i j K` line (reference src/util.rs:38-63).  Returns false
// when the reference would print "Ignoring line".  Trailing text after the
// fixed-point number is ignored, exactly as the reference ignores the
// unconsumed remainder.
static bool parse_digits_u32(const char*& p, const char* end, uint32_t& out, bool& overflow) {
  const char* s = p;
  uint64_t v = 0;
  overflow = false;
  while (p < end && *p >= '0' && *p <= '9') {
    v = v * 10 + (uint64_t)(*p - '0');
    if (v > 0xffffffffULL) overflow = true;
    ++p;
  }
  out = (uint32_t)v;
  return p > s;
}
static inline bool is_sp(char c) { return c == ' ' || c == '\t'; }

static int parse_line(const char* p, const char* end, uint32_t& i, uint32_t& j, double& k) {
  uint32_t ints[2];
  for (int t = 0; t < 2; ++t) {
    while (p < end && is_sp(*p)) ++p;                // space0
    bool ovf;
    if (!parse_digits_u32(p, end, ints[t], ovf)) return 0;
    if (ovf) return -1;                              // u32::from_str(..).unwrap() panics
    const char* s = p;
    while (p < end && is_sp(*p)) ++p;                // space1
    if (p == s) return 0;
  }
  const char* s = p;
  if (p < end && *p == '-') ++p;
  const char* d0 = p;
  while (p < end && *p >= '0' && *p <= '9') ++p;
  if (p == d0) return 0;                            // digit1
  if (p < end && *p == '.') {
    ++p;
    while (p < end && *p >= '0' && *p <= '9') ++p;
  }
  std::string num(s, p);
  k = strtod(num.c_str(), nullptr);                 // correctly rounded, as Rust's parse
  i = ints[0];
  j = ints[1];
  return 1;
}

// read_adjacency_list (src/util.rs:76-109) + from_instance_file (src/ising.rs:286-324).
static int instance_from_text(const char* text, size_t len, bool qubo, Instance& I, std::string& err) {
  std::vector<std::map<uint32_t, float>> adj;
  const char* p = text;
  const char* end = text + len;
  while (p < end) {
    const char* e = (const char*)memchr(p, '\n', (size_t)(end - p));
    const char* le = e ? e : end;
    const char* lend = le;
    if (lend > p && lend[-1] == '\r') --lend;  // BufRead::lines strips "\r\n"
    uint32_t i, j;
    double k;
    int r = parse_line(p, lend, i, j, k);
    if (r < 0) { err = "integer overflow in instance line"; return -1; }
    if (r > 0) {
      size_t m = (size_t)std::max(i, j) + 1;
      if (adj.size() < m) adj.resize(m);
      adj[i][j] = (float)k;
      if (i != j) adj[j][i] = (float)k;
    }
    p = e ? e + 1 : end;
  }
  const uint32_t n = (uint32_t)adj.size();
  I = Instance();
  I.n = n;
  I.bias.assign(n, 0.0f);
  I.row_ptr.assign(n + 1, 0);
  float offset = 0.0f;
  for (uint32_t i = 0; i < n; ++i) {
    for (const auto& kv : adj[i]) {
      const uint32_t j = kv.first;
      const float K = kv.second;
      if (qubo) {
        if (i != j) {
          offset += K / 8.0f;
          I.col.push_back(j); I.K.push_back(K / 4.0f);
          I.bias[i] += K / 4.0f;
        } else {
          offset += K / 2.0f;
          I.bias[i] += K / 2.0f;
          I.col.push_back(j); I.K.push_back(K / 2.0f);
        }
      } else {
        if (i != j) { I.col.push_back(j); I.K.push_back(K); }
        else I.bias[i] = K;
      }
    }
    I.row_ptr[i + 1] = (uint32_t)I.col.size();
  }
  I.offset = offset;
  build_icm_graph(I);
  return 0;
}

// energy_ref (src/ising.rs:438-454): f32, rows in order.
static float energy_ref(const Instance& I, const int8_t* s) {
  float total = I.offset;
  for (uint32_t i = 0; i < I.n; ++i) {
    float h = 0.0f;
    const float si = (float)s[i];
    h += I.bias[i];
    for (uint32_t e = I.row_ptr[i]; e < I.row_ptr[i + 1]; ++e) {
      const float sj = (float)s[I.col[e]];
      h += (I.K[e] * sj) / 2.0f;
    }
    total += h * si;
  }
  return total;
}
static double energy_f64(const Instance& I, const int8_t* s) {
  double total = I.offset;
  for (uint32_t i = 0; i < I.n; ++i) {
    double h = I.bias[i];
    for (uint32_t e = I.row_ptr[i]; e < I.row_ptr[i + 1]; ++e)
      h += (double)I.K[e] * (double)s[I.col[e]] * 0.5;
    total += h * (double)s[i];
  }
  return total;
}
// delta_energy (src/ising.rs:468-480).
static inline float delta_energy(const Instance& I, const int8_t* s, uint32_t i) {
  float de = 0.0f;
  de += I.bias[i];
  for (uint32_t e = I.row_ptr[i]; e < I.row_ptr[i + 1]; ++e) de += I.K[e] * (float)s[I.col[e]];
  const float si = (float)s[i];
  de *= -2.0f * si;
  return de;
}

struct IsingState {
  std::vector<int8_t> arr;
  float energy = 0.0f;
  bool energy_init = false;
};

static inline float energy_cached(const Instance& I, IsingState& st) {  // src/ising.rs:455-463
  if (st.energy_init) return st.energy;
  st.energy = energy_ref(I, st.arr.data());
  st.energy_init = true;
  return st.energy;
}

// MetropolisSampler::advance_impl (tamc-core/src/metropolis.rs:43-57).
// Returns true and sets de when the move is accepted.
static inline bool advance_impl(const Instance& I, float beta, int8_t* s, uint32_t i, Xoshiro& rng, float& de) {
  const float d = delta_energy(I, s, i);
  if (d < 0.0f) { s[i] = (int8_t)-s[i]; de = d; return true; }
  const float p = expf(-beta * d);
  const float x = std_f32(rng);
  if (x < p) { s[i] = (int8_t)-s[i]; de = d; return true; }
  return false;
}
// IsingSampler::sweep (src/ising.rs:225-233).
static void ising_sweep(const Instance& I, float beta, IsingState& st, Xoshiro& rng) {
  float de = 0.0f;
  int8_t* s = st.arr.data();
  for (uint32_t i = 0; i < I.n; ++i) {
    float d;
    de += advance_impl(I, beta, s, i, rng, d) ? d : 0.0f;
  }
  st.energy += de;
}
// MetropolisSampler::sweep (tamc-core/src/metropolis.rs:77-83), no energy tracking.
static void plain_sweep(const Instance& I, float beta, int8_t* s, Xoshiro& rng) {
  for (uint32_t i = 0; i < I.n; ++i) { float d; advance_impl(I, beta, s, i, rng, d); }
}
// rand_ising_state (src/ising.rs:168-177).
static IsingState rand_state(const Instance& I, Xoshiro& rng) {
  IsingState st;
  st.arr.resize(I.n);
  for (uint32_t i = 0; i < I.n; ++i) st.arr[i] = rand_spin(rng);
  energy_cached(I, st);
  return st;
}

// ----------------------------------------------------------------- PT ----
enum Tag : uint8_t { T_NONE = 0, T_MIN = 1, T_MAX = 2, T_MIN_REFL = 3, T_MAX_REFL = 4 };

struct PTState {  // tamc-core/src/pt.rs:18-25
  std::vector<IsingState> states;
  std::vector<uint32_t> num_acceptances;
  uint32_t round_trips = 0;
  std::vector<uint8_t> tags;
  std::vector<uint32_t> diffusion_hist;  // [n][2]
  explicit PTState(std::vector<IsingState> st) : states(std::move(st)) {
    const size_t n = states.size();
    num_acceptances.assign(n, 0);
    diffusion_hist.assign(2 * n, 0);
    tags.assign(n, T_NONE);
    tags[0] = T_MIN;
    tags[n - 1] = T_MAX;
  }
  void swap_states(size_t j) {  // pt.rs:49-53
    std::swap(states[j], states[j + 1]);
    std::swap(tags[j], tags[j + 1]);
    num_acceptances[j] += 1;
  }
  void update_round_trips() {  // pt.rs:54-84
    uint8_t& lo = tags[0];
    switch (lo) {
      case T_NONE: lo = T_MIN; break;
      case T_MAX_REFL: round_trips += 1; lo = T_MIN; break;
      case T_MAX: lo = T_MIN_REFL; break;
      default: break;
    }
    uint8_t& hi = tags.back();
    switch (hi) {
      case T_NONE: hi = T_MAX; break;
      case T_MIN_REFL: round_trips += 1; hi = T_MAX; break;
      case T_MIN: hi = T_MAX_REFL; break;
      default: break;
    }
    for (size_t k = 0; k < tags.size(); ++k) {
      if (tags[k] == T_MIN || tags[k] == T_MIN_REFL) diffusion_hist[2 * k] += 1;
      else if (tags[k] == T_MAX || tags[k] == T_MAX_REFL) diffusion_hist[2 * k + 1] += 1;
    }
  }
};

struct PtParams {
  uint32_t num_sweeps;
  double warmup_fraction;
  std::vector<float> betas;
  uint32_t lo_beta_idx;
  bool icm;
  uint32_t num_chains;
  uint32_t threads;
  int64_t sample;          // -1 = None
  int64_t sample_states;   // -1 = None
  uint8_t sample_limiting;
};

struct GsEntry { uint32_t step; float energy; std::vector<uint64_t> state; };

struct PtRun {
  const Instance* I;
  PtParams P;
  std::vector<float> delta_beta;
  uint32_t meas_init;
  std::vector<PTState> pt;
  Xoshiro rng;                            // serial mode
  std::vector<std::vector<Xoshiro>> rngs; // threaded mode [chain][slot]
  bool threaded;
  // results
  bool have_min = false;
  float minimum_e = 0.0f;
  std::vector<GsEntry> gs;
  std::vector<std::vector<float>> e;                       // [nt][..]
  std::vector<std::vector<int32_t>> q;                     // [nt][..]
  std::vector<std::vector<std::vector<float>>> sus;        // [nt][nchi][..]
  std::vector<std::vector<std::vector<uint8_t>>> samples;  // [slots][..][bytes]
  uint32_t next_sweep = 0;
  std::string err;
  // ICM cluster sizes of the most recent round (diagnostics), -1 = no move
  std::vector<int64_t> last_icm;
};

// houdayer_cluster_move (src/pt.rs:31-77).  Returns -1 if no site has q<0,
// -2 where the reference would panic (seed outside the petgraph node range),
// else the cluster size.
static int64_t houdayer(const Instance& I, IsingState& r1, IsingState& r2, Xoshiro& rng,
                        std::vector<uint32_t>& idxs, std::vector<uint8_t>& disc,
                        std::vector<uint32_t>& queue) {
  const uint32_t n = (uint32_t)r1.arr.size();
  idxs.clear();
  for (uint32_t i = 0; i < n; ++i)
    if (r1.arr[i] * r2.arr[i] < 0) idxs.push_back(i);
  if (idxs.empty()) return -1;
  const uint32_t init = idxs[gen_range_u32(rng, (uint32_t)idxs.size())];
  if (init >= I.g_nodes) return -2;
  disc.assign(I.g_nodes, 0);
  queue.clear();
  queue.push_back(init);
  disc[init] = 1;
  for (size_t h = 0; h < queue.size(); ++h) {
    const uint32_t u = queue[h];
    for (uint32_t e = I.g_row_ptr[u]; e < I.g_row_ptr[u + 1]; ++e) {
      const uint32_t v = I.g_col[e];
      if (!disc[v] && r1.arr[v] * r2.arr[v] < 0) { disc[v] = 1; queue.push_back(v); }
    }
  }
  for (uint32_t v : queue) std::swap(r1.arr[v], r2.arr[v]);
  r1.energy_init = false;
  r2.energy_init = false;
  return (int64_t)queue.size();
}

static int apply_icm(PtRun& R, Xoshiro& rng) {  // src/pt.rs:521-540
  R.last_icm.clear();
  if (!R.P.icm) return 0;
  std::vector<uint32_t> idxs, queue;
  std::vector<uint8_t> disc;
  const size_t nt = R.P.betas.size();
  for (size_t c = 0; c + 1 < R.pt.size(); c += 2) {
    for (size_t t = R.P.lo_beta_idx; t < nt; ++t) {
      int64_t r = houdayer(*R.I, R.pt[c].states[t], R.pt[c + 1].states[t], rng, idxs, disc, queue);
      if (r == -2) { R.err = "ICM seed site outside the coupling graph (reference panics)"; return -1; }
      R.last_icm.push_back(r);
    }
  }
  return 0;
}

// ParallelTemperingSampler::advance exchange part (tamc-core/src/pt.rs:120-132)
static void exchange_serial(PtRun& R, PTState& st, Xoshiro& rng) {
  const size_t n = st.states.size();
  std::vector<float> en(n), des(n - 1);
  for (size_t k = 0; k < n; ++k) en[k] = energy_cached(*R.I, st.states[k]);
  for (size_t k = 0; k + 1 < n; ++k) des[k] = en[k + 1] - en[k];
  for (size_t j = 0; j + 1 < n; ++j) {
    const float dlt = R.delta_beta[j] * des[j];
    if (dlt >= 0.0f || std_f32(rng) < expf(dlt)) {
      st.swap_states(j);
      if (j + 2 < n) des[j + 1] = des[j + 1] + des[j];
      des[j] = -des[j];
    }
  }
  st.update_round_trips();
}
// ThreadedPTSampler::advance exchange part (tamc-core/src/parallel/pt.rs:41-59)
static void exchange_threaded(PtRun& R, PTState& st, Xoshiro& rng) {
  const size_t n = st.states.size();
  std::vector<float> en(n), des(n - 1);
  for (size_t k = 0; k < n; ++k) en[k] = energy_cached(*R.I, st.states[k]);
  for (size_t k = 0; k + 1 < n; ++k) des[k] = en[k + 1] - en[k];
  for (size_t j = 0; j + 1 < n; ++j) {
    const float dlt = R.delta_beta[j] * des[j];
    if (dlt >= 0.0f || std_f32(rng) < expf(dlt)) st.swap_states(j);
  }
  st.update_round_trips();
}

static void write_to_bytes(const IsingState& s, std::vector<uint8_t>& b) {  // src/ising.rs:102-115
  const size_t n = s.arr.size();
  b.assign(n / 8 + (n % 8 ? 1 : 0), 0);
  for (size_t i = 0; i < n; ++i) if (!(s.arr[i] > 0)) b[i / 8] |= (uint8_t)(1u << (i % 8));
}
static std::vector<uint64_t> as_u64_vec(const IsingState& s) {  // src/ising.rs:123-137
  const size_t n = s.arr.size();
  std::vector<uint64_t> w(n / 64 + (n % 64 ? 1 : 0), 0);
  for (size_t i = 0; i < n; ++i) if (!(s.arr[i] > 0)) w[i / 64] |= (1ULL << (i % 64));
  return w;
}

static void measure(PtRun& R) {  // src/pt.rs:167-201
  const size_t nc = R.pt.size(), nb = R.pt[0].states.size();
  const size_t n = R.I->n;
  const size_t nchi = R.I->suscept.size();
  std::vector<int8_t> ov(nchi ? n : 0);
  for (size_t i = 0; i < nb; ++i) {
    for (size_t j = 0; j < nc; ++j) R.e[i].push_back(energy_cached(*R.I, R.pt[j].states[i]));
    for (size_t j = 0; j < nc / 2; ++j) {
      const auto& a = R.pt[2 * j].states[i].arr;
      const auto& b = R.pt[2 * j + 1].states[i].arr;
      if (nchi > 0) {
        for (size_t k = 0; k < n; ++k) ov[k] = (int8_t)(a[k] * b[k]);
        for (size_t k = 0; k < nchi; ++k) {
          double chi = 0.0;
          const auto& w = R.I->suscept[k];
          for (size_t s = 0; s < n; ++s) chi += w[s] * (double)ov[s];
          R.sus[i][k].push_back((float)chi);
        }
      }
      int64_t q = 0;
      for (size_t k = 0; k < n; ++k) q += (int64_t)(a[k] * b[k]);
      R.q[i].push_back((int32_t)q);
    }
  }
}
static void sample_states(PtRun& R) {  // src/pt.rs:202-226
  const size_t nc = R.pt.size(), nb = R.pt[0].states.size();
  std::vector<uint8_t> b;
  if (R.P.sample_limiting == 0) {
    for (size_t i = 0; i < nb; ++i)
      for (size_t j = 0; j < nc; ++j) { write_to_bytes(R.pt[j].states[i], b); R.samples[i].push_back(b); }
  } else if (R.P.sample_limiting == 1) {
    for (size_t i = 0; i < nb / 2; ++i) {
      const size_t is = nb - i - 1;
      for (size_t j = 0; j < nc; ++j) { write_to_bytes(R.pt[j].states[is], b); R.samples[i].push_back(b); }
    }
  } else {
    for (size_t j = 0; j < nc; ++j) { write_to_bytes(R.pt[j].states[nb - 1], b); R.samples[0].push_back(b); }
  }
}
static void apply_measurements(PtRun& R, uint32_t i) {  // src/pt.rs:542-583
  if (i < R.meas_init) return;
  const uint32_t stp = i - R.meas_init;
  if (R.P.sample >= 0 && (stp % (uint32_t)R.P.sample == 0 || i == R.P.num_sweeps - 1)) measure(R);
  if (R.P.sample_states >= 0 && (stp % (uint32_t)R.P.sample_states == 0 || i == R.P.num_sweeps - 1))
    sample_states(R);
  size_t best_c = 0, best_t = 0;
  float best_e = 0.0f;
  for (size_t c = 0; c < R.pt.size(); ++c) {
    size_t i1 = 0;
    float e1 = energy_cached(*R.I, R.pt[c].states[0]);
    for (size_t t = 1; t < R.pt[c].states.size(); ++t) {
      const float e = energy_cached(*R.I, R.pt[c].states[t]);
      if (e < e1) { e1 = e; i1 = t; }
    }
    if (c == 0 || e1 < best_e) { best_e = e1; best_c = c; best_t = i1; }
  }
  if (!R.have_min || best_e < R.minimum_e) {
    R.have_min = true;
    R.minimum_e = best_e;
    R.gs.push_back(GsEntry{i, best_e, as_u64_vec(R.pt[best_c].states[best_t])});
  }
}

}  // namespace orc

// ================================================================ C API ====
using namespace orc;

extern "C" {

// -- RNG known-answer helpers
void orc_splitmix64(uint64_t seed, uint64_t* out, uint32_t n) {
  uint64_t st = seed;
  for (uint32_t i = 0; i < n; ++i) out[i] = splitmix64_next(st);
}
void orc_xoshiro_seed(uint64_t seed, uint64_t* s4) {
  Xoshiro x = seed_from_u64(seed);
  memcpy(s4, x.s, 32);
}
void orc_xoshiro_next(uint64_t* s4, uint64_t* out, uint32_t n) {
  Xoshiro x;
  memcpy(x.s, s4, 32);
  for (uint32_t i = 0; i < n; ++i) out[i] = x.next();
  memcpy(s4, x.s, 32);
}
void orc_xoshiro_jump(uint64_t* s4) {
  Xoshiro x;
  memcpy(x.s, s4, 32);
  x.jump();
  memcpy(s4, x.s, 32);
}
void orc_gen_range(uint64_t* s4, uint32_t range, uint32_t* out, uint32_t n) {
  Xoshiro x;
  memcpy(x.s, s4, 32);
  for (uint32_t i = 0; i < n; ++i) out[i] = gen_range_u32(x, range);
  memcpy(s4, x.s, 32);
}
float orc_expf(float x) { return expf(x); }

// -- beta ladders: BetaOptions::get_beta_arr (src/pt.rs:246-256) with
// geometric_beta_schedule (tamc-core/src/sa.rs:13-22).
void orc_geometric_betas(float beta_min, float beta_max, uint32_t n, float* out) {
  const double lb0 = log((double)beta_min), lbf = log((double)beta_max);
  const double d = (lbf - lb0) / (double)(n - 1);
  for (uint32_t i = 0; i < n; ++i) out[i] = (float)exp(lb0 + d * (double)i);
}
// lo_beta_idx (src/pt.rs:316-341): lo_num_beta wins over lo_beta.
uint32_t orc_lo_beta_idx(const float* betas, uint32_t nb, int has_lo_num, uint32_t lo_num, int has_lo_beta, float lo_beta) {
  if (has_lo_num) { uint32_t l = lo_num < nb ? lo_num : nb; return nb - l; }
  if (has_lo_beta) {
    for (uint32_t i = 0; i < nb; ++i) if (betas[i] >= lo_beta) return i;
    return nb - 1;
  }
  return 0;
}

// -- instances
void* orc_inst_from_text(const char* text, uint64_t len, int qubo, char* err, uint64_t errlen) {
  Instance* I = new Instance();
  std::string e;
  if (instance_from_text(text, (size_t)len, qubo != 0, *I, e) != 0) {
    if (err && errlen) snprintf(err, (size_t)errlen, "%s", e.c_str());
    delete I;
    return nullptr;
  }
  return I;
}
void* orc_inst_from_csr(uint32_t n, const uint32_t* row_ptr, const uint32_t* col, const float* K,
                        const float* bias, float offset) {
  Instance* I = new Instance();
  I->n = n;
  I->offset = offset;
  I->bias.assign(bias, bias + n);
  I->row_ptr.assign(row_ptr, row_ptr + n + 1);
  I->col.assign(col, col + row_ptr[n]);
  I->K.assign(K, K + row_ptr[n]);
  build_icm_graph(*I);
  return I;
}
int orc_inst_add_suscept(void* h, const double* w, uint32_t n) {
  Instance* I = (Instance*)h;
  I->suscept.emplace_back(w, w + n);
  return 0;
}
void orc_inst_free(void* h) { delete (Instance*)h; }
uint32_t orc_inst_n(const void* h) { return ((const Instance*)h)->n; }
uint64_t orc_inst_nnz(const void* h) { return ((const Instance*)h)->col.size(); }
float orc_inst_offset(const void* h) { return ((const Instance*)h)->offset; }
uint32_t orc_inst_graph_nodes(const void* h) { return ((const Instance*)h)->g_nodes; }
void orc_inst_csr(const void* h, uint32_t* row_ptr, uint32_t* col, float* K, float* bias) {
  const Instance* I = (const Instance*)h;
  memcpy(row_ptr, I->row_ptr.data(), (I->n + 1) * 4);
  memcpy(col, I->col.data(), I->col.size() * 4);
  memcpy(K, I->K.data(), I->K.size() * 4);
  memcpy(bias, I->bias.data(), I->n * 4);
}
float orc_energy_ref(const void* h, const int8_t* s) { return energy_ref(*(const Instance*)h, s); }
double orc_energy_f64(const void* h, const int8_t* s) { return energy_f64(*(const Instance*)h, s); }
float orc_delta_energy(const void* h, const int8_t* s, uint32_t i) { return delta_energy(*(const Instance*)h, s, i); }

// -- PT-ICM runner (PtIcmRunner::run / run_parallel, src/pt.rs:354-412).
// sample/sample_states < 0 mean None.
static PtRun* pt_make(const void* inst, uint32_t num_sweeps, double warmup_fraction, const float* betas,
                      uint32_t nb, uint32_t lo_beta_idx, int icm, uint32_t num_chains, uint32_t threads,
                      int64_t sample, int64_t sample_states, uint32_t sample_limiting, Xoshiro master) {
  PtRun* R = new PtRun();
  R->I = (const Instance*)inst;
  R->P.num_sweeps = num_sweeps;
  R->P.warmup_fraction = warmup_fraction;
  R->P.betas.assign(betas, betas + nb);
  R->P.lo_beta_idx = lo_beta_idx;
  R->P.icm = icm != 0;
  R->P.num_chains = num_chains;
  R->P.threads = threads;
  R->P.sample = sample;
  R->P.sample_states = sample_states;
  R->P.sample_limiting = (uint8_t)sample_limiting;
  R->threaded = threads > 1;
  for (uint32_t k = 0; k + 1 < nb; ++k) R->delta_beta.push_back(betas[k + 1] - betas[k]);
  const double mi = warmup_fraction * (double)num_sweeps;
  R->meas_init = mi <= 0.0 ? 0u : (mi >= 4294967295.0 ? 0xffffffffu : (uint32_t)mi);
  R->rng = master;
  for (uint32_t c = 0; c < num_chains; ++c) {  // generate_init_state (src/pt.rs:506-519)
    std::vector<IsingState> st;
    for (uint32_t t = 0; t < nb; ++t) st.push_back(rand_state(*R->I, R->rng));
    R->pt.emplace_back(std::move(st));
  }
  if (R->threaded) {  // src/pt.rs:365-373
    R->rngs.resize(num_chains);
    for (uint32_t c = 0; c < num_chains; ++c)
      for (uint32_t t = 0; t < nb; ++t) { R->rngs[c].push_back(R->rng); R->rng.jump(); }
  }
  const size_t nchi = R->I->suscept.size();
  R->e.resize(nb); R->q.resize(nb);
  R->sus.assign(nb, std::vector<std::vector<float>>(nchi));
  if (R->P.sample_limiting == 0) R->samples.resize(nb);
  else if (R->P.sample_limiting == 1) R->samples.resize(nb / 2);
  else R->samples.resize(1);
  return R;
}
void* orc_pt_new(const void* inst, uint32_t num_sweeps, double warmup_fraction, const float* betas,
                 uint32_t nb, uint32_t lo_beta_idx, int icm, uint32_t num_chains, uint32_t threads,
                 int64_t sample, int64_t sample_states, uint32_t sample_limiting, uint64_t seed) {
  return pt_make(inst, num_sweeps, warmup_fraction, betas, nb, lo_beta_idx, icm, num_chains, threads, sample,
                 sample_states, sample_limiting, seed_from_u64(seed));
}
void orc_pt_free(void* h) { delete (PtRun*)h; }
const char* orc_pt_error(void* h) { return ((PtRun*)h)->err.c_str(); }

// Runs sweeps [next, end): pt_loop (src/pt.rs:459-504) or parallel_pt_loop (:414-457).
int orc_pt_run(void* h, uint32_t end, int nthreads) {
  PtRun& R = *(PtRun*)h;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif
  const uint32_t nb = (uint32_t)R.P.betas.size();
  const uint32_t nc = (uint32_t)R.pt.size();
  for (uint32_t i = R.next_sweep; i < end; ++i) {
    if (!R.threaded) {
      if (apply_icm(R, R.rng)) return -1;
      for (uint32_t c = 0; c < nc; ++c) {  // EnsembleSampler (tamc-core/src/ensembles.rs:20-28)
        exchange_serial(R, R.pt[c], R.rng);
        for (uint32_t t = 0; t < nb; ++t) ising_sweep(*R.I, R.P.betas[t], R.pt[c].states[t], R.rng);
      }
    } else {
      if (apply_icm(R, R.rngs[0][0])) return -1;
      for (uint32_t c = 0; c < nc; ++c) exchange_threaded(R, R.pt[c], R.rngs[c][0]);
#pragma omp parallel for collapse(2) schedule(dynamic, 1)
      for (uint32_t c = 0; c < nc; ++c)
        for (uint32_t t = 0; t < nb; ++t) ising_sweep(*R.I, R.P.betas[t], R.pt[c].states[t], R.rngs[c][t]);
    }
    apply_measurements(R, i);
    R.next_sweep = i + 1;
  }
  return 0;
}
// state access (slot order)
void orc_pt_state(void* h, uint32_t c, uint32_t t, int8_t* out, float* energy, int* init) {
  PtRun& R = *(PtRun*)h;
  const IsingState& s = R.pt[c].states[t];
  memcpy(out, s.arr.data(), s.arr.size());
  *energy = s.energy;
  *init = s.energy_init ? 1 : 0;
}
void orc_pt_set_state(void* h, uint32_t c, uint32_t t, const int8_t* in) {
  PtRun& R = *(PtRun*)h;
  IsingState& s = R.pt[c].states[t];
  memcpy(s.arr.data(), in, s.arr.size());
  s.energy_init = false;
  energy_cached(*R.I, s);
}
void orc_pt_acceptance(void* h, uint32_t c, uint32_t* out) {
  PtRun& R = *(PtRun*)h;
  memcpy(out, R.pt[c].num_acceptances.data(), R.pt[c].num_acceptances.size() * 4);
}
void orc_pt_tags(void* h, uint32_t c, uint8_t* tags, uint32_t* round_trips, uint32_t* diffusion_hist) {
  PtRun& R = *(PtRun*)h;
  memcpy(tags, R.pt[c].tags.data(), R.pt[c].tags.size());
  *round_trips = R.pt[c].round_trips;
  memcpy(diffusion_hist, R.pt[c].diffusion_hist.data(), R.pt[c].diffusion_hist.size() * 4);
}
void orc_pt_rng(void* h, int c, int t, uint64_t* s4) {
  PtRun& R = *(PtRun*)h;
  const Xoshiro& x = (c < 0) ? R.rng : R.rngs[(size_t)c][(size_t)t];
  memcpy(s4, x.s, 32);
}
uint32_t orc_pt_gs_count(void* h) { return (uint32_t)((PtRun*)h)->gs.size(); }
void orc_pt_gs_entry(void* h, uint32_t k, uint32_t* step, float* energy, uint64_t* words) {
  PtRun& R = *(PtRun*)h;
  *step = R.gs[k].step;
  *energy = R.gs[k].energy;
  memcpy(words, R.gs[k].state.data(), R.gs[k].state.size() * 8);
}
uint32_t orc_pt_num_e(void* h, uint32_t t) { return (uint32_t)((PtRun*)h)->e[t].size(); }
void orc_pt_e(void* h, uint32_t t, float* out) { PtRun& R = *(PtRun*)h; memcpy(out, R.e[t].data(), R.e[t].size() * 4); }
uint32_t orc_pt_num_q(void* h, uint32_t t) { return (uint32_t)((PtRun*)h)->q[t].size(); }
void orc_pt_q(void* h, uint32_t t, int32_t* out) { PtRun& R = *(PtRun*)h; memcpy(out, R.q[t].data(), R.q[t].size() * 4); }
void orc_pt_sus(void* h, uint32_t t, uint32_t k, float* out) {
  PtRun& R = *(PtRun*)h;
  memcpy(out, R.sus[t][k].data(), R.sus[t][k].size() * 4);
}
uint32_t orc_pt_num_sample_slots(void* h) { return (uint32_t)((PtRun*)h)->samples.size(); }
uint32_t orc_pt_num_samples(void* h, uint32_t s) { return (uint32_t)((PtRun*)h)->samples[s].size(); }
void orc_pt_sample(void* h, uint32_t s, uint32_t k, uint8_t* out) {
  PtRun& R = *(PtRun*)h;
  memcpy(out, R.samples[s][k].data(), R.samples[s][k].size());
}
uint32_t orc_pt_icm_count(void* h) { return (uint32_t)((PtRun*)h)->last_icm.size(); }
void orc_pt_icm_sizes(void* h, int64_t* out) {
  PtRun& R = *(PtRun*)h;
  memcpy(out, R.last_icm.data(), R.last_icm.size() * 8);
}

// -- Simulated annealing: SaRunner::run / run_parallel (src/sa.rs:110-165)
// with sa_loop (:167-199) and simulated_annealing (tamc-core/src/sa.rs:27-48).
// Writes r_eff = threads * (num_replicas / threads) energies (energy_ref) and
// states (int8, replica-major).  Returns r_eff, or 0 on bad parameters.
uint32_t orc_sa_run(const void* inst, const float* betas, uint32_t nbeta, uint32_t num_replicas,
                    uint32_t threads, uint64_t seed, int nthreads, float* energies, int8_t* states) {
  const Instance& I = *(const Instance*)inst;
  if (threads == 0 || num_replicas == 0) return 0;
  Xoshiro master = seed_from_u64(seed);
  uint32_t parts, per;
  if (num_replicas > 1) { parts = threads; per = num_replicas / threads; }
  else { parts = 1; per = 1; }
  std::vector<Xoshiro> rv;
  for (uint32_t p = 0; p < parts; ++p) { rv.push_back(master); master.jump(); }
  const uint32_t r_eff = parts * per;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif
#pragma omp parallel for schedule(dynamic, 1)
  for (uint32_t p = 0; p < parts; ++p) {
    Xoshiro& rng = rv[p];
    std::vector<IsingState> st;
    for (uint32_t r = 0; r < per; ++r) st.push_back(rand_state(I, rng));
    for (uint32_t b = 0; b < nbeta; ++b)
      for (uint32_t r = 0; r < per; ++r) plain_sweep(I, betas[b], st[r].arr.data(), rng);
    for (uint32_t r = 0; r < per; ++r) {
      const size_t g = (size_t)p * per + r;
      energies[g] = energy_ref(I, st[r].arr.data());
      memcpy(states + g * I.n, st[r].arr.data(), I.n);
    }
  }
  return r_eff;
}

// Bounded SA sample for timing: runs `parts` partitions of `per` replicas for
// nbeta sweeps; same code path as orc_sa_run.
}  // extern "C"

// -- GLA (run_gla, src/gla.rs:121-195) with the master stream seed_from_u64(seed)
// in place of the reference's OS-entropy seed.  Partition k is
// sites[part_ptr[k] .. part_ptr[k+1]) (file order, already checked as
// read_graph_partition does).  Writes part_e[nparts], up to bnd_cap boundary
// groups (count in *nbnd), *total and the joined state joined[n].
// Returns 0, -2 where the reference panics, -3 if bnd_cap is too small.
extern "C" int orc_gla_run(const void* inst, const uint32_t* part_ptr, const uint32_t* sites, uint32_t nparts,
                           uint32_t num_sweeps, double warmup_fraction, const float* betas, uint32_t nb,
                           uint32_t lo_beta_idx, int icm, uint32_t num_chains, int64_t sample,
                           int64_t sample_states, uint32_t sample_limiting, uint64_t seed, float* part_e,
                           uint32_t bnd_cap, uint32_t* nbnd, uint32_t* bnd_src, uint32_t* bnd_dst, float* bnd_e,
                           float* total, int8_t* joined) {
  const Instance& I = *(const Instance*)inst;
  // to_energy_graph (src/ising.rs:414-425): coupling entries with i < j
  struct E { uint32_t i, j; float K; };
  std::vector<E> edges;
  uint32_t nodes = 0;
  for (uint32_t i = 0; i < I.n; ++i)
    for (uint32_t e = I.row_ptr[i]; e < I.row_ptr[i + 1]; ++e)
      if (I.col[e] > i) { edges.push_back(E{i, I.col[e], I.K[e]}); nodes = std::max(nodes, I.col[e] + 1); }
  if (nodes < I.n) return -2;  // g[NodeIndex::new(i)] = h past the graph's nodes
  std::vector<int64_t> pmap(I.n, -1);
  std::vector<std::vector<uint32_t>> parts(nparts);
  for (uint32_t k = 0; k < nparts; ++k) {
    parts[k].assign(sites + part_ptr[k], sites + part_ptr[k + 1]);
    for (uint32_t x : parts[k]) pmap[x] = k;
    std::sort(parts[k].begin(), parts[k].end());  // partition_graph.add_node(p sorted)
  }
  for (uint32_t i = 0; i < nodes; ++i)
    if (pmap[i] < 0) return -2;  // partition_mapping[&i] on a missing key
  // partition graph: directed edge (p_i, p_j) per first appearance
  std::vector<std::pair<uint32_t, uint32_t>> keys;
  std::vector<std::vector<E>> groups;
  for (const E& e : edges) {
    const uint32_t a = (uint32_t)pmap[e.i], b = (uint32_t)pmap[e.j];
    if (a == b) continue;
    size_t x = 0;
    while (x < keys.size() && !(keys[x].first == a && keys[x].second == b)) ++x;
    if (x == keys.size()) { keys.emplace_back(a, b); groups.emplace_back(); }
    groups[x].push_back(e);
  }
  if (keys.size() > bnd_cap) return -3;
  // sub-instances (induced_subgraph_instance_sorted) and their runs:
  // rng_vec[k] = master cloned, then jumped; init and pt_loop on it
  Xoshiro master = seed_from_u64(seed);
  std::vector<std::vector<int8_t>> best(nparts);
  for (uint32_t k = 0; k < nparts; ++k) {
    const std::vector<uint32_t>& nodes_k = parts[k];
    Instance S;
    S.n = (uint32_t)nodes_k.size();
    S.offset = 0.0f;
    S.row_ptr.push_back(0);
    for (uint32_t ni : nodes_k) {
      S.bias.push_back(I.bias[ni]);
      for (uint32_t e = I.row_ptr[ni]; e < I.row_ptr[ni + 1]; ++e) {
        auto it = std::lower_bound(nodes_k.begin(), nodes_k.end(), I.col[e]);
        if (it != nodes_k.end() && *it == I.col[e]) {
          S.col.push_back((uint32_t)(it - nodes_k.begin()));
          S.K.push_back(I.K[e]);
        }
      }
      S.row_ptr.push_back((uint32_t)S.col.size());
    }
    for (const auto& w : I.suscept) {
      std::vector<double> sw;
      for (uint32_t ni : nodes_k) sw.push_back(w[ni]);
      S.suscept.push_back(sw);
    }
    build_icm_graph(S, true);
    Xoshiro rk = master;
    master.jump();
    PtRun* R = pt_make(&S, num_sweeps, warmup_fraction, betas, nb, lo_beta_idx, icm, num_chains, 1, sample,
                       sample_states, sample_limiting, rk);
    const int rc = orc_pt_run(R, num_sweeps, 0);  // serial loop: no OpenMP
    if (rc != 0 || R->gs.empty()) { delete R; return -2; }
    part_e[k] = R->gs.back().energy;
    best[k].assign(S.n, 1);
    for (uint32_t i = 0; i < S.n; ++i) best[k][i] = ((R->gs.back().state[i / 64] >> (i % 64)) & 1u) ? -1 : 1;
    delete R;
  }
  float bulk = 0.0f;
  for (uint32_t k = 0; k < nparts; ++k) bulk += part_e[k];
  float tb = 0.0f;
  for (size_t x = 0; x < keys.size(); ++x) {
    const uint32_t a = keys[x].first, b = keys[x].second;
    float bnd = 0.0f;
    for (const E& e : groups[x]) {
      const size_t is = std::lower_bound(parts[a].begin(), parts[a].end(), e.i) - parts[a].begin();
      const size_t js = std::lower_bound(parts[b].begin(), parts[b].end(), e.j) - parts[b].begin();
      const int8_t prod = (int8_t)(best[a][is] * best[b][js]);
      bnd += e.K * (float)prod;
    }
    tb += bnd;
    bnd_src[x] = a;
    bnd_dst[x] = b;
    bnd_e[x] = bnd;
  }
  *nbnd = (uint32_t)keys.size();
  *total = bulk + tb;
  for (uint32_t k = 0; k < nparts; ++k)
    for (size_t x = 0; x < parts[k].size(); ++x) joined[parts[k][x]] = best[k][x];
  return 0;
}
