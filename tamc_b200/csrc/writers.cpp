// writers.cpp -- result files in the reference's formats:
//   * YAML PtIcmMinResults (src/pt.rs:96-102 + flattened MinResults,
//     src/ising_results.rs:5-13) and AnnealMinResults (src/sa.rs:28-34), in the
//     layout serde_yaml 0.8 emits (block style, 2-space indent, compact nested
//     sequences, shortest round-trip floats, `~` for None);
//   * bincode 1.x default encoding (little-endian, fixed-width ints, u64
//     lengths) of PtIcmThermalSamples (src/pt.rs:117-125) and AnnealState
//     (src/sa.rs:68-72).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "internal.h"

namespace tamc {

// Shortest round-trip decimal in the style of the ryu crate's pretty printer.
static std::string fmt_shortest(double v, bool is_f32) {
  if (std::isnan(v)) return ".nan";
  if (std::isinf(v)) return v > 0 ? ".inf" : "-.inf";
  if (v == 0.0) return std::signbit(v) ? "-0.0" : "0.0";
  char buf[64];
  int prec = 1;
  for (; prec <= 17; ++prec) {
    snprintf(buf, sizeof buf, "%.*e", prec - 1, v);
    if (is_f32 ? (strtof(buf, nullptr) == (float)v) : (strtod(buf, nullptr) == v)) break;
  }
  // buf = [-]d.ddde[+-]XX
  std::string s(buf);
  bool neg = s[0] == '-';
  if (neg) s = s.substr(1);
  const size_t epos = s.find('e');
  int exp10 = atoi(s.c_str() + epos + 1);
  std::string digits;
  for (size_t k = 0; k < epos; ++k)
    if (s[k] != '.') digits += s[k];
  while (digits.size() > 1 && digits.back() == '0') digits.pop_back();
  const int len = (int)digits.size();
  const int kk = exp10 + 1;  // position of the decimal point
  std::string out;
  if (len <= kk && kk <= 16) {
    out = digits + std::string((size_t)(kk - len), '0') + ".0";
  } else if (0 < kk && kk <= 16) {
    out = digits.substr(0, (size_t)kk) + "." + digits.substr((size_t)kk);
  } else if (-5 < kk && kk <= 0) {
    out = "0." + std::string((size_t)(-kk), '0') + digits;
  } else if (len == 1) {
    out = digits + "e" + std::to_string(kk - 1);
  } else {
    out = digits.substr(0, 1) + "." + digits.substr(1) + "e" + std::to_string(kk - 1);
  }
  return neg ? "-" + out : out;
}
std::string fmt_f32(float v) { return fmt_shortest((double)v, true); }

// Rust's Display of an f32 (`{}`): the shortest round-trip digits written out
// in positional notation, with no `.0` on whole numbers.
std::string fmt_f32_display(float v) {
  if (std::isnan(v)) return "NaN";
  if (std::isinf(v)) return v > 0 ? "inf" : "-inf";
  if (v == 0.0f) return std::signbit(v) ? "-0" : "0";
  char buf[64];
  int prec = 1;
  for (; prec <= 9; ++prec) {
    snprintf(buf, sizeof buf, "%.*e", prec - 1, (double)v);
    if (strtof(buf, nullptr) == v) break;
  }
  std::string s(buf);
  const bool neg = s[0] == '-';
  if (neg) s = s.substr(1);
  const size_t epos = s.find('e');
  const int exp10 = atoi(s.c_str() + epos + 1);
  std::string digits;
  for (size_t k = 0; k < epos; ++k)
    if (s[k] != '.') digits += s[k];
  while (digits.size() > 1 && digits.back() == '0') digits.pop_back();
  const int len = (int)digits.size(), kk = exp10 + 1;
  std::string out;
  if (kk <= 0) out = "0." + std::string((size_t)(-kk), '0') + digits;
  else if (kk >= len) out = digits + std::string((size_t)(kk - len), '0');
  else out = digits.substr(0, (size_t)kk) + "." + digits.substr((size_t)kk);
  return neg ? "-" + out : out;
}
std::string fmt_f64(double v) { return fmt_shortest(v, false); }

namespace {
struct Y {
  std::string o;
  void kv(int ind, const std::string& k, const std::string& v) { o += std::string(ind, ' ') + k + ": " + v + "\n"; }
  void key(int ind, const std::string& k) { o += std::string(ind, ' ') + k + ":\n"; }
  template <class T, class F>
  void seq(int ind, const std::string& k, const std::vector<T>& v, F f) {
    if (v.empty()) { kv(ind, k, "[]"); return; }
    key(ind, k);
    for (auto& x : v) o += std::string(ind + 2, ' ') + "- " + f(x) + "\n";
  }
};

void yaml_beta(Y& y, int ind, const BetaSpec& b) {
  y.key(ind, "beta");
  if (b.geometric) {
    y.key(ind + 2, "Geometric");
    y.kv(ind + 4, "beta_min", fmt_f32(b.beta_min));
    y.kv(ind + 4, "beta_max", fmt_f32(b.beta_max));
    y.kv(ind + 4, "num_beta", std::to_string(b.num_beta));
  } else {
    if (b.arr.empty()) {
      y.kv(ind + 2, "Arr", "[]");
    } else {
      y.key(ind + 2, "Arr");
      for (float v : b.arr) y.o += std::string(ind + 4, ' ') + "- " + fmt_f32(v) + "\n";
    }
  }
}
}  // namespace

// PtIcmParams fields (src/pt.rs:259-272) at indentation `ind`
static void yaml_pt_params(Y& y, int ind, const PtParamsHost& p) {
  y.kv(ind, "num_sweeps", std::to_string(p.num_sweeps));
  y.kv(ind, "warmup_fraction", fmt_f64(p.warmup_fraction));
  yaml_beta(y, ind, p.beta);
  y.kv(ind, "lo_beta", p.has_lo_beta ? fmt_f32(p.lo_beta) : "~");
  y.kv(ind, "lo_num_beta", p.has_lo_num_beta ? std::to_string(p.lo_num_beta) : "~");
  y.kv(ind, "icm", p.icm ? "true" : "false");
  y.kv(ind, "num_replica_chains", std::to_string(p.num_replica_chains));
  y.kv(ind, "threads", std::to_string(p.threads));
  y.kv(ind, "sample", p.has_sample ? std::to_string(p.sample) : "~");
  y.kv(ind, "sample_states", p.has_sample_states ? std::to_string(p.sample_states) : "~");
  y.kv(ind, "sample_limiting", p.has_sample_limiting ? std::to_string(p.sample_limiting) : "~");
}

std::string yaml_pt_method(const PtParamsHost& p) {
  Y y;
  y.o = "---\n";
  y.key(0, "PT");
  yaml_pt_params(y, 2, p);
  return y.o;
}

std::string yaml_pt_min_results(const PtMinResultsOut& r) {
  Y y;
  y.o = "---\n";
  const PtParamsHost& p = *r.params;
  y.key(0, "params");
  yaml_pt_params(y, 2, p);
  y.kv(0, "timing", fmt_f64(r.timing_us));
  y.seq(0, "gs_time_steps", r.gs_time_steps, [](uint32_t v) { return std::to_string(v); });
  y.seq(0, "gs_energies", r.gs_energies, [](float v) { return fmt_f32(v); });
  if (r.gs_states.empty()) {
    y.kv(0, "gs_states", "[]");
  } else {
    y.key(0, "gs_states");
    for (auto& st : r.gs_states) {
      if (st.empty()) { y.o += "  - []\n"; continue; }
      for (size_t k = 0; k < st.size(); ++k)
        y.o += std::string(k == 0 ? "  - - " : "    - ") + std::to_string(st[k]) + "\n";
    }
  }
  y.kv(0, "num_measurements", "0");
  y.kv(0, "instance_size", std::to_string(r.instance_size));
  y.seq(0, "acceptance_counts", r.acceptance_counts, [](uint32_t v) { return std::to_string(v); });
  return y.o;
}

std::string yaml_anneal_min_results(const AnnealMinResultsOut& r) {
  Y y;
  y.o = "---\n";
  y.key(0, "params");
  yaml_beta(y, 2, r.params->beta);
  y.kv(2, "num_replicas", std::to_string(r.num_replicas_eff));
  y.kv(2, "threads", std::to_string(r.params->threads));
  y.kv(0, "timing", fmt_f64(r.timing_us));
  y.kv(0, "min_energy", fmt_f32(r.min_energy));
  y.seq(0, "energies", r.energies, [](float v) { return fmt_f32(v); });
  return y.o;
}

namespace {
struct B {
  std::string o;
  void u8(uint8_t v) { o.push_back((char)v); }
  void u32(uint32_t v) { o.append((const char*)&v, 4); }
  void i32(int32_t v) { o.append((const char*)&v, 4); }
  void u64(uint64_t v) { o.append((const char*)&v, 8); }
  void f32(float v) { o.append((const char*)&v, 4); }
  void len(size_t n) { u64((uint64_t)n); }
};
}  // namespace

std::string bincode_thermal_samples(const ThermalSamplesOut& t) {
  B b;
  b.u8(t.compression_level);
  b.u64(t.instance_size);
  b.len(t.beta_arr.size());
  for (float v : t.beta_arr) b.f32(v);
  b.len(t.samples.size());
  for (auto& s : t.samples) {
    b.len(s.size());
    for (auto& bytes : s) {
      b.len(bytes.size());
      b.o.append((const char*)bytes.data(), bytes.size());
    }
  }
  b.len(t.e.size());
  for (auto& r : t.e) {
    b.len(r.size());
    for (float v : r) b.f32(v);
  }
  b.len(t.q.size());
  for (auto& r : t.q) {
    b.len(r.size());
    for (int32_t v : r) b.i32(v);
  }
  b.len(t.suscept.size());
  for (auto& r : t.suscept) {
    b.len(r.size());
    for (auto& c : r) {
      b.len(c.size());
      for (float v : c) b.f32(v);
    }
  }
  return b.o;
}

std::string bincode_anneal_state(uint32_t instance_size, uint32_t num_replicas, const std::vector<uint8_t>& bytes) {
  B b;
  b.u32(instance_size);
  b.u32(num_replicas);
  b.len(bytes.size());
  b.o.append((const char*)bytes.data(), bytes.size());
  return b.o;
}

namespace {
// Minimal pickle (protocol 3) emitter: dicts with string keys, lists, ints,
// floats, strings, bools and None -- the value kinds serde-pickle produces for
// these result structs (structs as dicts, Vec<u8> as lists of ints).
struct Pk {
  std::string o;
  Pk() { o += "\x80\x03"; }
  void str(const std::string& s) {
    o.push_back('X');
    const uint32_t n = (uint32_t)s.size();
    o.append((const char*)&n, 4);
    o += s;
  }
  void i64(int64_t v) {
    if (v >= 0 && v < 256) { o.push_back('K'); o.push_back((char)v); return; }
    if (v >= 0 && v < 65536) { o.push_back('M'); const uint16_t x = (uint16_t)v; o.append((const char*)&x, 2); return; }
    if (v >= INT32_MIN && v <= INT32_MAX) { o.push_back('J'); const int32_t x = (int32_t)v; o.append((const char*)&x, 4); return; }
    o.push_back('\x8a');
    o.push_back(8);
    o.append((const char*)&v, 8);
  }
  void u64(uint64_t v) {
    if (v <= (uint64_t)INT64_MAX) { i64((int64_t)v); return; }
    o.push_back('\x8a');
    o.push_back(9);
    o.append((const char*)&v, 8);
    o.push_back(0);
  }
  void f64(double v) {
    o.push_back('G');
    uint64_t b;
    memcpy(&b, &v, 8);
    for (int k = 7; k >= 0; --k) o.push_back((char)((b >> (8 * k)) & 0xff));
  }
  void none() { o.push_back('N'); }
  void boolean(bool b) { o.push_back(b ? '\x88' : '\x89'); }
  void dict_begin() { o.push_back('}'); o.push_back('('); }
  void dict_end() { o.push_back('u'); }
  void list_begin() { o.push_back(']'); o.push_back('('); }
  void list_end() { o.push_back('e'); }
  void tuple_begin() { o.push_back('('); }
  void tuple_end() { o.push_back('t'); }
  std::string finish() { o.push_back('.'); return o; }
};

void pk_beta(Pk& p, const BetaSpec& b) {
  p.dict_begin();
  if (b.geometric) {
    p.str("Geometric");
    p.dict_begin();
    p.str("beta_min"); p.f64(b.beta_min);
    p.str("beta_max"); p.f64(b.beta_max);
    p.str("num_beta"); p.u64(b.num_beta);
    p.dict_end();
  } else {
    p.str("Arr");
    p.list_begin();
    for (float v : b.arr) p.f64(v);
    p.list_end();
  }
  p.dict_end();
}
}  // namespace

std::string pickle_thermal_samples(const ThermalSamplesOut& t) {
  Pk p;
  p.dict_begin();
  p.str("compression_level"); p.u64(t.compression_level);
  p.str("instance_size"); p.u64(t.instance_size);
  p.str("beta_arr"); p.list_begin(); for (float v : t.beta_arr) p.f64(v); p.list_end();
  p.str("samples");
  p.list_begin();
  for (auto& s : t.samples) {
    p.list_begin();
    for (auto& b : s) { p.list_begin(); for (uint8_t x : b) p.u64(x); p.list_end(); }
    p.list_end();
  }
  p.list_end();
  p.str("e"); p.list_begin(); for (auto& r : t.e) { p.list_begin(); for (float v : r) p.f64(v); p.list_end(); } p.list_end();
  p.str("q"); p.list_begin(); for (auto& r : t.q) { p.list_begin(); for (int32_t v : r) p.i64(v); p.list_end(); } p.list_end();
  p.str("suscept");
  p.list_begin();
  for (auto& r : t.suscept) {
    p.list_begin();
    for (auto& c : r) { p.list_begin(); for (float v : c) p.f64(v); p.list_end(); }
    p.list_end();
  }
  p.list_end();
  p.dict_end();
  return p.finish();
}

std::string pickle_anneal_min_results(const AnnealMinResultsOut& r) {
  Pk p;
  p.dict_begin();
  p.str("params");
  p.dict_begin();
  p.str("beta"); pk_beta(p, r.params->beta);
  p.str("num_replicas"); p.u64(r.num_replicas_eff);
  p.str("threads"); p.u64(r.params->threads);
  p.dict_end();
  p.str("timing"); p.f64(r.timing_us);
  p.str("min_energy"); p.f64(r.min_energy);
  p.str("energies"); p.list_begin(); for (float v : r.energies) p.f64(v); p.list_end();
  p.dict_end();
  return p.finish();
}

std::string pickle_anneal_state(uint32_t instance_size, uint32_t num_replicas, const std::vector<uint8_t>& bytes) {
  Pk p;
  p.dict_begin();
  p.str("instance_size"); p.u64(instance_size);
  p.str("num_replicas"); p.u64(num_replicas);
  p.str("bytes"); p.list_begin(); for (uint8_t b : bytes) p.u64(b); p.list_end();
  p.dict_end();
  return p.finish();
}

// GlaResults (src/gla.rs:61-69) in bincode's default encoding: instance_size
// u32, num_partitions u32, partition_energies Vec<f32>, boundary_energies
// Vec<(u32, u32, f32)>, final_state Vec<u8> (left empty by run_gla), total_energy f32.
std::string bincode_gla_results(const GlaResultsOut& r) {
  B b;
  b.u32(r.instance_size);
  b.u32(r.num_partitions);
  b.len(r.partition_energies.size());
  for (float v : r.partition_energies) b.f32(v);
  b.len(r.bnd_energies.size());
  for (size_t k = 0; k < r.bnd_energies.size(); ++k) {
    b.u32(r.bnd_src[k]);
    b.u32(r.bnd_dst[k]);
    b.f32(r.bnd_energies[k]);
  }
  b.len(0);
  b.f32(r.total_energy);
  return b.o;
}

std::string pickle_gla_results(const GlaResultsOut& r) {
  Pk p;
  p.dict_begin();
  p.str("instance_size"); p.u64(r.instance_size);
  p.str("num_partitions"); p.u64(r.num_partitions);
  p.str("partition_energies"); p.list_begin(); for (float v : r.partition_energies) p.f64(v); p.list_end();
  p.str("boundary_energies");
  p.list_begin();
  for (size_t k = 0; k < r.bnd_energies.size(); ++k) {
    p.tuple_begin();
    p.u64(r.bnd_src[k]);
    p.u64(r.bnd_dst[k]);
    p.f64(r.bnd_energies[k]);
    p.tuple_end();
  }
  p.list_end();
  p.str("final_state"); p.list_begin(); p.list_end();
  p.str("total_energy"); p.f64(r.total_energy);
  p.dict_end();
  return p.finish();
}

}  // namespace tamc
