// method.cpp -- YAML method files (a block/flow YAML subset sufficient for
// tamc's `Method` schema, src/lib.rs:80-84, PtIcmParams src/pt.rs:259-272,
// SaParams src/sa.rs:21-26, BetaOptions src/pt.rs:236-257) and beta ladders.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>

#include "internal.h"

namespace tamc {
namespace {

struct YNode {
  enum Kind { NUL, SCALAR, MAP, SEQ } kind = NUL;
  std::string s;
  bool quoted = false;
  std::vector<std::pair<std::string, YNode>> map;
  std::vector<YNode> seq;
  const YNode* get(const std::string& k) const {
    for (auto& kv : map)
      if (kv.first == k) return &kv.second;
    return nullptr;
  }
};

struct Line {
  int indent;
  std::string text;
  int no;
};

[[noreturn]] void yerr(int line, const std::string& m) {
  fail(TAMC_E_PARSE, "method file line " + std::to_string(line + 1) + ": " + m);
}

std::string rstrip(const std::string& s) {
  size_t e = s.size();
  while (e > 0 && (s[e - 1] == ' ' || s[e - 1] == '\t' || s[e - 1] == '\r')) --e;
  return s.substr(0, e);
}

// strip a trailing comment that is outside quotes
std::string strip_comment(const std::string& s) {
  bool sq = false, dq = false;
  for (size_t i = 0; i < s.size(); ++i) {
    const char c = s[i];
    if (c == '\'' && !dq) sq = !sq;
    else if (c == '"' && !sq) dq = !dq;
    else if (c == '#' && !sq && !dq && (i == 0 || s[i - 1] == ' ' || s[i - 1] == '\t')) return s.substr(0, i);
  }
  return s;
}

// ----- flow-style parsing
struct Flow {
  const std::string& s;
  size_t p = 0;
  int line;
  Flow(const std::string& str, int ln) : s(str), line(ln) {}
  void ws() {
    while (p < s.size() && (s[p] == ' ' || s[p] == '\t' || s[p] == '\n')) ++p;
  }
  YNode scalar(const char* stops) {
    ws();
    YNode n;
    n.kind = YNode::SCALAR;
    if (p < s.size() && (s[p] == '"' || s[p] == '\'')) {
      const char q = s[p++];
      while (p < s.size() && s[p] != q) {
        if (q == '"' && s[p] == '\\' && p + 1 < s.size()) ++p;
        n.s += s[p++];
      }
      if (p >= s.size()) yerr(line, "unterminated quoted scalar");
      ++p;
      n.quoted = true;
      return n;
    }
    const size_t b = p;
    while (p < s.size() && !strchr(stops, s[p])) ++p;
    n.s = rstrip(s.substr(b, p - b));
    if (n.s.empty() || n.s == "~" || n.s == "null" || n.s == "Null" || n.s == "NULL") n.kind = YNode::NUL;
    return n;
  }
  YNode value() {
    ws();
    if (p < s.size() && s[p] == '[') {
      ++p;
      YNode n;
      n.kind = YNode::SEQ;
      ws();
      if (p < s.size() && s[p] == ']') { ++p; return n; }
      for (;;) {
        n.seq.push_back(value());
        ws();
        if (p < s.size() && s[p] == ',') { ++p; ws(); if (p < s.size() && s[p] == ']') { ++p; return n; } continue; }
        if (p < s.size() && s[p] == ']') { ++p; return n; }
        yerr(line, "expected ',' or ']' in flow sequence");
      }
    }
    if (p < s.size() && s[p] == '{') {
      ++p;
      YNode n;
      n.kind = YNode::MAP;
      ws();
      if (p < s.size() && s[p] == '}') { ++p; return n; }
      for (;;) {
        YNode k = scalar(":,}");
        ws();
        if (p >= s.size() || s[p] != ':') yerr(line, "expected ':' in flow mapping");
        ++p;
        n.map.emplace_back(k.s, value());
        ws();
        if (p < s.size() && s[p] == ',') { ++p; continue; }
        if (p < s.size() && s[p] == '}') { ++p; return n; }
        yerr(line, "expected ',' or '}' in flow mapping");
      }
    }
    return scalar(",]}");
  }
};

// find "key:" at top level of a line; returns position of ':' or npos
size_t key_colon(const std::string& t) {
  bool sq = false, dq = false;
  int depth = 0;
  for (size_t i = 0; i < t.size(); ++i) {
    const char c = t[i];
    if (c == '\'' && !dq) sq = !sq;
    else if (c == '"' && !sq) dq = !dq;
    else if (!sq && !dq) {
      if (c == '[' || c == '{') ++depth;
      else if (c == ']' || c == '}') --depth;
      else if (c == ':' && depth == 0 && (i + 1 == t.size() || t[i + 1] == ' ' || t[i + 1] == '\t')) return i;
    }
  }
  return std::string::npos;
}

std::string unquote_key(std::string k) {
  k = rstrip(k);
  if (k.size() >= 2 && (k[0] == '"' || k[0] == '\'') && k.back() == k[0]) return k.substr(1, k.size() - 2);
  return k;
}

struct Block {
  std::vector<Line> L;
  size_t i = 0;

  YNode inline_value(const std::string& t, int line) {
    // a flow collection may continue over following more-indented lines
    std::string acc = t;
    if (!acc.empty() && (acc[0] == '[' || acc[0] == '{')) {
      auto balanced = [](const std::string& s) {
        int d = 0;
        bool sq = false, dq = false;
        for (char c : s) {
          if (c == '\'' && !dq) sq = !sq;
          else if (c == '"' && !sq) dq = !dq;
          else if (!sq && !dq) {
            if (c == '[' || c == '{') ++d;
            else if (c == ']' || c == '}') --d;
          }
        }
        return d <= 0;
      };
      while (!balanced(acc) && i < L.size()) acc += " " + L[i++].text;
      Flow f(acc, line);
      YNode n = f.value();
      return n;
    }
    Flow f(acc, line);
    return f.scalar("");
  }

  YNode parse(int indent) {
    if (i >= L.size()) return YNode();
    const Line& ln = L[i];
    if (ln.text == "-" || ln.text.rfind("- ", 0) == 0) return parse_seq(ln.indent);
    if (key_colon(ln.text) != std::string::npos) return parse_map(ln.indent);
    ++i;
    (void)indent;
    return inline_value(ln.text, ln.no);
  }

  YNode parse_seq(int indent) {
    YNode n;
    n.kind = YNode::SEQ;
    while (i < L.size() && L[i].indent == indent && (L[i].text == "-" || L[i].text.rfind("- ", 0) == 0)) {
      Line cur = L[i];
      std::string rest = cur.text.size() > 1 ? cur.text.substr(2) : std::string();
      size_t lead = 0;
      while (lead < rest.size() && rest[lead] == ' ') ++lead;
      rest = rest.substr(lead);
      if (rest.empty()) {
        ++i;
        if (i < L.size() && L[i].indent > indent) n.seq.push_back(parse(L[i].indent));
        else n.seq.push_back(YNode());
      } else if (rest[0] != '[' && rest[0] != '{' && (rest == "-" || rest.rfind("- ", 0) == 0 ||
                                                       key_colon(rest) != std::string::npos)) {
        // compact nested block: re-interpret the rest as a line at deeper indent
        L[i].indent = indent + 2 + (int)lead;
        L[i].text = rest;
        n.seq.push_back(parse(L[i].indent));
      } else {
        ++i;
        n.seq.push_back(inline_value(rest, cur.no));
      }
    }
    return n;
  }

  YNode parse_map(int indent) {
    YNode n;
    n.kind = YNode::MAP;
    while (i < L.size() && L[i].indent == indent) {
      const Line cur = L[i];
      const size_t c = key_colon(cur.text);
      if (c == std::string::npos) yerr(cur.no, "expected 'key: value'");
      const std::string key = unquote_key(cur.text.substr(0, c));
      std::string rest = cur.text.substr(c + 1);
      size_t lead = 0;
      while (lead < rest.size() && (rest[lead] == ' ' || rest[lead] == '\t')) ++lead;
      rest = rest.substr(lead);
      ++i;
      YNode v;
      if (rest.empty()) {
        if (i < L.size() && L[i].indent > indent) v = parse(L[i].indent);
        else if (i < L.size() && L[i].indent == indent && (L[i].text == "-" || L[i].text.rfind("- ", 0) == 0))
          v = parse_seq(indent);
      } else {
        v = inline_value(rest, cur.no);
      }
      for (auto& kv : n.map)
        if (kv.first == key) yerr(cur.no, "duplicate key '" + key + "'");
      n.map.emplace_back(key, std::move(v));
    }
    if (i < L.size() && L[i].indent > indent) yerr(L[i].no, "bad indentation");
    return n;
  }
};

YNode parse_yaml(const std::string& text) {
  Block b;
  std::istringstream is(text);
  std::string raw;
  int no = 0;
  while (std::getline(is, raw)) {
    std::string t = rstrip(strip_comment(raw));
    const int ln = no++;
    if (t.find('\t') != std::string::npos && t.find_first_not_of(" \t") != std::string::npos) {
      const size_t f = t.find_first_not_of(" ");
      if (t[f] == '\t') yerr(ln, "tabs are not allowed for indentation");
    }
    size_t ind = t.find_first_not_of(' ');
    if (ind == std::string::npos) continue;
    std::string body = t.substr(ind);
    if (body == "---" || body.rfind("--- ", 0) == 0) {
      body = body.size() > 3 ? body.substr(4) : std::string();
      if (body.empty()) continue;
    }
    if (body == "...") break;
    b.L.push_back({(int)ind, body, ln});
  }
  if (b.L.empty()) fail(TAMC_E_PARSE, "empty method file");
  YNode root = b.parse(b.L[0].indent);
  if (b.i != b.L.size()) yerr(b.L[b.i].no, "unexpected content");
  return root;
}

// ----- typed accessors
bool to_u64(const YNode& n, uint64_t& v) {
  if (n.kind != YNode::SCALAR || n.quoted || n.s.empty()) return false;
  const char* s = n.s.c_str();
  char* e;
  if (s[0] == '-') return false;
  if (s[0] == '+') ++s;
  int base = 10;
  if (s[0] == '0' && (s[1] == 'x' || s[1] == 'X')) { base = 16; s += 2; }
  else if (s[0] == '0' && s[1] == 'o') { base = 8; s += 2; }
  errno = 0;
  v = strtoull(s, &e, base);
  return *e == 0 && e != s && errno == 0;
}
bool to_f64(const YNode& n, double& v) {
  if (n.kind != YNode::SCALAR || n.quoted || n.s.empty()) return false;
  const std::string& s = n.s;
  if (s == ".inf" || s == ".Inf" || s == ".INF" || s == "+.inf") { v = INFINITY; return true; }
  if (s == "-.inf" || s == "-.Inf" || s == "-.INF") { v = -INFINITY; return true; }
  if (s == ".nan" || s == ".NaN" || s == ".NAN") { v = NAN; return true; }
  char* e;
  v = strtod(s.c_str(), &e);
  if (*e != 0 || e == s.c_str()) return false;
  for (char c : s)
    if (!(isdigit((unsigned char)c) || c == '.' || c == '-' || c == '+' || c == 'e' || c == 'E')) return false;
  return true;
}
bool to_bool(const YNode& n, bool& v) {
  if (n.kind != YNode::SCALAR || n.quoted) return false;
  if (n.s == "true" || n.s == "True" || n.s == "TRUE") { v = true; return true; }
  if (n.s == "false" || n.s == "False" || n.s == "FALSE") { v = false; return true; }
  return false;
}

const YNode& req(const YNode& m, const char* k, const char* ctx) {
  const YNode* v = m.get(k);
  if (!v) fail(TAMC_E_PARSE, std::string(ctx) + ": missing field `" + k + "`");
  return *v;
}
uint32_t get_u32(const YNode& v, const char* k) {
  uint64_t x;
  if (!to_u64(v, x) || x > 0xffffffffull) fail(TAMC_E_PARSE, std::string("field `") + k + "`: expected u32");
  return (uint32_t)x;
}
uint8_t get_u8(const YNode& v, const char* k) {
  uint64_t x;
  if (!to_u64(v, x) || x > 255) fail(TAMC_E_PARSE, std::string("field `") + k + "`: expected u8");
  return (uint8_t)x;
}
double get_f64(const YNode& v, const char* k) {
  double x;
  if (!to_f64(v, x)) fail(TAMC_E_PARSE, std::string("field `") + k + "`: expected a number");
  return x;
}
bool get_bool(const YNode& v, const char* k) {
  bool x;
  if (!to_bool(v, x)) fail(TAMC_E_PARSE, std::string("field `") + k + "`: expected a bool");
  return x;
}
bool is_none(const YNode* v) { return !v || v->kind == YNode::NUL; }

// externally tagged enum: a single-key map {Variant: body}
const YNode& variant(const YNode& n, std::string& tag, const char* ctx) {
  if (n.kind == YNode::MAP && n.map.size() == 1) {
    tag = n.map[0].first;
    return n.map[0].second;
  }
  if (n.kind == YNode::SCALAR) {
    tag = n.s;
    return n;
  }
  fail(TAMC_E_PARSE, std::string(ctx) + ": expected an externally tagged enum");
}

BetaSpec parse_beta(const YNode& n) {
  std::string tag;
  const YNode& b = variant(n, tag, "beta");
  BetaSpec s;
  if (tag == "Geometric") {
    if (b.kind != YNode::MAP) fail(TAMC_E_PARSE, "beta.Geometric: expected a mapping");
    s.geometric = true;
    s.beta_min = (float)get_f64(req(b, "beta_min", "Geometric"), "beta_min");
    s.beta_max = (float)get_f64(req(b, "beta_max", "Geometric"), "beta_max");
    s.num_beta = get_u32(req(b, "num_beta", "Geometric"), "num_beta");
  } else if (tag == "Arr") {
    if (b.kind != YNode::SEQ) fail(TAMC_E_PARSE, "beta.Arr: expected a sequence");
    s.geometric = false;
    for (auto& x : b.seq) s.arr.push_back((float)get_f64(x, "Arr"));
  } else {
    fail(TAMC_E_PARSE, "beta: unknown variant `" + tag + "`, expected `Geometric` or `Arr`");
  }
  return s;
}

}  // namespace

std::vector<float> geometric_betas(float bmin, float bmax, uint32_t n) {
  // geometric_beta_schedule (tamc-core/src/sa.rs:13-22) evaluated in f64, cast to f32.
  std::vector<float> out(n);
  const double lb0 = std::log((double)bmin), lbf = std::log((double)bmax);
  const double d = (lbf - lb0) / (double)(n - 1);
  for (uint32_t i = 0; i < n; ++i) out[i] = (float)std::exp(lb0 + d * (double)i);
  return out;
}

std::vector<float> BetaSpec::resolve() const {
  return geometric ? geometric_betas(beta_min, beta_max, num_beta) : arr;
}

uint32_t resolve_lo_beta_idx(const PtParamsHost& p, const std::vector<float>& betas, bool* warn) {
  const uint32_t nb = (uint32_t)betas.size();
  if (warn) *warn = false;
  if (p.has_lo_num_beta) {
    const uint32_t l = std::min(p.lo_num_beta, nb);
    return nb - l;
  }
  if (p.has_lo_beta) {
    for (uint32_t i = 0; i < nb; ++i)
      if (betas[i] >= p.lo_beta) return i;
    if (warn) *warn = true;
    return nb - 1;
  }
  if (p.icm) fail(TAMC_E_REFPANIC, "Must specify either lo_beta or lo_num_beta for ICM");
  return 0;
}

// PtIcmParams (src/pt.rs:259-272) from a mapping, with the ladder and lo_beta_idx resolved.
static void parse_pt_body(const YNode& body, Method& m) {
  {
    PtParamsHost& p = m.pt;
    p.num_sweeps = get_u32(req(body, "num_sweeps", "PT"), "num_sweeps");
    p.warmup_fraction = get_f64(req(body, "warmup_fraction", "PT"), "warmup_fraction");
    p.beta = parse_beta(req(body, "beta", "PT"));
    const YNode* v;
    if (!is_none(v = body.get("lo_beta"))) { p.has_lo_beta = true; p.lo_beta = (float)get_f64(*v, "lo_beta"); }
    if (!is_none(v = body.get("lo_num_beta"))) { p.has_lo_num_beta = true; p.lo_num_beta = get_u32(*v, "lo_num_beta"); }
    p.icm = get_bool(req(body, "icm", "PT"), "icm");
    p.num_replica_chains = get_u32(req(body, "num_replica_chains", "PT"), "num_replica_chains");
    p.threads = get_u32(req(body, "threads", "PT"), "threads");
    if (!is_none(v = body.get("sample"))) { p.has_sample = true; p.sample = get_u32(*v, "sample"); }
    if (!is_none(v = body.get("sample_states"))) { p.has_sample_states = true; p.sample_states = get_u32(*v, "sample_states"); }
    if (!is_none(v = body.get("sample_limiting"))) { p.has_sample_limiting = true; p.sample_limiting = get_u8(*v, "sample_limiting"); }
    m.betas = p.beta.resolve();
    for (size_t k = 1; k < m.betas.size(); ++k)
      if (!(m.betas[k] - m.betas[k - 1] >= 0.0f)) fail(TAMC_E_REFPANIC, "beta array must be non-decreasing");
    if (m.betas.empty()) fail(TAMC_E_REFPANIC, "beta array must not be empty");
    m.lo_beta_idx = resolve_lo_beta_idx(p, m.betas, nullptr);
  }
}

void parse_method_yaml(const std::string& text, Method& m) {
  YNode root = parse_yaml(text);
  std::string tag;
  const YNode& body = variant(root, tag, "method");
  if (tag == "PT") {
    if (body.kind != YNode::MAP) fail(TAMC_E_PARSE, "PT: expected a mapping");
    parse_pt_body(body, m);
    m.kind = TAMC_METHOD_PT;
  } else if (tag == "SA") {
    if (body.kind != YNode::MAP) fail(TAMC_E_PARSE, "SA: expected a mapping");
    m.sa.beta = parse_beta(req(body, "beta", "SA"));
    m.sa.num_replicas = get_u32(req(body, "num_replicas", "SA"), "num_replicas");
    m.sa.threads = get_u32(req(body, "threads", "SA"), "threads");
    m.kind = TAMC_METHOD_SA;
    m.betas = m.sa.beta.resolve();
    for (size_t k = 1; k < m.betas.size(); ++k)
      if (!(m.betas[k] - m.betas[k - 1] >= 0.0f)) fail(TAMC_E_REFPANIC, "beta array must be non-decreasing");
  } else if (tag == "GLA") {
    // GlaParams (src/gla.rs:28-33)
    if (body.kind != YNode::MAP) fail(TAMC_E_PARSE, "GLA: expected a mapping");
    m.gla.num_threads = get_u32(req(body, "num_threads", "GLA"), "num_threads");
    const YNode& pt = req(body, "pt_params", "GLA");
    if (pt.kind != YNode::MAP) fail(TAMC_E_PARSE, "GLA.pt_params: expected a mapping");
    parse_pt_body(pt, m);
    const YNode& pf = req(body, "partition_file", "GLA");
    if (pf.kind != YNode::SCALAR) fail(TAMC_E_PARSE, "field `partition_file`: expected a string");
    m.gla.partition_file = pf.s;
    m.kind = TAMC_METHOD_GLA;
  } else {
    fail(TAMC_E_PARSE, "unknown variant `" + tag + "`, expected one of `PT`, `SA`, `GLA`");
  }
}

}  // namespace tamc

using namespace tamc;

extern "C" {

int tamc_method_parse(const char* yaml, uint64_t len, tamc_method** out) {
  TAMC_API_BEGIN
  if (!out || (!yaml && len)) fail(TAMC_E_INVAL, "null argument");
  auto* m = new tamc_method();
  try {
    parse_method_yaml(std::string(yaml, (size_t)len), m->m);
  } catch (...) {
    delete m;
    throw;
  }
  *out = m;
  TAMC_API_END
}

int tamc_method_read(const char* path, tamc_method** out) {
  TAMC_API_BEGIN
  if (!path) fail(TAMC_E_INVAL, "null path");
  std::ifstream f(path, std::ios::binary);
  if (!f) fail(TAMC_E_IO, std::string("Could not open '") + path + "'");
  std::stringstream ss;
  ss << f.rdbuf();
  const std::string s = ss.str();
  return tamc_method_parse(s.data(), s.size(), out);
  TAMC_API_END
}

int tamc_method_kind(const tamc_method* m) { return m ? m->m.kind : 0; }

int tamc_method_gla(const tamc_method* m, uint32_t* num_threads, const char** partition_file, tamc_pt_params* p) {
  TAMC_API_BEGIN
  if (!m) fail(TAMC_E_INVAL, "null method");
  if (m->m.kind != TAMC_METHOD_GLA) fail(TAMC_E_INVAL, "not a GLA method");
  if (num_threads) *num_threads = m->m.gla.num_threads;
  if (partition_file) *partition_file = m->m.gla.partition_file.c_str();
  if (p) return tamc_method_pt(m, p);
  TAMC_API_END
}

int tamc_method_pt(const tamc_method* m, tamc_pt_params* p) {
  TAMC_API_BEGIN
  if (!m || !p) fail(TAMC_E_INVAL, "null argument");
  if (m->m.kind != TAMC_METHOD_PT && m->m.kind != TAMC_METHOD_GLA) fail(TAMC_E_INVAL, "not a PT method");
  const PtParamsHost& q = m->m.pt;
  p->num_sweeps = q.num_sweeps;
  p->warmup_fraction = q.warmup_fraction;
  p->num_beta = (uint32_t)m->m.betas.size();
  p->betas = m->m.betas.data();
  p->lo_beta_idx = m->m.lo_beta_idx;
  p->icm = q.icm;
  p->num_replica_chains = q.num_replica_chains;
  p->threads = q.threads;
  p->sample = q.has_sample ? (int64_t)q.sample : -1;
  p->sample_states = q.has_sample_states ? (int64_t)q.sample_states : -1;
  p->sample_limiting = q.has_sample_limiting ? q.sample_limiting : 0;
  TAMC_API_END
}

int tamc_method_sa(const tamc_method* m, const float** betas, uint32_t* nbeta, uint32_t* num_replicas,
                   uint32_t* threads) {
  TAMC_API_BEGIN
  if (!m) fail(TAMC_E_INVAL, "null method");
  if (m->m.kind != TAMC_METHOD_SA) fail(TAMC_E_INVAL, "not an SA method");
  if (betas) *betas = m->m.betas.data();
  if (nbeta) *nbeta = (uint32_t)m->m.betas.size();
  if (num_replicas) *num_replicas = m->m.sa.num_replicas;
  if (threads) *threads = m->m.sa.threads;
  TAMC_API_END
}

void tamc_method_free(tamc_method* m) { delete m; }

int tamc_geometric_betas(float beta_min, float beta_max, uint32_t n, float* out) {
  TAMC_API_BEGIN
  if (!out && n) fail(TAMC_E_INVAL, "null output");
  std::vector<float> b = geometric_betas(beta_min, beta_max, n);
  for (uint32_t i = 0; i < n; ++i) out[i] = b[i];
  TAMC_API_END
}

}  // extern "C"
