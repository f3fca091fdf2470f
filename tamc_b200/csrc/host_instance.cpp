// host_instance.cpp -- instance files, susceptibility vectors, graph colouring
// and the host-side C ABI for instances.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <numeric>
#include <sstream>

#include "internal.h"

namespace tamc {

static thread_local std::string g_last_error;
void set_error(const std::string& msg) { g_last_error = msg; }

static inline bool is_sp(char c) { return c == ' ' || c == '\t'; }

// One `i j K` line as nom parses it (src/util.rs:38-63): space0 u32 space1
// u32 space1 then `-?digits(.digits*)?`; the remainder of the line is ignored.
// Returns 1 parsed, 0 "Ignoring line", -1 integer overflow (the reference
// unwraps u32::from_str and aborts).
static int parse_ijk(const char* p, const char* end, uint32_t& i, uint32_t& j, double& k) {
  uint32_t v[2];
  for (int t = 0; t < 2; ++t) {
    while (p < end && is_sp(*p)) ++p;
    const char* d = p;
    uint64_t acc = 0;
    bool ovf = false;
    while (p < end && *p >= '0' && *p <= '9') {
      acc = acc * 10u + (uint64_t)(*p - '0');
      if (acc > 0xffffffffull) ovf = true;
      ++p;
    }
    if (p == d) return 0;
    if (ovf) return -1;
    v[t] = (uint32_t)acc;
    const char* s = p;
    while (p < end && is_sp(*p)) ++p;
    if (p == s) return 0;
  }
  const char* s = p;
  if (p < end && *p == '-') ++p;
  const char* d = p;
  while (p < end && *p >= '0' && *p <= '9') ++p;
  if (p == d) return 0;
  if (p < end && *p == '.') {
    ++p;
    while (p < end && *p >= '0' && *p <= '9') ++p;
  }
  char buf[512];
  const size_t L = (size_t)(p - s);
  std::string big;
  const char* num;
  if (L < sizeof(buf)) {
    memcpy(buf, s, L);
    buf[L] = 0;
    num = buf;
  } else {
    big.assign(s, L);
    num = big.c_str();
  }
  k = strtod(num, nullptr);  // correctly rounded decimal -> f64, like Rust's str::parse
  i = v[0];
  j = v[1];
  return 1;
}

void parse_instance_text(const char* text, size_t len, bool qubo, HostInstance& out) {
  // Directed entries (row, col, K, line order); the BTreeMap insert semantics
  // of read_adjacency_list (src/util.rs:84-99) keep the last write per (row,col).
  struct E { uint32_t r, c; float K; uint64_t seq; };
  std::vector<E> ent;
  uint64_t nrows = 0, seq = 0;
  const char* p = text;
  const char* end = text + len;
  uint64_t lineno = 0;
  while (p < end) {
    const char* nl = (const char*)memchr(p, '\n', (size_t)(end - p));
    const char* le = nl ? nl : end;
    const char* lend = le;
    if (lend > p && lend[-1] == '\r') --lend;
    uint32_t i, j;
    double k;
    const int r = parse_ijk(p, lend, i, j, k);
    if (r < 0) fail(TAMC_E_PARSE, "instance line " + std::to_string(lineno) + ": integer does not fit in u32");
    if (r > 0) {
      nrows = std::max<uint64_t>(nrows, (uint64_t)std::max(i, j) + 1);
      const float kf = (float)k;
      ent.push_back({i, j, kf, seq++});
      if (i != j) ent.push_back({j, i, kf, seq++});
    }
    ++lineno;
    p = nl ? nl + 1 : end;
  }
  std::sort(ent.begin(), ent.end(), [](const E& a, const E& b) {
    if (a.r != b.r) return a.r < b.r;
    if (a.c != b.c) return a.c < b.c;
    return a.seq < b.seq;
  });
  size_t w = 0;
  for (size_t t = 0; t < ent.size(); ++t) {
    if (w > 0 && ent[w - 1].r == ent[t].r && ent[w - 1].c == ent[t].c) ent[w - 1] = ent[t];
    else ent[w++] = ent[t];
  }
  ent.resize(w);
  if (nrows > 0xffffffffull) fail(TAMC_E_PARSE, "instance too large");
  HostInstance h;
  h.n = (uint32_t)nrows;
  h.bias.assign(h.n, 0.0f);
  h.row_ptr.assign((size_t)h.n + 1, 0);
  h.col.reserve(ent.size());
  h.J.reserve(ent.size());
  float offset = 0.0f;
  size_t t = 0;
  // BqmIsingInstance::from_instance_file (src/ising.rs:297-321), f32 arithmetic in row order.
  for (uint32_t i = 0; i < h.n; ++i) {
    for (; t < ent.size() && ent[t].r == i; ++t) {
      const uint32_t j = ent[t].c;
      const float K = ent[t].K;
      if (qubo) {
        if (i != j) {
          offset += K / 8.0f;
          h.col.push_back(j);
          h.J.push_back(K / 4.0f);
          h.bias[i] += K / 4.0f;
        } else {
          offset += K / 2.0f;
          h.bias[i] += K / 2.0f;
          h.col.push_back(j);
          h.J.push_back(K / 2.0f);
        }
      } else {
        if (i != j) {
          h.col.push_back(j);
          h.J.push_back(K);
        } else {
          h.bias[i] = K;
        }
      }
    }
    h.row_ptr[i + 1] = (uint32_t)h.col.size();
  }
  h.offset = offset;
  out = std::move(h);
}

uint32_t HostInstance::graph_nodes() const {
  uint32_t mx = 0;
  bool any = false;
  for (uint32_t i = 0; i < n; ++i)
    for (uint32_t e = row_ptr[i]; e < row_ptr[i + 1]; ++e)
      if (col[e] != i || diag_in_graph) {
        any = true;
        mx = std::max(mx, std::max(i, col[e]));
      }
  return any ? mx + 1 : 0;
}

HostInstance induced_sorted(const HostInstance& h, const std::vector<uint32_t>& nodes) {
  HostInstance s;
  s.n = (uint32_t)nodes.size();
  s.offset = 0.0f;
  s.diag_in_graph = true;
  s.row_ptr.assign(1, 0);
  s.bias.reserve(s.n);
  for (uint32_t ni : nodes) {
    s.bias.push_back(h.bias[ni]);
    for (uint32_t e = h.row_ptr[ni]; e < h.row_ptr[ni + 1]; ++e) {
      const auto it = std::lower_bound(nodes.begin(), nodes.end(), h.col[e]);
      if (it != nodes.end() && *it == h.col[e]) {
        s.col.push_back((uint32_t)(it - nodes.begin()));
        s.J.push_back(h.J[e]);
      }
    }
    s.row_ptr.push_back((uint32_t)s.col.size());
  }
  for (const auto& w : h.suscept) {
    std::vector<double> sw;
    sw.reserve(s.n);
    for (uint32_t ni : nodes) sw.push_back(w[ni]);
    s.suscept.push_back(std::move(sw));
  }
  return s;
}

bool HostInstance::has_self_loops() const {
  for (uint32_t i = 0; i < n; ++i)
    for (uint32_t e = row_ptr[i]; e < row_ptr[i + 1]; ++e)
      if (col[e] == i) return true;
  return false;
}

float HostInstance::energy_ref(const int8_t* s) const {
  float total = offset;
  for (uint32_t i = 0; i < n; ++i) {
    float h = 0.0f;
    const float si = (float)s[i];
    h += bias[i];
    for (uint32_t e = row_ptr[i]; e < row_ptr[i + 1]; ++e) h += (J[e] * (float)s[col[e]]) / 2.0f;
    total += h * si;
  }
  return total;
}

void HostInstance::coloring(uint32_t& ncolors, std::vector<uint32_t>& color) const {
  const uint32_t UN = 0xffffffffu;
  color.assign(n, UN);
  // 1) bipartite BFS 2-colouring (checkerboard on even lattices)
  bool bip = true;
  std::vector<uint32_t> q;
  q.reserve(n);
  for (uint32_t s = 0; s < n && bip; ++s) {
    if (color[s] != UN) continue;
    color[s] = 0;
    q.clear();
    q.push_back(s);
    for (size_t h = 0; h < q.size() && bip; ++h) {
      const uint32_t u = q[h];
      for (uint32_t e = row_ptr[u]; e < row_ptr[u + 1]; ++e) {
        const uint32_t v = col[e];
        if (v == u) continue;
        if (color[v] == UN) {
          color[v] = color[u] ^ 1u;
          q.push_back(v);
        } else if (color[v] == color[u]) {
          bip = false;
          break;
        }
      }
    }
  }
  if (bip) {
    // isolated vertices / unbalanced components: rebalance free choices
    ncolors = n > 1 ? 2 : 1;
    if (n == 1) color[0] = 0;
    return;
  }
  // 2) largest-degree-first greedy
  color.assign(n, UN);
  std::vector<uint32_t> order(n);
  std::iota(order.begin(), order.end(), 0u);
  std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
    return (row_ptr[a + 1] - row_ptr[a]) > (row_ptr[b + 1] - row_ptr[b]);
  });
  std::vector<uint32_t> mark;
  uint32_t nc = 0;
  std::vector<uint32_t> csize;
  for (uint32_t u : order) {
    mark.assign(nc + 1, 0);
    for (uint32_t e = row_ptr[u]; e < row_ptr[u + 1]; ++e) {
      const uint32_t v = col[e];
      if (v != u && color[v] != UN && color[v] <= nc) mark[color[v]] = 1;
    }
    uint32_t c = 0;
    while (c < nc && mark[c]) ++c;
    // among admissible colours prefer the smallest class (equitable tendency)
    for (uint32_t c2 = c + 1; c2 < nc; ++c2)
      if (!mark[c2] && csize[c2] < csize[c]) c = c2;
    if (c == nc) {
      ++nc;
      csize.push_back(0);
    }
    color[u] = c;
    csize[c]++;
  }
  // 3) equitable rebalancing: move vertices from classes above the mean into
  //    admissible classes below it.
  const uint32_t target = (n + nc - 1) / nc;
  for (int pass = 0; pass < 4; ++pass) {
    bool moved = false;
    for (uint32_t u = 0; u < n; ++u) {
      const uint32_t cu = color[u];
      if (csize[cu] <= target) continue;
      mark.assign(nc, 0);
      for (uint32_t e = row_ptr[u]; e < row_ptr[u + 1]; ++e) {
        const uint32_t v = col[e];
        if (v != u) mark[color[v]] = 1;
      }
      uint32_t best = cu;
      for (uint32_t c = 0; c < nc; ++c)
        if (!mark[c] && csize[c] + 1 < csize[best]) best = c;
      if (best != cu) {
        csize[cu]--;
        csize[best]++;
        color[u] = best;
        moved = true;
      }
    }
    if (!moved) break;
  }
  ncolors = nc;
}

// read_txt_vec (src/util.rs:112-139): one fixed-point number per line after
// optional leading spaces; other lines are ignored.
std::vector<double> read_txt_vec_file(const std::string& path) {
  std::ifstream f(path, std::ios::binary);
  if (!f) fail(TAMC_E_IO, "cannot open susceptibility file '" + path + "'");
  std::vector<double> out;
  std::string line;
  while (std::getline(f, line)) {
    if (!line.empty() && line.back() == '\r') line.pop_back();
    const char* p = line.c_str();
    const char* end = p + line.size();
    while (p < end && is_sp(*p)) ++p;
    const char* s = p;
    if (p < end && *p == '-') ++p;
    const char* d = p;
    while (p < end && *p >= '0' && *p <= '9') ++p;
    if (p == d) continue;
    if (p < end && *p == '.') {
      ++p;
      while (p < end && *p >= '0' && *p <= '9') ++p;
    }
    out.push_back(strtod(std::string(s, p).c_str(), nullptr));
  }
  return out;
}

}  // namespace tamc

using namespace tamc;

extern "C" {

const char* tamc_last_error(void) { return tamc::g_last_error.c_str(); }
const char* tamc_version(void) { return "tamc_b200 1.0 (sm_100a)"; }

int tamc_instance_parse(const char* text, uint64_t len, int qubo, tamc_host_instance** out) {
  TAMC_API_BEGIN
  if (!out || (!text && len)) fail(TAMC_E_INVAL, "null argument");
  auto* h = new tamc_host_instance();
  try {
    parse_instance_text(text, (size_t)len, qubo != 0, h->h);
  } catch (...) {
    delete h;
    throw;
  }
  *out = h;
  TAMC_API_END
}

int tamc_instance_read(const char* path, int qubo, tamc_host_instance** out) {
  TAMC_API_BEGIN
  if (!path || !out) fail(TAMC_E_INVAL, "null argument");
  std::ifstream f(path, std::ios::binary);
  if (!f) fail(TAMC_E_IO, std::string("Unable to read adjacency from instance file '") + path + "'");
  std::stringstream ss;
  ss << f.rdbuf();
  const std::string s = ss.str();
  return tamc_instance_parse(s.data(), s.size(), qubo, out);
  TAMC_API_END
}

int tamc_instance_from_csr(uint32_t n, const uint32_t* row_ptr, const uint32_t* col, const float* J,
                           const float* bias, float offset, tamc_host_instance** out) {
  TAMC_API_BEGIN
  if (!row_ptr || !out || (n && !bias)) fail(TAMC_E_INVAL, "null argument");
  if (row_ptr[0] != 0) fail(TAMC_E_INVAL, "row_ptr[0] must be 0");
  for (uint32_t i = 0; i < n; ++i)
    if (row_ptr[i + 1] < row_ptr[i]) fail(TAMC_E_INVAL, "row_ptr must be non-decreasing");
  const uint32_t nnz = row_ptr[n];
  if (nnz && (!col || !J)) fail(TAMC_E_INVAL, "null argument");
  for (uint32_t e = 0; e < nnz; ++e)
    if (col[e] >= n) fail(TAMC_E_INVAL, "column index out of range");
  auto* h = new tamc_host_instance();
  h->h.n = n;
  h->h.offset = offset;
  h->h.row_ptr.assign(row_ptr, row_ptr + n + 1);
  h->h.col.assign(col, col + nnz);
  h->h.J.assign(J, J + nnz);
  h->h.bias.assign(bias, bias + n);
  *out = h;
  TAMC_API_END
}

int tamc_instance_add_suscept_file(tamc_host_instance* inst, const char* path) {
  TAMC_API_BEGIN
  if (!inst || !path) fail(TAMC_E_INVAL, "null argument");
  std::vector<double> v = read_txt_vec_file(path);
  if (v.size() != inst->h.n)
    fail(TAMC_E_INVAL, std::string("suscept file ") + path + " - Expected " + std::to_string(inst->h.n) +
                           " coefficients, but got " + std::to_string(v.size()));
  inst->h.suscept.push_back(std::move(v));
  TAMC_API_END
}

int tamc_instance_add_suscept(tamc_host_instance* inst, const double* w, uint32_t n) {
  TAMC_API_BEGIN
  if (!inst || (n && !w)) fail(TAMC_E_INVAL, "null argument");
  if (n != inst->h.n) fail(TAMC_E_INVAL, "suscept vector length must equal the instance size");
  inst->h.suscept.emplace_back(w, w + n);
  TAMC_API_END
}

int tamc_instance_dims(const tamc_host_instance* inst, uint32_t* n, uint64_t* nnz, float* offset, uint32_t* nchi) {
  TAMC_API_BEGIN
  if (!inst) fail(TAMC_E_INVAL, "null instance");
  if (n) *n = inst->h.n;
  if (nnz) *nnz = inst->h.col.size();
  if (offset) *offset = inst->h.offset;
  if (nchi) *nchi = (uint32_t)inst->h.suscept.size();
  TAMC_API_END
}

int tamc_instance_csr(const tamc_host_instance* inst, uint32_t* row_ptr, uint32_t* col, float* J, float* bias) {
  TAMC_API_BEGIN
  if (!inst) fail(TAMC_E_INVAL, "null instance");
  const auto& h = inst->h;
  if (row_ptr) memcpy(row_ptr, h.row_ptr.data(), h.row_ptr.size() * 4);
  if (col && !h.col.empty()) memcpy(col, h.col.data(), h.col.size() * 4);
  if (J && !h.J.empty()) memcpy(J, h.J.data(), h.J.size() * 4);
  if (bias && h.n) memcpy(bias, h.bias.data(), h.bias.size() * 4);
  TAMC_API_END
}

uint32_t tamc_instance_graph_nodes(const tamc_host_instance* inst) { return inst ? inst->h.graph_nodes() : 0; }

int tamc_instance_coloring(const tamc_host_instance* inst, uint32_t* ncolors, uint32_t* color) {
  TAMC_API_BEGIN
  if (!inst || !ncolors) fail(TAMC_E_INVAL, "null argument");
  std::vector<uint32_t> c;
  inst->h.coloring(*ncolors, c);
  if (color && !c.empty()) memcpy(color, c.data(), c.size() * 4);
  TAMC_API_END
}

float tamc_instance_energy_ref(const tamc_host_instance* inst, const int8_t* spins) {
  return inst->h.energy_ref(spins);
}

void tamc_instance_free(tamc_host_instance* inst) { delete inst; }

}  // extern "C"

namespace tamc {

void parse_partition(const char* text, size_t len, uint32_t n, std::vector<std::vector<uint32_t>>& parts) {
  parts.clear();
  std::vector<char> in_part(n, 0);
  const char* p = text;
  const char* end = text + len;
  while (p < end) {
    const char* eol = static_cast<const char*>(memchr(p, '\n', (size_t)(end - p)));
    if (!eol) eol = end;
    // one line: many1(delimited(space0, digit1 as u32, multispace0)); a line
    // without a leading number is skipped, text after the last number ignored
    std::vector<uint32_t> v;
    const char* q = p;
    for (;;) {
      const char* r = q;
      while (r < eol && (*r == ' ' || *r == '\t')) ++r;
      if (r >= eol || *r < '0' || *r > '9') break;
      uint64_t x = 0;
      while (r < eol && *r >= '0' && *r <= '9') {
        x = x * 10 + (uint64_t)(*r - '0');
        // u32::from_str(..).unwrap() on the digits
        if (x > 0xffffffffull) fail(TAMC_E_REFPANIC, "partition index does not fit in u32 (the reference panics)");
        ++r;
      }
      while (r < eol && (*r == ' ' || *r == '\t' || *r == '\r')) ++r;
      v.push_back((uint32_t)x);
      q = r;
    }
    if (!v.empty()) {
      const uint32_t ip = (uint32_t)parts.size();
      for (uint32_t i : v) {
        if (i >= n)
          fail(TAMC_E_INVAL, "Partitition must be specified for instance size " + std::to_string(n) +
                                 ". Found index " + std::to_string(i));
        if (in_part[i])
          fail(TAMC_E_INVAL, "Index " + std::to_string(i) + " specified more than once in partition " +
                                 std::to_string(ip));
        in_part[i] = 1;
      }
      parts.push_back(std::move(v));
    }
    p = eol + 1;
  }
}

}  // namespace tamc
