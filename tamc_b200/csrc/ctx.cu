// ctx.cu -- device contexts and device-resident instances.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "device.cuh"

extern "C" const unsigned char tamc_expf_blob_begin[];
extern "C" const unsigned char tamc_expf_blob_end[];

namespace tamc {

std::atomic<uint64_t> g_h2d_bytes{0}, g_d2h_bytes{0};

static inline uint64_t sm64(uint64_t& st) {
  st += 0x9e3779b97f4a7c15ULL;
  uint64_t z = st;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

Xo xo_seed_from_u64(uint64_t seed) {
  uint64_t st = seed;
  Xo x;
  x.s0 = sm64(st);
  x.s1 = sm64(st);
  x.s2 = sm64(st);
  x.s3 = sm64(st);
  if (!(x.s0 | x.s1 | x.s2 | x.s3)) return xo_seed_from_u64(0);
  return x;
}

void xo_jump(Xo& x) {
  static const uint64_t J[4] = {0x180ec6d33cfd0abaULL, 0xd5a61266f0c9392cULL, 0xa9582618e03fc9aaULL,
                                0x39abdc4529b1661cULL};
  uint64_t t0 = 0, t1 = 0, t2 = 0, t3 = 0;
  for (int i = 0; i < 4; ++i)
    for (int b = 0; b < 64; ++b) {
      if (J[i] & (1ULL << b)) {
        t0 ^= x.s0;
        t1 ^= x.s1;
        t2 ^= x.s2;
        t3 ^= x.s3;
      }
      x.next();
    }
  x.s0 = t0;
  x.s1 = t1;
  x.s2 = t2;
  x.s3 = t3;
}

template <class T>
static T* dmalloc_copy(const T* h, size_t count) {
  T* d = nullptr;
  const size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
  TAMC_CUDA(cudaMalloc((void**)&d, bytes));
  if (count) TAMC_CUDA(copy_sync(d, h, count * sizeof(T), cudaMemcpyHostToDevice));
  return d;
}

// The arrays of one instance upload, packed at 256-byte offsets into one host
// staging buffer, then one device allocation and one copy.
struct UploadPack {
  std::vector<char> host;
  std::vector<std::pair<void**, size_t>> slots;
  template <class T>
  void add(T** slot, const T* h, size_t count) {
    const size_t off = (host.size() + 255) & ~(size_t)255;
    const size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
    host.resize(off + bytes, 0);
    if (count) memcpy(host.data() + off, h, count * sizeof(T));
    slots.emplace_back(reinterpret_cast<void**>(slot), off);
  }
  void commit(void*& arena, size_t& bytes) {
    bytes = host.size();
    arena = dev_alloc(bytes);
    TAMC_CUDA(copy_sync(arena, host.data(), bytes, cudaMemcpyHostToDevice));
    bind(arena);
  }
  // the arrays' device addresses inside `arena`
  void bind(void* arena) {
    for (auto& s : slots) *s.first = static_cast<char*>(arena) + s.second;
  }
};

// ---------------------------------------------------- device-memory cache ----
namespace {
std::mutex g_cache_mu;
struct DevCache {
  std::map<size_t, std::vector<void*>> ready, pending;
  size_t bytes = 0;
};
std::map<int, DevCache> g_cache;
constexpr size_t kCacheMaxBlock = 8u << 20;      // larger blocks bypass the cache
constexpr size_t kCacheMaxBytes = 1ull << 30;    // per device
size_t size_class(size_t b) {
  size_t c = 256;
  while (c < b) c <<= 1;
  return c;
}
void free_all_locked(DevCache& C) {
  for (auto* m : {&C.ready, &C.pending})
    for (auto& kv : *m)
      for (void* p : kv.second) cudaFree(p);
  C.ready.clear();
  C.pending.clear();
  C.bytes = 0;
}

// Side L when the coupling graph is exactly the periodic square (d = 2) or
// cubic (d = 3) lattice of side 16 or 32 in the file's site order (site
// x L^2 + y L + z, z fastest; every row the 2d neighbours at +-1 along each
// axis modulo L, in any order, no self-coupling), else 0.  Rows of such a
// lattice fill half or whole 32-bit words, which the plain form's bitmap
// Houdayer search relies on.
uint32_t lattice_side(const HostInstance& h, uint32_t udeg) {
  if (udeg != 4 && udeg != 6) return 0;
  const uint32_t d = udeg / 2;
  for (uint32_t L : {16u, 32u}) {
    const uint64_t n = d == 2 ? (uint64_t)L * L : (uint64_t)L * L * L;
    if (n != h.n) continue;
    for (uint32_t i = 0; i < h.n; ++i) {
      const uint32_t r0 = h.row_ptr[i], r1 = h.row_ptr[i + 1];
      if (r1 - r0 != udeg) return 0;
      uint32_t want[6];
      uint32_t k = 0, stride = 1;
      for (uint32_t a = 0; a < d; ++a, stride *= L) {
        const uint32_t c = (i / stride) % L;
        want[k++] = i - c * stride + ((c + 1) % L) * stride;
        want[k++] = i - c * stride + ((c + L - 1) % L) * stride;
      }
      std::sort(want, want + udeg);
      uint32_t got[6];
      for (uint32_t e = 0; e < udeg; ++e) got[e] = h.col[r0 + e];
      std::sort(got, got + udeg);
      for (uint32_t e = 0; e < udeg; ++e)
        if (got[e] != want[e]) return 0;
    }
    return L;
  }
  return 0;
}
}  // namespace

void* dev_alloc(size_t bytes) {
  bytes = std::max<size_t>(bytes, 1);
  void* p = nullptr;
  if (bytes > kCacheMaxBlock) {
    if (cudaMalloc(&p, bytes) != cudaSuccess) fail(TAMC_E_NOMEM, "device allocation failed");
    return p;
  }
  int dev = 0;
  TAMC_CUDA(cudaGetDevice(&dev));
  const size_t c = size_class(bytes);
  {
    std::lock_guard<std::mutex> lk(g_cache_mu);
    DevCache& C = g_cache[dev];
    for (int attempt = 0; attempt < 2; ++attempt) {
      auto it = C.ready.find(c);
      if (it != C.ready.end() && !it->second.empty()) {
        p = it->second.back();
        it->second.pop_back();
        C.bytes -= c;
        return p;
      }
      if (attempt == 0 && !C.pending.empty()) {
        // freed blocks become reusable once nothing in flight can still read them
        TAMC_CUDA(cudaDeviceSynchronize());
        for (auto& kv : C.pending) {
          auto& r = C.ready[kv.first];
          r.insert(r.end(), kv.second.begin(), kv.second.end());
        }
        C.pending.clear();
      }
    }
  }
  if (cudaMalloc(&p, c) != cudaSuccess) {
    cudaGetLastError();
    {
      std::lock_guard<std::mutex> lk(g_cache_mu);
      cudaDeviceSynchronize();
      free_all_locked(g_cache[dev]);
    }
    if (cudaMalloc(&p, c) != cudaSuccess) fail(TAMC_E_NOMEM, "device allocation failed");
  }
  return p;
}

void dev_free(void* p, size_t bytes) {
  if (!p) return;
  bytes = std::max<size_t>(bytes, 1);
  if (bytes > kCacheMaxBlock) {
    cudaFree(p);
    return;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return;
  const size_t c = size_class(bytes);
  std::lock_guard<std::mutex> lk(g_cache_mu);
  DevCache& C = g_cache[dev];
  if (C.bytes + c > kCacheMaxBytes) {
    cudaFree(p);
    return;
  }
  C.pending[c].push_back(p);
  C.bytes += c;
}

void dev_cache_release(int device) {
  std::lock_guard<std::mutex> lk(g_cache_mu);
  auto it = g_cache.find(device);
  if (it == g_cache.end()) return;
  cudaDeviceSynchronize();
  free_all_locked(it->second);
  g_cache.erase(it);
}

}  // namespace tamc

using namespace tamc;

void tamc_gpu_retain(tamc_gpu* g) { g->refs.fetch_add(1); }
void tamc_gpu_release(tamc_gpu* g) {
  if (g->refs.fetch_sub(1) != 1) return;
  cudaSetDevice(g->device);
  cudaStreamSynchronize(g->stream);
  runner_pool_release(g);
  cudaFree(g->d_exp);
  cudaStreamDestroy(g->stream);
  if (g->up_stream) cudaStreamDestroy(g->up_stream);
  if (g->up_pin) cudaFreeHost(g->up_pin);
  dev_cache_release(g->device);
  delete g;
}
void tamc_inst_retain(tamc_inst* d) { d->refs.fetch_add(1); }
void tamc_inst_release(tamc_inst* d) {
  if (d->refs.fetch_sub(1) != 1) return;
  tamc_gpu* g = d->g;
  cudaSetDevice(g->device);
  if (d->arena) dev_free(d->arena, d->arena_bytes);  // holds every array of the instance
  d->sa_scratch.release();
  delete d;
  tamc_gpu_release(g);
}

// Host side of an upload: every array of the instance (reference order, ICM
// graph, colour order, lattice layouts) into `pack`, and the host fields of
// `d`.  Touches no device state, so uploads of several instances prepare in
// parallel.
static void inst_prepare(tamc_inst* d, const HostInstance& h, UploadPack& pack) {
  d->host = h;
  d->n = h.n;
  d->nnz = h.col.size();
  d->offset = h.offset;
  d->nchi = (uint32_t)h.suscept.size();
  d->self_loops = h.has_self_loops();
  for (uint32_t i = 0; i < h.n; ++i) d->max_deg = std::max(d->max_deg, h.row_ptr[i + 1] - h.row_ptr[i]);
  pack.add(&d->d_rp, h.row_ptr.data(), h.row_ptr.size());
  pack.add(&d->d_col, h.col.data(), h.col.size());
  pack.add(&d->d_J, h.J.data(), h.J.size());
  pack.add(&d->d_bias, h.bias.data(), h.bias.size());
  // ICM graph: off-diagonal entries over the petgraph node range
  d->g_nodes = h.graph_nodes();
  std::vector<uint32_t> grp(d->g_nodes + 1, 0), gcol;
  for (uint32_t i = 0; i < d->g_nodes; ++i) {
    for (uint32_t e = h.row_ptr[i]; e < h.row_ptr[i + 1]; ++e)
      if (h.col[e] != i) gcol.push_back(h.col[e]);
    grp[i + 1] = (uint32_t)gcol.size();
  }
  pack.add(&d->d_grp, grp.data(), grp.size());
  pack.add(&d->d_gcol, gcol.data(), gcol.size());
  std::vector<double> sus((size_t)d->nchi * h.n);
  for (uint32_t k = 0; k < d->nchi; ++k) std::copy(h.suscept[k].begin(), h.suscept[k].end(), sus.begin() + (size_t)k * h.n);
  pack.add(&d->d_sus, sus.data(), sus.size());
  // colour order
  std::vector<uint32_t> color;
  h.coloring(d->ncolors, color);
  if (h.n == 0) d->ncolors = 0;
  d->color_off.assign(d->ncolors + 1, 0);
  for (uint32_t i = 0; i < h.n; ++i) d->color_off[color[i] + 1]++;
  for (uint32_t c = 0; c < d->ncolors; ++c) d->color_off[c + 1] += d->color_off[c];
  std::vector<uint32_t> fill(d->color_off.begin(), d->color_off.end() - (d->ncolors ? 1 : 0));
  d->h_perm.assign(h.n, 0);
  std::vector<uint32_t> iperm(h.n);
  for (uint32_t i = 0; i < h.n; ++i) {
    const uint32_t s = fill[color[i]]++;
    d->h_perm[s] = i;
    iperm[i] = s;
  }
  std::vector<uint32_t> frp(h.n + 1, 0);
  std::vector<uint2> fent;
  fent.reserve(h.col.size());
  std::vector<float> fbias(h.n), fkd(h.n, 0.0f);
  std::vector<double> fsus((size_t)d->nchi * h.n);
  for (uint32_t s = 0; s < h.n; ++s) {
    const uint32_t i = d->h_perm[s];
    fbias[s] = h.bias[i];
    for (uint32_t e = h.row_ptr[i]; e < h.row_ptr[i + 1]; ++e) {
      uint32_t jb;
      memcpy(&jb, &h.J[e], 4);
      fent.push_back(make_uint2(iperm[h.col[e]], jb));
      if (h.col[e] == i) fkd[s] += h.J[e];
    }
    frp[s + 1] = (uint32_t)fent.size();
    for (uint32_t k = 0; k < d->nchi; ++k) fsus[(size_t)k * h.n + s] = h.suscept[k][i];
  }
  pack.add(&d->d_color_off, d->color_off.data(), d->color_off.size());
  pack.add(&d->d_perm, d->h_perm.data(), d->h_perm.size());
  pack.add(&d->d_iperm, iperm.data(), iperm.size());
  pack.add(&d->d_frp, frp.data(), frp.size());
  d->udeg = h.n ? frp[1] : 0;
  for (uint32_t s = 0; s < h.n && d->udeg; ++s)
    if (frp[s + 1] - frp[s] != d->udeg) d->udeg = 0;
  pack.add(&d->d_fent, fent.data(), fent.size());
  if (h.n <= 65536) {
    std::vector<uint16_t> c16((fent.size() + 7) / 8 * 8 + 8, 0);
    for (size_t e = 0; e < fent.size(); ++e) c16[e] = (uint16_t)fent[e].x;
    pack.add(&d->d_fcol16, c16.data(), c16.size());
  }
  // +-J instances (every coupling +-1, no field, no self-coupling, rows of 4 or
  // 6 entries) take the multi-spin-coded sweep of the colour-ordered mode
  d->pmj = (d->udeg == 4 || d->udeg == 6) && !d->self_loops;
  for (uint32_t s = 0; s < h.n && d->pmj; ++s)
    if (fbias[s] != 0.0f) d->pmj = 0;
  for (size_t e = 0; e < fent.size() && d->pmj; ++e)
    if ((fent[e].y & 0x7fffffffu) != 0x3f800000u) d->pmj = 0;  // |J| == 1.0f
  d->lat_L = lattice_side(h, d->udeg);
  std::vector<float> fJt;
  std::vector<uint16_t> fcolt;
  if (d->lat_L) {
    // couplings and columns by (neighbour slot, colour row) for the bitmap
    // Houdayer kernel: contiguous 16-byte staging, conflict-free reads of
    // the m-th entries of consecutive rows
    const uint32_t D = d->udeg;
    fJt.resize(fent.size());
    fcolt.resize(fent.size());
    for (uint32_t s = 0; s < h.n; ++s)
      for (uint32_t m = 0; m < D; ++m) {
        memcpy(&fJt[(size_t)m * h.n + s], &fent[(size_t)s * D + m].y, 4);
        fcolt[(size_t)m * h.n + s] = (uint16_t)fent[(size_t)s * D + m].x;
      }
    pack.add(&d->d_fJt, fJt.data(), fJt.size());
    pack.add(&d->d_fcolt, fcolt.data(), fcolt.size());
  }
  pack.add(&d->d_fbias, fbias.data(), fbias.size());
  pack.add(&d->d_fkd, fkd.data(), fkd.size());
  pack.add(&d->d_fsus, fsus.data(), fsus.size());
}

extern "C" {

int tamc_gpu_open(int device, tamc_gpu** out) {
  TAMC_API_BEGIN
  if (!out) fail(TAMC_E_INVAL, "null output");
  int ndev = 0;
  TAMC_CUDA(cudaGetDeviceCount(&ndev));
  if (device < 0 || device >= ndev) fail(TAMC_E_INVAL, "no such CUDA device");
  TAMC_CUDA(cudaSetDevice(device));
  cudaDeviceProp prop;
  TAMC_CUDA(cudaGetDeviceProperties(&prop, device));
  if (prop.major < 10) fail(TAMC_E_UNSUPPORTED, "this library is built for sm_100a (B200)");
  auto* g = new tamc_gpu();
  g->device = device;
  g->num_sms = prop.multiProcessorCount;
  // dynamic shared memory a launch may ask for: the opt-in limit less 1 KB for
  // the kernels' static shared memory (job descriptor copies, counters)
  g->smem_optin = prop.sharedMemPerBlockOptin - 1024;
  try {
    TAMC_CUDA(cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking));
    const size_t blob = (size_t)(tamc_expf_blob_end - tamc_expf_blob_begin);
    uint32_t hdr[3];
    if (blob < 12) fail(TAMC_E_INVAL, "expf table missing from the library");
    memcpy(hdr, tamc_expf_blob_begin, 12);
    if (hdr[0] != 0x54505845u || hdr[1] != TAMC_EXPF_NUM_BUCKETS ||
        blob != 12 + 4 * ((size_t)hdr[1] + 1 + 2 * (size_t)hdr[2]))
      fail(TAMC_E_INVAL, "corrupt expf table in the library");
    g->d_exp = dmalloc_copy((const uint32_t*)(tamc_expf_blob_begin + 12), (blob - 12) / 4);
    g->exp.off = g->d_exp;
    g->exp.keys = g->d_exp + hdr[1] + 1;
    g->exp.vals = g->exp.keys + hdr[2];
  } catch (...) {
    if (g->stream) cudaStreamDestroy(g->stream);
    delete g;
    throw;
  }
  *out = g;
  TAMC_API_END
}

int tamc_gpu_close(tamc_gpu* g) {
  TAMC_API_BEGIN
  if (!g) return TAMC_OK;
  tamc_gpu_release(g);
  TAMC_API_END
}

int tamc_gpu_sync(tamc_gpu* g) {
  TAMC_API_BEGIN
  if (!g) fail(TAMC_E_INVAL, "null context");
  TAMC_CUDA(cudaStreamSynchronize(g->stream));
  TAMC_API_END
}

float tamc_ref_expf(float x) {
  const uint32_t* blob = (const uint32_t*)tamc_expf_blob_begin;
  const uint32_t nb = blob[1], ne = blob[2];
  const uint32_t* off = blob + 3;
  return tamc_expf_exact(x, off, off + nb + 1, off + nb + 1 + ne);
}

void tamc_copy_bytes(uint64_t* h2d, uint64_t* d2h) {
  if (h2d) *h2d = g_h2d_bytes.load();
  if (d2h) *d2h = g_d2h_bytes.load();
}

void* tamc_gpu_stream(tamc_gpu* g) { return g ? (void*)g->stream : nullptr; }
uint64_t tamc_gpu_launch_count(tamc_gpu* g) { return g ? g->launches.load() : 0; }

int tamc_gpu_instance_upload(tamc_gpu* g, const tamc_host_instance* hi, tamc_inst** out) {
  TAMC_API_BEGIN
  TraceRange tr("tamc upload");
  if (!g || !hi || !out) fail(TAMC_E_INVAL, "null argument");
  // an instance without sites has nothing to sample; refused here rather than
  // launching empty grids
  if (hi->h.n == 0) fail(TAMC_E_INVAL, "instance has no sites");
  TAMC_CUDA(cudaSetDevice(g->device));
  auto* d = new tamc_inst();
  d->g = g;
  tamc_gpu_retain(g);
  try {
    UploadPack pack;
    inst_prepare(d, hi->h, pack);
    pack.commit(d->arena, d->arena_bytes);
  } catch (...) {
    tamc_gpu_instance_destroy(d);
    throw;
  }
  *out = d;
  TAMC_API_END
}

int tamc_gpu_instance_upload_many(tamc_gpu* g, uint32_t count, const tamc_host_instance* const* his,
                                  tamc_inst** outs) {
  TAMC_API_BEGIN
  TraceRange tr("tamc upload_many");
  if (!g || (count && (!his || !outs))) fail(TAMC_E_INVAL, "null argument");
  for (uint32_t k = 0; k < count; ++k) {
    if (!his[k]) fail(TAMC_E_INVAL, "null instance at index " + std::to_string(k));
    if (his[k]->h.n == 0) fail(TAMC_E_INVAL, "instance at index " + std::to_string(k) + " has no sites");
  }
  if (count == 0) return TAMC_OK;
  TAMC_CUDA(cudaSetDevice(g->device));
  std::vector<tamc_inst*> ds(count, nullptr);
  auto drop_all = [&] {
    if (g->up_stream) cudaStreamSynchronize(g->up_stream);  // no copy still reads the staging block
    for (tamc_inst* d : ds)
      if (d) tamc_gpu_instance_destroy(d);
  };
  try {
    for (uint32_t k = 0; k < count; ++k) {
      ds[k] = new tamc_inst();
      ds[k]->g = g;
      tamc_gpu_retain(g);
    }
    // on up to 16 threads: host preparation of every instance, then (after
    // the staging offsets are known) its copy into the pinned staging block
    std::vector<UploadPack> packs(count);
    std::vector<size_t> off(count + 1, 0);
    std::vector<std::exception_ptr> errs(count);
    const uint32_t hw = std::max(1u, std::thread::hardware_concurrency());
    auto parallel = [&](uint32_t k0, uint32_t k1, auto&& f) {
      std::atomic<uint32_t> next{k0};
      auto work = [&] {
        for (uint32_t k; (k = next.fetch_add(1)) < k1;) {
          try {
            f(k);
          } catch (...) {
            errs[k] = std::current_exception();
          }
        }
      };
      std::vector<std::thread> pool;
      for (uint32_t t = 1; t < std::min({k1 - k0, hw, 16u}); ++t) {
        try {
          pool.emplace_back(work);
        } catch (...) {
          break;  // no more threads: the ones running and this one share the work
        }
      }
      work();
      for (auto& th : pool) th.join();
      for (uint32_t k = k0; k < k1; ++k)
        if (errs[k]) std::rethrow_exception(errs[k]);
    };
    parallel(0, count, [&](uint32_t k) { inst_prepare(ds[k], his[k]->h, packs[k]); });
    for (uint32_t k = 0; k < count; ++k) off[k + 1] = off[k] + ((packs[k].host.size() + 255) & ~(size_t)255);
    // staged in rounds of at most `cap` bytes (one instance at least): fill
    // the block, one device allocation and one asynchronous copy per instance
    // on the upload stream, one wait; the instances are complete on return,
    // as after tamc_gpu_instance_upload
    size_t cap = (size_t)256 << 20;
    if (const char* e = getenv("TAMC_UPLOAD_STAGE_BYTES")) cap = std::max<size_t>(256, strtoull(e, nullptr, 10));
    std::lock_guard<std::mutex> lk(g->up_mu);
    if (!g->up_stream) TAMC_CUDA(cudaStreamCreateWithFlags(&g->up_stream, cudaStreamNonBlocking));
    for (uint32_t k0 = 0, k1; k0 < count; k0 = k1) {
      k1 = k0 + 1;
      while (k1 < count && off[k1 + 1] - off[k0] <= cap) ++k1;
      const size_t bytes = off[k1] - off[k0];
      if (bytes > g->up_pin_bytes) {
        if (g->up_pin) TAMC_CUDA(cudaFreeHost(g->up_pin));
        g->up_pin = nullptr;
        g->up_pin_bytes = 0;
        const size_t want = bytes > cap ? bytes : std::min(cap, bytes + bytes / 4);
        TAMC_CUDA(cudaHostAlloc((void**)&g->up_pin, want, cudaHostAllocDefault));
        g->up_pin_bytes = want;
      }
      auto pin = [&](uint32_t k) { return g->up_pin + (off[k] - off[k0]); };
      parallel(k0, k1, [&](uint32_t k) { memcpy(pin(k), packs[k].host.data(), packs[k].host.size()); });
      for (uint32_t k = k0; k < k1; ++k) {
        ds[k]->arena_bytes = packs[k].host.size();
        ds[k]->arena = dev_alloc(ds[k]->arena_bytes);
        TAMC_CUDA(copy_async(ds[k]->arena, pin(k), ds[k]->arena_bytes, cudaMemcpyHostToDevice, g->up_stream));
        packs[k].bind(ds[k]->arena);
      }
      TAMC_CUDA(cudaStreamSynchronize(g->up_stream));
    }
  } catch (...) {
    drop_all();
    throw;
  }
  for (uint32_t k = 0; k < count; ++k) outs[k] = ds[k];
  TAMC_API_END
}

int tamc_gpu_instance_destroy(tamc_inst* d) {
  TAMC_API_BEGIN
  if (!d) return TAMC_OK;
  tamc_inst_release(d);
  TAMC_API_END
}

}  // extern "C"
