// C ABI of libphotonprop_b200.so (declared in include/photonprop_b200.h).
//
// A context holds the device-resident physics tables, a stream, the device
// buffers of the host-buffer entry points, the work-queue scratch of the
// batched kernel, the tuned launch shape per mode and a small cache of
// instantiated CUDA graphs (scan -> batched kernel -> finalise) keyed by the
// call's shapes and buffers.
#include <cuda_runtime.h>

#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "pp_internal.h"

namespace pp {
static std::atomic<uint64_t> g_launches{0};
// Launches enqueued while a thread captures a graph run only when the graph
// is launched; they are counted then.
static thread_local bool g_capturing = false;
void count_launches(uint64_t n) {
  if (!g_capturing) g_launches.fetch_add(n, std::memory_order_relaxed);
}
}  // namespace pp

namespace {

thread_local std::string g_create_error;

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
};

// Grows a context buffer.  *grew is set when the buffer moved, which
// invalidates every cached graph (they hold raw pointers).
cudaError_t ensure(DevBuf& b, size_t bytes, bool* grew) {
  if (bytes == 0) bytes = 16;
  if (b.bytes >= bytes) return cudaSuccess;
  b.release();
  *grew = true;
  cudaError_t e = cudaMalloc(&b.p, bytes);
  if (e == cudaSuccess) b.bytes = bytes;
  return e;
}

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int d) {
    cudaGetDevice(&prev);
    if (prev != d) cudaSetDevice(d);
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

struct GraphKey {
  const void* pairs;
  int64_t n_pairs;
  const void* hits;
  int64_t cap;
  const void* counters;
  const void* stats;
  const void* hist;
  const void* stream;
  const void* offsets;
  const void* queue;
  int grid, block;
  uint32_t chunk;
  pp_run_opts opts;
  bool operator==(const GraphKey& o) const { return std::memcmp(this, &o, sizeof(GraphKey)) == 0; }
};

struct GraphEntry {
  GraphKey key;
  cudaGraphExec_t exec = nullptr;
  uint64_t last_use = 0;
};

constexpr int kGraphCache = 4;
constexpr int kKernelsPerBatch = 3;  // scan, batched, finalise

}  // namespace

struct pp_ctx {
  int device = 0;
  int sm_count = 0;
  std::string device_name;
  std::mutex mu;
  std::string err;
  std::vector<unsigned char> h_tables;
  void* d_tables = nullptr;
  void* d_casc = nullptr;  // cascade emitter tables (float)
  cudaStream_t stream = nullptr;
  // buffers of the host-buffer entry points
  DevBuf pairs, hits, counters, stats, hist;
  // work-queue scratch of the batched kernel
  DevBuf offsets, queue;
  // launch shape per mode (0 = resolve at launch)
  int tuned_block[2] = {256, 256};
  int tuned_bps[2] = {0, 0};
  int tuned_chunk[2] = {4096, 4096};
  GraphEntry graphs[kGraphCache];
  uint64_t graph_clock = 0;
  pp_medium_desc medium;
  pp_pmt_desc pmt;
  // fit stage: constants and device buffers
  pp::FitConsts fitk;
  DevBuf fit_counts, fit_rec, fit_moments, fit_out, fit_cs;
  DevBuf llh_chunks;  // event likelihood: first hit chunk of every module
  DevBuf pilot;       // fit waves: the pilot launch's pairs

  pp_status fail(pp_status s, const std::string& msg) {
    err = msg;
    return s;
  }
  pp_status cuda_fail(cudaError_t e, const char* where) {
    err = std::string(where) + ": " + cudaGetErrorString(e);
    return PP_ERR_CUDA;
  }
  void drop_graphs() {
    for (auto& g : graphs) {
      if (g.exec) cudaGraphExecDestroy(g.exec);
      g.exec = nullptr;
    }
  }
};

namespace {

pp_status validate_opts(pp_ctx* c, const pp_run_opts* o) {
  if (!o) return c->fail(PP_ERR_ARG, "opts is NULL");
  if (o->mode != PP_MODE_COMPAT && o->mode != PP_MODE_PHYSICAL) return c->fail(PP_ERR_ARG, "unknown mode");
  if (o->max_steps < 1 || o->max_steps > (1 << 24) - 2)
    return c->fail(PP_ERR_ARG, "max_steps must be in [1, 2^24 - 2] (the step is part of the Philox counter)");
  if (!(std::fabs(o->g) < 1.f)) return c->fail(PP_ERR_ARG, "|g| must be < 1");
  if (o->hist_bins < 0) return c->fail(PP_ERR_ARG, "hist_bins must be >= 0");
  if (o->hist_bins > 0 && !(o->hist_bin_width > 0.f)) return c->fail(PP_ERR_ARG, "hist_bin_width must be > 0");
  if (o->mode == PP_MODE_PHYSICAL && !std::isfinite(o->t_max)) return c->fail(PP_ERR_ARG, "t_max must be finite");
  if (o->block_size != 0 && (o->block_size < 32 || o->block_size > 512 || o->block_size % 32))
    return c->fail(PP_ERR_ARG, "block_size must be a multiple of 32 in [32, 512]");
  if (o->blocks_per_sm < 0 || o->chunk_photons < 0) return c->fail(PP_ERR_ARG, "negative launch tuning value");
  return PP_OK;
}

pp_status validate_pairs(pp_ctx* c, const pp_pair* p, int64_t n, int mode) {
  if (n < 0) return c->fail(PP_ERR_ARG, "n_pairs must be >= 0");
  if (n > 0 && !p) return c->fail(PP_ERR_ARG, "pairs is NULL");
  if (n > (int64_t)INT32_MAX) return c->fail(PP_ERR_ARG, "too many pairs");
  for (int64_t i = 0; i < n; ++i) {
    const pp_pair& q = p[i];
    char buf[160];
    if (q.n_photons < 0 || q.n_photons > (1ll << 40)) {
      snprintf(buf, sizeof buf, "pair %lld: n_photons must be in [0, 2^40]", (long long)i);
      return c->fail(PP_ERR_ARG, buf);
    }
    if (!(q.radius > 0.f) || !std::isfinite(q.radius)) {
      snprintf(buf, sizeof buf, "pair %lld: radius must be > 0", (long long)i);
      return c->fail(PP_ERR_ARG, buf);
    }
    if (q.emitter == PP_EMITTER_CHERENKOV_CONE || q.emitter == PP_EMITTER_CASCADE) {
      if (mode == PP_MODE_COMPAT) {
        snprintf(buf, sizeof buf,
                 "pair %lld: %s emission has no reference-compatible form "
                 "(the reference's initialize_direction throws ArgumentError)",
                 (long long)i, q.emitter == PP_EMITTER_CASCADE ? "cascade" : "Cherenkov-cone");
        return c->fail(PP_ERR_ARG, buf);
      }
      const float n2 = q.dir[0] * q.dir[0] + q.dir[1] * q.dir[1] + q.dir[2] * q.dir[2];
      if (!(std::fabs(n2 - 1.f) < 1e-3f) || !(q.track_len >= 0.f)) {
        snprintf(buf, sizeof buf, "pair %lld: cone and cascade emitters need a unit direction and track_len >= 0",
                 (long long)i);
        return c->fail(PP_ERR_ARG, buf);
      }
    } else if (q.emitter != PP_EMITTER_ISOTROPIC) {
      snprintf(buf, sizeof buf, "pair %lld: unknown emitter %d", (long long)i, q.emitter);
      return c->fail(PP_ERR_ARG, buf);
    }
  }
  return PP_OK;
}

bool any_cascade(const pp_pair* p, int64_t n) {
  for (int64_t i = 0; i < n; ++i)
    if (p[i].emitter == PP_EMITTER_CASCADE) return true;
  return false;
}

void resolve_launch(pp_ctx* c, const pp_run_opts& o, int& grid, int& block, uint32_t& chunk) {
  const int m = o.mode;
  block = o.block_size > 0 ? o.block_size : c->tuned_block[m];
  if (block != 128) block = 256;  // the batched kernel exists for 4- and 8-warp blocks
  int bps = o.blocks_per_sm > 0 ? o.blocks_per_sm : c->tuned_bps[m];
  const int maxb = pp::batched_max_blocks_per_sm(m, block, (o.flags & PP_OPT_CASCADE) != 0);
  if (bps <= 0 || bps > maxb) bps = maxb > 0 ? maxb : 1;
  grid = c->sm_count * bps;
  chunk = (uint32_t)(o.chunk_photons > 0 ? o.chunk_photons : c->tuned_chunk[m]);
}

// memset stats/hist, scan (resets queue and counters), batched kernel, finalise.
cudaError_t enqueue_batched(pp_ctx* c, const pp::LaunchArgs& a, int grid, int block, cudaStream_t s) {
  cudaError_t e;
  if (a.stats && (e = cudaMemsetAsync(a.stats, 0, (size_t)a.n_pairs * PP_STATS * sizeof(double), s))) return e;
  if (a.hist && a.opts.hist_bins > 0 &&
      (e = cudaMemsetAsync(a.hist, 0, (size_t)a.n_pairs * a.opts.hist_bins * sizeof(double), s)))
    return e;
  if ((e = pp::launch_chunk_scan(a, s))) return e;
  if ((e = pp::launch_batched(a, grid, block, s))) return e;
  return pp::launch_finalize(a.pairs, a.n_pairs, a.stats, a.hist, a.opts.hist_bins,
                             (a.opts.flags & PP_OPT_NORMALIZE) ? 1 : 0, c->sm_count, s);
}

// Replays a cached graph for this key or captures a new one.  Streams that
// cannot be captured (the legacy default stream) get direct launches.
cudaError_t run_batched(pp_ctx* c, const pp::LaunchArgs& a, cudaStream_t s, bool use_graph) {
  int grid, block;
  uint32_t chunk;
  resolve_launch(c, a.opts, grid, block, chunk);
  pp::LaunchArgs b = a;
  b.chunk = chunk;
  if (!use_graph || s == nullptr) return enqueue_batched(c, b, grid, block, s);
  GraphKey k;
  std::memset(&k, 0, sizeof k);
  k.pairs = b.pairs;
  k.n_pairs = b.n_pairs;
  k.hits = b.hits;
  k.cap = (int64_t)b.hit_cap;
  k.counters = b.counters;
  k.stats = b.stats;
  k.hist = b.hist;
  k.stream = s;
  k.offsets = b.chunk_offsets;
  k.queue = b.queue;
  k.grid = grid;
  k.block = block;
  k.chunk = chunk;
  k.opts = b.opts;
  for (auto& g : c->graphs) {
    if (g.exec && g.key == k) {
      g.last_use = ++c->graph_clock;
      pp::count_launches(kKernelsPerBatch);
      return cudaGraphLaunch(g.exec, s);
    }
  }
  cudaGraph_t graph = nullptr;
  cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
  if (e) return e;
  pp::g_capturing = true;
  cudaError_t le = enqueue_batched(c, b, grid, block, s);
  pp::g_capturing = false;
  e = cudaStreamEndCapture(s, &graph);
  if (le) {
    if (graph) cudaGraphDestroy(graph);
    return le;
  }
  if (e) return e;
  GraphEntry* slot = &c->graphs[0];
  for (auto& g : c->graphs) {
    if (!g.exec) {
      slot = &g;
      break;
    }
    if (g.last_use < slot->last_use) slot = &g;
  }
  if (slot->exec) cudaGraphExecDestroy(slot->exec);
  slot->exec = nullptr;
  e = cudaGraphInstantiate(&slot->exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e) {
    slot->exec = nullptr;
    return e;
  }
  slot->key = k;
  slot->last_use = ++c->graph_clock;
  pp::count_launches(kKernelsPerBatch);
  return cudaGraphLaunch(slot->exec, s);
}

pp::LaunchArgs base_args(pp_ctx* c, const pp_run_opts* o) {
  pp::LaunchArgs a;
  std::memset(&a, 0, sizeof a);
  a.tables = c->d_tables;
  a.opts = *o;
  return a;
}

bool aligned(const void* p, uintptr_t a) { return ((uintptr_t)p % a) == 0; }

size_t hit_bytes(const pp_run_opts* o) { return (o->flags & PP_OPT_COMPACT_HITS) ? sizeof(pp_hit32) : sizeof(pp_hit); }

pp_status alloc_fail(pp_ctx* c, cudaError_t e, const char* what) {
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();
    return c->fail(PP_ERR_OOM, std::string("device allocation failed: ") + what);
  }
  return c->cuda_fail(e, what);
}

}  // namespace

extern "C" {

int pp_abi_version(void) { return PP_ABI_VERSION; }

const char* pp_version(void) { return "photonprop_b200 0.1.0 (sm_100a)"; }

uint64_t pp_launch_count(void) { return pp::g_launches.load(); }

uint64_t pp_pair_seed(uint64_t global_seed, uint64_t index) {
  // splitmix64 (Steele, Lea, Flood 2014) of seed + golden-ratio * (index + 1)
  uint64_t z = global_seed + 0x9E3779B97F4A7C15ull * (index + 1ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

pp_status pp_default_opts(int32_t mode, pp_run_opts* o) {
  if (!o || (mode != PP_MODE_COMPAT && mode != PP_MODE_PHYSICAL)) return PP_ERR_ARG;
  std::memset(o, 0, sizeof *o);
  o->mode = mode;
  if (mode == PP_MODE_COMPAT) {
    o->max_steps = 10;
    o->g = 0.99f;
    o->t_max = 0.f;
    o->hist_bins = 0;
    o->hist_bin_width = 1.f;
  } else {
    o->max_steps = 1000;
    o->g = 0.95f;
    o->t_max = 500.f;
    o->hist_t0 = 0.f;
    o->hist_bin_width = 1.f;
    o->hist_bins = 500;
    o->flags = PP_OPT_PMT_WEIGHT;
  }
  return PP_OK;
}

pp_status pp_create(pp_ctx** out, int device, const pp_medium_desc* medium, const pp_spectrum_desc* spectrum,
                    const pp_pmt_desc* pmt) {
  if (!out || !medium || !spectrum) {
    g_create_error = "pp_create: NULL argument";
    return PP_ERR_ARG;
  }
  *out = nullptr;
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || device < 0 || device >= ndev) {
    g_create_error = std::string("pp_create: no CUDA device ") + std::to_string(device) +
                     (e ? std::string(" (") + cudaGetErrorString(e) + ")" : std::string());
    cudaGetLastError();
    return e ? PP_ERR_CUDA : PP_ERR_ARG;
  }
  if (medium->n_abs < 0 || medium->n_abs > PP_MAX_ABS || (pmt && (pmt->n < 0 || pmt->n > PP_MAX_PMT))) {
    g_create_error = "pp_create: table size out of range";
    return PP_ERR_ARG;
  }
  // spectrum knots
  double knots[PP_MAX_KNOTS];
  int n_knots = 0;
  if (spectrum->kind == PP_SPECTRUM_MONOCHROMATIC) {
    if (!(spectrum->wl_min > 0.0)) {
      g_create_error = "pp_create: monochromatic wavelength must be > 0";
      return PP_ERR_ARG;
    }
    knots[0] = spectrum->wl_min;
    n_knots = 1;
  } else if (spectrum->kind == PP_SPECTRUM_CHERENKOV) {
    if (pp_cherenkov_knots(medium, spectrum->wl_min, spectrum->wl_max, spectrum->n_knots, knots) != PP_OK) {
      g_create_error = "pp_create: invalid Cherenkov spectrum (need 2 <= n_knots <= 64, 0 < wl_min < wl_max)";
      return PP_ERR_ARG;
    }
    n_knots = spectrum->n_knots;
  } else {
    g_create_error = "pp_create: unknown spectrum kind (the reference throws ArgumentError)";
    return PP_ERR_ARG;
  }
  pp_ctx* c = new pp_ctx();
  c->device = device;
  c->medium = *medium;
  std::memset(&c->pmt, 0, sizeof c->pmt);
  if (pmt) c->pmt = *pmt;
  DeviceGuard guard(device);
  cudaDeviceProp prop;
  if ((e = cudaGetDeviceProperties(&prop, device))) {
    g_create_error = std::string("pp_create: ") + cudaGetErrorString(e);
    delete c;
    return PP_ERR_CUDA;
  }
  c->sm_count = prop.multiProcessorCount;
  c->device_name = prop.name;
  double coeffs[11];
  pp::medium_coeffs(medium, coeffs);
  float fk[PP_MAX_KNOTS], aw[PP_MAX_ABS], al[PP_MAX_ABS];
  std::vector<float> pw(PP_MAX_PMT), pa(PP_MAX_PMT);
  for (int i = 0; i < n_knots; ++i) fk[i] = (float)knots[i];
  double dwl[PP_MAX_ABS], dlen[PP_MAX_ABS];
  int n_abs = medium->n_abs;
  if (n_abs > 0) {
    for (int i = 0; i < n_abs; ++i) {
      dwl[i] = medium->abs_wl[i];
      dlen[i] = medium->abs_len[i];
    }
  } else {
    pp::default_abs_table(dwl, dlen, &n_abs);
  }
  for (int i = 0; i < n_abs; ++i) {
    aw[i] = (float)dwl[i];
    al[i] = (float)dlen[i];
  }
  const int n_pmt = pmt ? pmt->n : 0;
  for (int i = 0; i < n_pmt; ++i) {
    pw[i] = (float)pmt->wavelength[i];
    pa[i] = (float)pmt->acceptance[i];
  }
  pp::fill_fit_consts(&c->fitk, pp_refractive_index(medium, 800.0), pp_group_index(medium, 800.0));
  c->h_tables.resize(pp::dev_tables_size());
  pp::fill_dev_tables(c->h_tables.data(), coeffs, fk, n_knots, aw, al, n_abs, pw.data(), pa.data(), n_pmt);
  {
    std::vector<double> fwd(pp::kCascNF + 1), inv(pp::kCascNI + 1);
    pp::cascade_tables(fwd.data(), inv.data());
    std::vector<float> ft(fwd.begin(), fwd.end());
    ft.insert(ft.end(), inv.begin(), inv.end());
    if ((e = cudaMalloc(&c->d_casc, ft.size() * sizeof(float))) ||
        (e = cudaMemcpy(c->d_casc, ft.data(), ft.size() * sizeof(float), cudaMemcpyHostToDevice))) {
      g_create_error = std::string("pp_create: ") + cudaGetErrorString(e);
      cudaGetLastError();
      if (c->d_casc) cudaFree(c->d_casc);
      delete c;
      return e == cudaErrorMemoryAllocation ? PP_ERR_OOM : PP_ERR_CUDA;
    }
    pp::set_cascade_tables(c->h_tables.data(), static_cast<const float*>(c->d_casc), fwd.front(), fwd.back());
  }
  if ((e = cudaMalloc(&c->d_tables, c->h_tables.size())) ||
      (e = cudaMemcpy(c->d_tables, c->h_tables.data(), c->h_tables.size(), cudaMemcpyHostToDevice)) ||
      (e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking))) {
    g_create_error = std::string("pp_create: ") + cudaGetErrorString(e);
    cudaGetLastError();
    if (c->d_tables) cudaFree(c->d_tables);
    cudaFree(c->d_casc);
    delete c;
    return e == cudaErrorMemoryAllocation ? PP_ERR_OOM : PP_ERR_CUDA;
  }
  *out = c;
  return PP_OK;
}

void pp_destroy(pp_ctx* c) {
  if (!c) return;
  {
    std::lock_guard<std::mutex> lk(c->mu);
    DeviceGuard guard(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    c->drop_graphs();
    for (DevBuf* b : {&c->pairs, &c->hits, &c->counters, &c->stats, &c->hist, &c->offsets, &c->queue, &c->fit_counts,
                      &c->fit_rec, &c->fit_moments, &c->fit_out, &c->fit_cs, &c->llh_chunks, &c->pilot})
      b->release();
    if (c->d_tables) cudaFree(c->d_tables);
    if (c->d_casc) cudaFree(c->d_casc);
    if (c->stream) cudaStreamDestroy(c->stream);
  }
  delete c;
}

const char* pp_last_error(const pp_ctx* c) { return c ? c->err.c_str() : g_create_error.c_str(); }

int pp_device(const pp_ctx* c) { return c ? c->device : -1; }

pp_status pp_get_knots(const pp_ctx* c, float* out, int32_t cap, int32_t* n) {
  if (!c || !n) return PP_ERR_ARG;
  float k[PP_MAX_KNOTS];
  int nk = 0;
  pp::get_dev_knots(c->h_tables.data(), k, &nk);
  *n = nk;
  if (out)
    for (int i = 0; i < nk && i < cap; ++i) out[i] = k[i];
  return PP_OK;
}

pp_status pp_propagate_device(pp_ctx* c, const pp_pair* d_pairs, int64_t n_pairs, const pp_run_opts* opts,
                              pp_hit* d_hits, int64_t cap, uint64_t* d_counters, double* d_stats,
                              double* d_hist, void* stream) {
  pp::Range range_("pp_propagate_device");
  if (!c) return PP_ERR_ARG;
  std::lock_guard<std::mutex> lk(c->mu);
  pp_status st = validate_opts(c, opts);
  if (st) return st;
  if (n_pairs < 0 || n_pairs > (int64_t)INT32_MAX || (n_pairs > 0 && !d_pairs) || !d_counters || !d_stats ||
      (opts->hist_bins > 0 && !d_hist) || cap < 0 || (cap > 0 && !d_hits))
    return c->fail(PP_ERR_ARG, "pp_propagate_device: bad buffer arguments");
  if (!aligned(d_pairs, 16) || !aligned(d_hits, 16) || !aligned(d_counters, 8) || !aligned(d_stats, 8) ||
      !aligned(d_hist, 8))
    return c->fail(PP_ERR_ARG, "pp_propagate_device: pairs/hits need 16-byte, counters/stats/hist 8-byte alignment");
  DeviceGuard guard(c->device);
  cudaError_t e;
  bool grew = false;
  if ((e = ensure(c->offsets, (size_t)(n_pairs + 1) * sizeof(unsigned long long), &grew)) ||
      (e = ensure(c->queue, 64, &grew)))
    return alloc_fail(c, e, "work-queue scratch");
  if (grew) c->drop_graphs();
  pp::LaunchArgs a = base_args(c, opts);
  a.pairs = d_pairs;
  a.n_pairs = n_pairs;
  a.chunk_offsets = static_cast<unsigned long long*>(c->offsets.p);
  a.queue = static_cast<unsigned long long*>(c->queue.p);
  a.hits = d_hits;
  a.hit_cap = (unsigned long long)cap;
  a.counters = reinterpret_cast<unsigned long long*>(d_counters);
  a.stats = d_stats;
  a.hist = opts->hist_bins > 0 ? d_hist : nullptr;
  if ((e = run_batched(c, a, static_cast<cudaStream_t>(stream), true))) return c->cuda_fail(e, "pp_propagate_device");
  return PP_OK;
}

pp_status pp_propagate(pp_ctx* c, const pp_pair* pairs, int64_t n_pairs, const pp_run_opts* opts, pp_hit* hits,
                       int64_t cap, int64_t* n_hits, double* stats, double* hist) {
  pp::Range range_("pp_propagate");
  if (!c) return PP_ERR_ARG;
  std::lock_guard<std::mutex> lk(c->mu);
  pp_status st = validate_opts(c, opts);
  if (st) return st;
  if ((st = validate_pairs(c, pairs, n_pairs, opts->mode))) return st;
  if (cap < 0 || (cap > 0 && !hits) || !n_hits || !stats || (opts->hist_bins > 0 && !hist))
    return c->fail(PP_ERR_ARG, "pp_propagate: bad buffer arguments");
  pp_run_opts o_local = *opts;
  if (any_cascade(pairs, n_pairs)) o_local.flags |= PP_OPT_CASCADE;
  opts = &o_local;
  DeviceGuard guard(c->device);
  const int bins = opts->hist_bins;
  cudaError_t e;
  bool grew = false;
  if ((e = ensure(c->pairs, (size_t)n_pairs * sizeof(pp_pair), &grew)) ||
      (e = ensure(c->hits, (size_t)cap * sizeof(pp_hit), &grew)) || (e = ensure(c->counters, 64, &grew)) ||
      (e = ensure(c->stats, (size_t)n_pairs * PP_STATS * sizeof(double), &grew)) ||
      (e = ensure(c->hist, (size_t)n_pairs * (size_t)(bins > 0 ? bins : 1) * sizeof(double), &grew)) ||
      (e = ensure(c->offsets, (size_t)(n_pairs + 1) * sizeof(unsigned long long), &grew)) || (e = ensure(c->queue, 64, &grew)))
    return alloc_fail(c, e, "pp_propagate buffers");
  if (grew) c->drop_graphs();
  cudaStream_t s = c->stream;
  if (n_pairs > 0 &&
      (e = cudaMemcpyAsync(c->pairs.p, pairs, (size_t)n_pairs * sizeof(pp_pair), cudaMemcpyHostToDevice, s)))
    return c->cuda_fail(e, "copy pairs");
  pp::LaunchArgs a = base_args(c, opts);
  a.pairs = static_cast<const pp_pair*>(c->pairs.p);
  a.n_pairs = n_pairs;
  a.chunk_offsets = static_cast<unsigned long long*>(c->offsets.p);
  a.queue = static_cast<unsigned long long*>(c->queue.p);
  a.hits = static_cast<pp_hit*>(c->hits.p);
  a.hit_cap = (unsigned long long)cap;
  a.counters = static_cast<unsigned long long*>(c->counters.p);
  a.stats = static_cast<double*>(c->stats.p);
  a.hist = bins > 0 ? static_cast<double*>(c->hist.p) : nullptr;
  if ((e = run_batched(c, a, s, true))) return c->cuda_fail(e, "batched launch");
  unsigned long long cnt[4];
  if ((e = cudaMemcpyAsync(cnt, c->counters.p, sizeof cnt, cudaMemcpyDeviceToHost, s)) ||
      (e = cudaStreamSynchronize(s)))
    return c->cuda_fail(e, "batched kernel");
  const int64_t total = (int64_t)cnt[0];
  *n_hits = total;
  const int64_t ncopy = std::min<int64_t>(total, cap);
  if (ncopy > 0 && !(opts->flags & PP_OPT_NO_HITS) &&
      (e = cudaMemcpyAsync(hits, c->hits.p, (size_t)ncopy * hit_bytes(opts), cudaMemcpyDeviceToHost, s)))
    return c->cuda_fail(e, "copy hits");
  if (n_pairs > 0 &&
      (e = cudaMemcpyAsync(stats, c->stats.p, (size_t)n_pairs * PP_STATS * sizeof(double), cudaMemcpyDeviceToHost, s)))
    return c->cuda_fail(e, "copy stats");
  if (bins > 0 && n_pairs > 0 &&
      (e = cudaMemcpyAsync(hist, c->hist.p, (size_t)n_pairs * bins * sizeof(double), cudaMemcpyDeviceToHost, s)))
    return c->cuda_fail(e, "copy hist");
  if ((e = cudaStreamSynchronize(s))) return c->cuda_fail(e, "copy back");
  if (!(opts->flags & PP_OPT_NO_HITS) && total > cap)
    return c->fail(PP_ERR_OVERFLOW, "more hits than hit_capacity; the first hit_capacity were returned");
  return PP_OK;
}

pp_status pp_propagate_plain_device(pp_ctx* c, const pp_pair* d_pair, const pp_pair* h_pair, int64_t pair_index,
                                    const pp_run_opts* opts, pp_hit* d_hits, int64_t cap, uint64_t* d_counters,
                                    double* d_stats, double* d_hist, void* stream) {
  if (!c) return PP_ERR_ARG;
  std::lock_guard<std::mutex> lk(c->mu);
  pp_status st = validate_opts(c, opts);
  if (st) return st;
  if (!d_pair || !h_pair || !d_counters || !d_stats || (opts->hist_bins > 0 && !d_hist) || cap < 0 ||
      (cap > 0 && !d_hits) || pair_index < 0 || pair_index > (int64_t)INT32_MAX)
    return c->fail(PP_ERR_ARG, "pp_propagate_plain_device: bad arguments");
  if (!aligned(d_pair, 16) || !aligned(d_hits, 16) || !aligned(d_counters, 8) || !aligned(d_stats, 8) ||
      !aligned(d_hist, 8))
    return c->fail(PP_ERR_ARG, "pp_propagate_plain_device: pair/hits need 16-byte, counters/stats/hist 8-byte alignment");
  if ((st = validate_pairs(c, h_pair, 1, opts->mode))) return st;
  pp_run_opts o_local = *opts;
  if (any_cascade(h_pair, 1)) o_local.flags |= PP_OPT_CASCADE;
  opts = &o_local;
  DeviceGuard guard(c->device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  pp::LaunchArgs a = base_args(c, opts);
  a.pairs = d_pair;
  a.n_pairs = 1;
  a.hits = d_hits;
  a.hit_cap = (unsigned long long)cap;
  a.counters = reinterpret_cast<unsigned long long*>(d_counters);
  a.stats = d_stats;
  a.hist = opts->hist_bins > 0 ? d_hist : nullptr;
  const int block = opts->block_size > 0 ? opts->block_size : 256;
  int bps = pp::plain_max_blocks_per_sm(opts->mode, block);
  if (bps < 1) bps = 1;
  const long long need = (h_pair->n_photons + block - 1) / block;
  int grid = (int)std::min<long long>((long long)c->sm_count * bps, std::max<long long>(need, 1));
  cudaError_t e;
  if ((e = cudaMemsetAsync(d_stats, 0, PP_STATS * sizeof(double), s))) return c->cuda_fail(e, "memset");
  if (a.hist && (e = cudaMemsetAsync(a.hist, 0, (size_t)opts->hist_bins * sizeof(double), s)))
    return c->cuda_fail(e, "memset");
  if ((e = pp::launch_reset_counters(a.counters, s)) ||
      (e = pp::launch_plain(a, d_pair, (int)pair_index, grid, block, s)) ||
      (e = pp::launch_finalize(d_pair, 1, d_stats, a.hist, opts->hist_bins, (opts->flags & PP_OPT_NORMALIZE) ? 1 : 0,
                               c->sm_count, s)))
    return c->cuda_fail(e, "plain launch");
  return PP_OK;
}

pp_status pp_propagate_plain(pp_ctx* c, const pp_pair* pairs, int64_t n_pairs, const pp_run_opts* opts,
                             pp_hit* hits, int64_t cap, int64_t* n_hits, double* stats, double* hist) {
  pp::Range range_("pp_propagate_plain");
  if (!c) return PP_ERR_ARG;
  pp_run_opts o_plain;
  {
    std::lock_guard<std::mutex> lk(c->mu);
    pp_status st = validate_opts(c, opts);
    if (st) return st;
    if ((st = validate_pairs(c, pairs, n_pairs, opts->mode))) return st;
    if (cap < 0 || (cap > 0 && !hits) || !n_hits || !stats || (opts->hist_bins > 0 && !hist))
      return c->fail(PP_ERR_ARG, "pp_propagate_plain: bad buffer arguments");
    if (any_cascade(pairs, n_pairs) && !(opts->flags & PP_OPT_CASCADE)) {
      o_plain = *opts;
      o_plain.flags |= PP_OPT_CASCADE;
      opts = &o_plain;
    }
    DeviceGuard guard(c->device);
    const int bins = opts->hist_bins;
    cudaError_t e;
    bool grew = false;
    if ((e = ensure(c->pairs, (size_t)n_pairs * sizeof(pp_pair), &grew)) ||
        (e = ensure(c->hits, (size_t)cap * sizeof(pp_hit), &grew)) || (e = ensure(c->counters, 64, &grew)) ||
        (e = ensure(c->stats, PP_STATS * sizeof(double), &grew)) ||
        (e = ensure(c->hist, (size_t)(bins > 0 ? bins : 1) * sizeof(double), &grew)))
      return alloc_fail(c, e, "pp_propagate_plain buffers");
    if (grew) c->drop_graphs();
    if (n_pairs > 0 && (e = cudaMemcpyAsync(c->pairs.p, pairs, (size_t)n_pairs * sizeof(pp_pair),
                                            cudaMemcpyHostToDevice, c->stream)))
      return c->cuda_fail(e, "copy pairs");
  }
  int64_t total = 0;
  const int bins = opts->hist_bins;
  for (int64_t p = 0; p < n_pairs; ++p) {
    const int64_t room = std::max<int64_t>(cap - std::min(total, cap), 0);
    pp_status st = pp_propagate_plain_device(
        c, static_cast<const pp_pair*>(c->pairs.p) + p, pairs + p, p, opts, static_cast<pp_hit*>(c->hits.p), room,
        static_cast<uint64_t*>(c->counters.p), static_cast<double*>(c->stats.p),
        bins > 0 ? static_cast<double*>(c->hist.p) : nullptr, c->stream);
    if (st) return st;
    std::lock_guard<std::mutex> lk(c->mu);
    DeviceGuard guard(c->device);
    unsigned long long cnt[4];
    cudaError_t e;
    if ((e = cudaMemcpyAsync(cnt, c->counters.p, sizeof cnt, cudaMemcpyDeviceToHost, c->stream)) ||
        (e = cudaStreamSynchronize(c->stream)))
      return c->cuda_fail(e, "plain kernel");
    const int64_t nh = (int64_t)cnt[0];
    const int64_t ncopy = std::min<int64_t>(nh, room);
    if (ncopy > 0 && !(opts->flags & PP_OPT_NO_HITS) &&
        (e = cudaMemcpyAsync(reinterpret_cast<char*>(hits) + (size_t)std::min(total, cap) * hit_bytes(opts), c->hits.p,
                             (size_t)ncopy * hit_bytes(opts), cudaMemcpyDeviceToHost, c->stream)))
      return c->cuda_fail(e, "copy hits");
    if ((e = cudaMemcpyAsync(stats + p * PP_STATS, c->stats.p, PP_STATS * sizeof(double), cudaMemcpyDeviceToHost,
                             c->stream)))
      return c->cuda_fail(e, "copy stats");
    if (bins > 0 && (e = cudaMemcpyAsync(hist + p * bins, c->hist.p, (size_t)bins * sizeof(double),
                                         cudaMemcpyDeviceToHost, c->stream)))
      return c->cuda_fail(e, "copy hist");
    if ((e = cudaStreamSynchronize(c->stream))) return c->cuda_fail(e, "copy back");
    total += nh;
  }
  *n_hits = total;
  if (!(opts->flags & PP_OPT_NO_HITS) && total > cap)
    return c->fail(PP_ERR_OVERFLOW, "more hits than hit_capacity; the first hit_capacity were returned");
  return PP_OK;
}

pp_status pp_cuda_propagate_photons(pp_ctx* c, float* pos, float* dir, float* wl, float* dist, int32_t* sp,
                                    int64_t* nsim, int32_t stack_len, int32_t n_blocks, int32_t threads,
                                    const pp_pair* st_pair, const pp_run_opts* opts, void* stream) {
  pp::Range range_("pp_cuda_propagate_photons");
  if (!c) return PP_ERR_ARG;
  std::lock_guard<std::mutex> lk(c->mu);
  pp_status st = validate_opts(c, opts);
  if (st) return st;
  if (!pos || !dir || !wl || !dist || !sp || !nsim || !st_pair || stack_len < 1 || n_blocks < 1 || threads < 32 ||
      threads > 1024 || threads % 32)
    return c->fail(PP_ERR_ARG, "pp_cuda_propagate_photons: bad arguments");
  if (!aligned(pos, 4) || !aligned(dir, 4) || !aligned(wl, 4) || !aligned(dist, 4) || !aligned(sp, 4) ||
      !aligned(nsim, 8))
    return c->fail(PP_ERR_ARG, "pp_cuda_propagate_photons: misaligned output array");
  if ((int64_t)stack_len * n_blocks > (int64_t)INT32_MAX)
    return c->fail(PP_ERR_ARG, "stack_len * n_blocks exceeds int32 indices");
  if ((st = validate_pairs(c, st_pair, 1, opts->mode))) return st;
  DeviceGuard guard(c->device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaError_t e;
  bool grew = false;
  if ((e = ensure(c->pairs, sizeof(pp_pair), &grew)) || (e = ensure(c->counters, 64, &grew)))
    return alloc_fail(c, e, "pp_cuda_propagate_photons buffers");
  if (grew) c->drop_graphs();
  if ((e = cudaMemcpyAsync(c->pairs.p, st_pair, sizeof(pp_pair), cudaMemcpyHostToDevice, s)))
    return c->cuda_fail(e, "copy source");
  pp::LaunchArgs a = base_args(c, opts);
  a.pairs = static_cast<const pp_pair*>(c->pairs.p);
  a.n_pairs = 1;
  a.counters = static_cast<unsigned long long*>(c->counters.p);
  const long long G = (long long)n_blocks * threads;
  const long long per_thread = (st_pair->n_photons + G - 1) / G;  // cld(photons, grid*block), :288
  if ((e = pp::launch_reset_counters(a.counters, s)) ||
      (e = pp::launch_stacks(a, a.pairs, pos, dir, wl, dist, sp, nsim, stack_len, n_blocks, threads, per_thread, s)))
    return c->cuda_fail(e, "stacks launch");
  // the reference call is synchronous (CUDA.jl launches block on copy-back)
  if ((e = cudaStreamSynchronize(s))) return c->cuda_fail(e, "stacks kernel");
  return PP_OK;
}

pp_status pp_device_eval(pp_ctx* c, int32_t op, const double* in, double* out, int64_t n) {
  if (!c) return PP_ERR_ARG;
  std::lock_guard<std::mutex> lk(c->mu);
  static const int in_w[] = {6, 1, 2, 6, 7, 1, 1, 1, 1, 1, 1, 2, 3};
  static const int out_w[] = {4, 1, 1, 3, 3, 1, 1, 1, 1, 1, 1, 1, 5};
  if (op < 0 || op > 12 || n < 0 || (n > 0 && (!in || !out))) return c->fail(PP_ERR_ARG, "pp_device_eval: bad arguments");
  if (n == 0) return PP_OK;
  DeviceGuard guard(c->device);
  double *din = nullptr, *dout = nullptr;
  const size_t bi = (size_t)n * in_w[op] * sizeof(double), bo = (size_t)n * out_w[op] * sizeof(double);
  cudaError_t e;
  if ((e = cudaMalloc(&din, bi)) || (e = cudaMalloc(&dout, bo))) {
    if (din) cudaFree(din);
    return alloc_fail(c, e, "pp_device_eval");
  }
  e = cudaMemcpyAsync(din, in, bi, cudaMemcpyHostToDevice, c->stream);
  if (!e) e = pp::launch_eval(op, din, dout, n, c->d_tables, c->stream);
  if (!e) e = cudaMemcpyAsync(out, dout, bo, cudaMemcpyDeviceToHost, c->stream);
  if (!e) e = cudaStreamSynchronize(c->stream);
  cudaFree(din);
  cudaFree(dout);
  if (e) return c->cuda_fail(e, "pp_device_eval");
  return PP_OK;
}

namespace {
// Uploads cos/sin of the observation angles into the context's buffer.
pp_status upload_angles(pp_ctx* c, const double* obs_angles, int32_t n_angles, cudaStream_t s) {
  if (n_angles < 1 || n_angles > PP_MAX_FIT_ANGLES || !obs_angles)
    return c->fail(PP_ERR_ARG, "need 1 <= n_angles <= PP_MAX_FIT_ANGLES observation angles");
  std::vector<float2> cs(n_angles);
  for (int i = 0; i < n_angles; ++i) {
    if (!std::isfinite(obs_angles[i])) return c->fail(PP_ERR_ARG, "observation angles must be finite");
    cs[i] = make_float2((float)std::cos(obs_angles[i]), (float)std::sin(obs_angles[i]));
  }
  bool grew = false;
  cudaError_t e;
  if ((e = ensure(c->fit_cs, cs.size() * sizeof(float2), &grew))) return alloc_fail(c, e, "fit angles");
  if ((e = cudaMemcpyAsync(c->fit_cs.p, cs.data(), cs.size() * sizeof(float2), cudaMemcpyHostToDevice, s)))
    return c->cuda_fail(e, "copy fit angles");
  return PP_OK;
}

// Fit stage over hits on the device (the caller's): moments, then fits.
pp_status fit_hits(pp_ctx* c, const pp_pair* d_pairs, int64_t n_pairs, int32_t mode, const pp_hit* d_hits,
                   int64_t cap, const uint64_t* d_counters, const double* obs_angles, int32_t n_angles,
                   double* d_moments, double* d_fits, cudaStream_t s) {
  pp_status st = upload_angles(c, obs_angles, n_angles, s);
  if (st) return st;
  bool grew = false;
  cudaError_t e;
  if ((e = ensure(c->fit_counts, (size_t)std::max<int64_t>(n_pairs, 1) * sizeof(unsigned long long), &grew)) ||
      (e = ensure(c->fit_rec, (size_t)std::max<int64_t>(cap, 1) * sizeof(pp::FitRec), &grew)))
    return alloc_fail(c, e, "fit scratch");
  if (n_pairs == 0) return PP_OK;
  if ((e = cudaMemsetAsync(d_moments, 0, (size_t)n_pairs * n_angles * PP_FIT_MOMENTS * sizeof(double), s)) ||
      (e = pp::launch_fit_moments_hits(c->fitk, c->d_tables, d_pairs, n_pairs, mode, d_hits, (unsigned long long)cap,
                                       reinterpret_cast<const unsigned long long*>(d_counters),
                                       static_cast<unsigned long long*>(c->fit_counts.p),
                                       static_cast<pp::FitRec*>(c->fit_rec.p),
                                       static_cast<const float2*>(c->fit_cs.p), n_angles, d_moments, c->sm_count,
                                       s)) ||
      (e = pp::launch_fit_gamma(d_moments, n_pairs, n_angles, d_pairs, 0, d_fits, s)))
    return c->cuda_fail(e, "fit stage");
  return PP_OK;
}
}  // namespace

// Expected hits of a pair from geometry alone: the sphere's solid-angle
// fraction r^2 / (4 d^2) of the photons (all of them from inside the sphere).
static double expected_hits_geo(const pp_pair& q) {
  const double dx = (double)q.target[0] - q.pos[0], dy = (double)q.target[1] - q.pos[1],
               dz = (double)q.target[2] - q.pos[2];
  const double d = std::sqrt(dx * dx + dy * dy + dz * dz), r = q.radius;
  const double f = d <= r ? 1.0 : std::min(1.0, std::max(r * r / (4.0 * (d - r) * (d - r)), 1e-7));
  return f * (double)q.n_photons;
}

// Per-pair hit estimates for planning waves from a pilot launch: the first
// min(N, P) photons of every pair, hit records off.  The photons of a pair
// are a fixed function of (seed, photon index), so these are the full run's
// first photons; their hit counts h, scaled by N / P with four Poisson
// standard deviations added, bound the full counts (exact where P = N).  P is
// 1/64 of the mean photons per pair (at least 65,536); no pilot runs when
// every photon of the batch fits the buffer (at most one hit per photon) or
// when the pilot would cost more than 1/8 of the batch (est stays empty).
static pp_status pilot_estimate(pp_ctx* c, const pp_pair* pairs, int64_t n_pairs, const pp_run_opts& o,
                                int64_t cap, std::vector<double>& est) {
  pp::Range range_("pp_propagate_fit pilot");
  est.clear();
  double photons = 0.0;
  for (int64_t i = 0; i < n_pairs; ++i) photons += (double)pairs[i].n_photons;
  if (n_pairs == 0 || photons <= (double)cap) return PP_OK;
  const int64_t P = std::max<int64_t>(65536, (int64_t)(photons / (64.0 * (double)n_pairs)));
  std::vector<pp_pair> pilot(pairs, pairs + n_pairs);
  double pilot_photons = 0.0;
  for (auto& q : pilot) {
    q.n_photons = std::min<int64_t>(q.n_photons, P);
    pilot_photons += (double)q.n_photons;
  }
  if (pilot_photons > photons / 8.0) return PP_OK;
  cudaStream_t s = c->stream;
  cudaError_t e;
  bool grew = false;
  if ((e = ensure(c->pilot, (size_t)n_pairs * sizeof(pp_pair), &grew))) return alloc_fail(c, e, "pilot pairs");
  pp_run_opts po = o;
  po.flags |= PP_OPT_NO_HITS;
  po.hist_bins = 0;
  pp::LaunchArgs a = base_args(c, &po);
  a.pairs = static_cast<const pp_pair*>(c->pilot.p);
  a.n_pairs = n_pairs;
  a.chunk_offsets = static_cast<unsigned long long*>(c->offsets.p);
  a.queue = static_cast<unsigned long long*>(c->queue.p);
  a.hits = static_cast<pp_hit*>(c->hits.p);
  a.hit_cap = 0;
  a.counters = static_cast<unsigned long long*>(c->counters.p);
  a.stats = static_cast<double*>(c->stats.p);
  a.hist = nullptr;
  std::vector<double> h(n_pairs);
  if ((e = cudaMemcpyAsync(c->pilot.p, pilot.data(), (size_t)n_pairs * sizeof(pp_pair), cudaMemcpyHostToDevice,
                           s)) ||
      (e = run_batched(c, a, s, false)) ||
      (e = cudaMemcpy2DAsync(h.data(), sizeof(double), a.stats, PP_STATS * sizeof(double), sizeof(double),
                             (size_t)n_pairs, cudaMemcpyDeviceToHost, s)) ||
      (e = cudaStreamSynchronize(s)))
    return c->cuda_fail(e, "pp_propagate_fit pilot");
  est.resize(n_pairs);
  for (int64_t i = 0; i < n_pairs; ++i) {
    const double n = (double)pairs[i].n_photons, p = (double)pilot[i].n_photons;
    est[i] = p >= n ? h[i] : (h[i] + 4.0 * std::sqrt(h[i]) + 4.0) * (n / p);
  }
  return PP_OK;
}

pp_status pp_propagate_fit(pp_ctx* c, const pp_pair* pairs, int64_t n_pairs, const pp_run_opts* opts,
                           const double* obs_angles, int32_t n_angles, int64_t cap, int64_t* n_hits, double* fits,
                           double* moments, double* stats, double* hist) {
  pp::Range range_("pp_propagate_fit");
  if (!c) return PP_ERR_ARG;
  std::lock_guard<std::mutex> lk(c->mu);
  pp_status st = validate_opts(c, opts);
  if (st) return st;
  if ((st = validate_pairs(c, pairs, n_pairs, opts->mode))) return st;
  if (cap < 1 || !n_hits || !fits) return c->fail(PP_ERR_ARG, "pp_propagate_fit: bad buffer arguments");
  if (n_angles < 1 || n_angles > PP_MAX_FIT_ANGLES || !obs_angles)
    return c->fail(PP_ERR_ARG, "need 1 <= n_angles <= PP_MAX_FIT_ANGLES observation angles");
  pp_run_opts o = *opts;
  o.flags &= ~(uint32_t)(PP_OPT_NO_HITS | PP_OPT_COMPACT_HITS);  // the fit reads full hit records
  if (any_cascade(pairs, n_pairs)) o.flags |= PP_OPT_CASCADE;
  if (!hist) o.hist_bins = 0;
  const int bins = o.hist_bins;
  DeviceGuard guard(c->device);
  cudaError_t e;
  bool grew = false;
  const size_t rows = (size_t)n_pairs * n_angles;
  if ((e = ensure(c->pairs, (size_t)n_pairs * sizeof(pp_pair), &grew)) ||
      (e = ensure(c->hits, (size_t)cap * sizeof(pp_hit), &grew)) || (e = ensure(c->counters, 64, &grew)) ||
      (e = ensure(c->stats, (size_t)n_pairs * PP_STATS * sizeof(double), &grew)) ||
      (e = ensure(c->hist, (size_t)n_pairs * (size_t)(bins > 0 ? bins : 1) * sizeof(double), &grew)) ||
      (e = ensure(c->offsets, (size_t)(n_pairs + 1) * sizeof(unsigned long long), &grew)) ||
      (e = ensure(c->queue, 64, &grew)) ||
      (e = ensure(c->fit_moments, rows * PP_FIT_MOMENTS * sizeof(double) + 8, &grew)) ||
      (e = ensure(c->fit_out, rows * PP_FIT_OUT * sizeof(double) + 8, &grew)) ||
      (e = ensure(c->fit_counts, (size_t)std::max<int64_t>(n_pairs, 1) * sizeof(unsigned long long), &grew)) ||
      (e = ensure(c->fit_rec, (size_t)cap * sizeof(pp::FitRec), &grew)))
    return alloc_fail(c, e, "pp_propagate_fit buffers");
  if (grew) c->drop_graphs();
  cudaStream_t s = c->stream;
  if ((st = upload_angles(c, obs_angles, n_angles, s))) return st;
  const pp_pair* d_pairs = static_cast<const pp_pair*>(c->pairs.p);
  double* d_mom = static_cast<double*>(c->fit_moments.p);
  if (n_pairs > 0 &&
      ((e = cudaMemcpyAsync(c->pairs.p, pairs, (size_t)n_pairs * sizeof(pp_pair), cudaMemcpyHostToDevice, s)) ||
       (e = cudaMemsetAsync(d_mom, 0, rows * PP_FIT_MOMENTS * sizeof(double), s))))
    return c->cuda_fail(e, "pp_propagate_fit setup");
  // Waves of pairs whose hits fit the hit buffer: each wave propagates, then
  // adds its hits' moments.  A pair's hits are estimated by a pilot launch
  // (or, without one, from geometry scaled by what the waves so far
  // produced); a wave that overflows still counted every pair's hits exactly
  // (its statistics are complete and the photons are a fixed function of the
  // seeds), so it is repacked with those counts and its reruns fit.
  std::vector<double> geo(n_pairs), exact(n_pairs, -1.0), est;
  for (int64_t i = 0; i < n_pairs; ++i) geo[i] = expected_hits_geo(pairs[i]);
  if ((st = pilot_estimate(c, pairs, n_pairs, o, cap, est))) return st;
  double scale = 4.0;
  int64_t total = 0;
  std::vector<double> wst;
  for (int64_t start = 0; start < n_pairs;) {
    auto pick = [&](int64_t from) {
      int64_t to = from;
      double acc = 0.0;
      while (to < n_pairs) {
        const double w = exact[to] >= 0.0 ? exact[to] : (est.empty() ? scale * geo[to] : est[to]);
        if (to > from && acc + w > (est.empty() ? 0.8 : 0.95) * (double)cap) break;
        acc += w;
        ++to;
      }
      return to;
    };
    int64_t end = pick(start);
    unsigned long long cnt[4];
    pp::Range wave_range("pp_propagate_fit wave");
    for (;;) {
      pp::LaunchArgs a = base_args(c, &o);
      a.pairs = d_pairs + start;
      a.n_pairs = end - start;
      a.pair_base = (uint32_t)start;
      a.chunk_offsets = static_cast<unsigned long long*>(c->offsets.p);
      a.queue = static_cast<unsigned long long*>(c->queue.p);
      a.hits = static_cast<pp_hit*>(c->hits.p);
      a.hit_cap = (unsigned long long)cap;
      a.counters = static_cast<unsigned long long*>(c->counters.p);
      a.stats = static_cast<double*>(c->stats.p) + start * PP_STATS;
      a.hist = bins > 0 ? static_cast<double*>(c->hist.p) + start * bins : nullptr;
      const bool whole = start == 0 && end == n_pairs;
      if ((e = run_batched(c, a, s, whole)) ||
          (e = cudaMemcpyAsync(cnt, c->counters.p, sizeof cnt, cudaMemcpyDeviceToHost, s)) ||
          (e = cudaStreamSynchronize(s)))
        return c->cuda_fail(e, "pp_propagate_fit wave");
      double wave_geo = 0.0;
      bool all_geo = true;
      for (int64_t i = start; i < end; ++i) {
        wave_geo += geo[i];
        all_geo = all_geo && exact[i] < 0.0;
      }
      if (all_geo && wave_geo > 0.0) scale = std::max(1.0, 1.25 * (double)cnt[0] / wave_geo);
      if (cnt[0] <= (unsigned long long)cap) break;
      wst.resize((size_t)(end - start) * PP_STATS);
      if ((e = cudaMemcpy(wst.data(), a.stats, wst.size() * sizeof(double), cudaMemcpyDeviceToHost)))
        return c->cuda_fail(e, "pp_propagate_fit wave statistics");
      for (int64_t i = start; i < end; ++i) exact[i] = wst[(size_t)(i - start) * PP_STATS];
      if (exact[start] > (double)cap) {
        *n_hits = (int64_t)exact[start];
        return c->fail(PP_ERR_OVERFLOW, "one pair has more hits than hit_capacity; raise hit_capacity");
      }
      end = pick(start);
    }
    if ((e = pp::launch_fit_moments_hits(c->fitk, c->d_tables, d_pairs, n_pairs, o.mode,
                                         static_cast<const pp_hit*>(c->hits.p), (unsigned long long)cap,
                                         static_cast<const unsigned long long*>(c->counters.p),
                                         static_cast<unsigned long long*>(c->fit_counts.p),
                                         static_cast<pp::FitRec*>(c->fit_rec.p),
                                         static_cast<const float2*>(c->fit_cs.p), n_angles, d_mom, c->sm_count, s)))
      return c->cuda_fail(e, "fit moments");
    total += (int64_t)cnt[0];
    start = end;
  }
  if ((e = pp::launch_fit_gamma(d_mom, n_pairs, n_angles, d_pairs, 0, static_cast<double*>(c->fit_out.p), s)) ||
      (rows && (e = cudaMemcpyAsync(fits, c->fit_out.p, rows * PP_FIT_OUT * sizeof(double), cudaMemcpyDeviceToHost, s))) ||
      (rows && moments &&
       (e = cudaMemcpyAsync(moments, d_mom, rows * PP_FIT_MOMENTS * sizeof(double), cudaMemcpyDeviceToHost, s))) ||
      (n_pairs > 0 && stats &&
       (e = cudaMemcpyAsync(stats, c->stats.p, (size_t)n_pairs * PP_STATS * sizeof(double), cudaMemcpyDeviceToHost, s))) ||
      (n_pairs > 0 && bins > 0 &&
       (e = cudaMemcpyAsync(hist, c->hist.p, (size_t)n_pairs * bins * sizeof(double), cudaMemcpyDeviceToHost, s))) ||
      (e = cudaStreamSynchronize(s)))
    return c->cuda_fail(e, "pp_propagate_fit copy back");
  *n_hits = total;
  return PP_OK;
}

pp_status pp_fit_hits_device(pp_ctx* c, const pp_pair* d_pairs, int64_t n_pairs, int32_t mode, const pp_hit* d_hits,
                             int64_t cap, const uint64_t* d_counters, const double* obs_angles, int32_t n_angles,
                             double* d_moments, double* d_fits, void* stream) {
  pp::Range range_("pp_fit_hits_device");
  if (!c) return PP_ERR_ARG;
  std::lock_guard<std::mutex> lk(c->mu);
  if (mode != PP_MODE_COMPAT && mode != PP_MODE_PHYSICAL) return c->fail(PP_ERR_ARG, "unknown mode");
  if (n_pairs < 0 || n_pairs > (int64_t)INT32_MAX || (n_pairs > 0 && (!d_pairs || !d_moments || !d_fits)) ||
      cap < 0 || (cap > 0 && !d_hits) || !d_counters)
    return c->fail(PP_ERR_ARG, "pp_fit_hits_device: bad buffer arguments");
  if (!aligned(d_pairs, 16) || !aligned(d_hits, 16) || !aligned(d_moments, 8) || !aligned(d_fits, 8))
    return c->fail(PP_ERR_ARG, "pp_fit_hits_device: pairs/hits need 16-byte, moments/fits 8-byte alignment");
  DeviceGuard guard(c->device);
  return fit_hits(c, d_pairs, n_pairs, mode, d_hits, cap, d_counters, obs_angles, n_angles, d_moments, d_fits,
                  static_cast<cudaStream_t>(stream));
}

pp_status pp_fit_photon_dist_device(pp_ctx* c, int64_t n, const double* d_tres, const double* d_theta,
                                    const double* d_ref_ix, const double* d_abs_weight, const double* d_wavelength,
                                    const double* obs_angles, int32_t n_angles, int64_t n_ph_gen, double* d_moments,
                                    double* d_fits, void* stream) {
  if (!c) return PP_ERR_ARG;
  std::lock_guard<std::mutex> lk(c->mu);
  if (n < 0 || (n > 0 && (!d_tres || !d_theta || !d_ref_ix || !d_abs_weight || !d_wavelength)) || !d_moments ||
      !d_fits || n_ph_gen < 0)
    return c->fail(PP_ERR_ARG, "pp_fit_photon_dist_device: bad arguments");
  DeviceGuard guard(c->device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  pp_status st = upload_angles(c, obs_angles, n_angles, s);
  if (st) return st;
  bool grew = false;
  cudaError_t e;
  if ((e = ensure(c->fit_rec, (size_t)std::max<int64_t>(n, 1) * sizeof(pp::FitRec), &grew)))
    return alloc_fail(c, e, "fit scratch");
  if ((e = pp::launch_fit_columns(c->fitk, c->d_tables, n, d_tres, d_theta, d_ref_ix, d_abs_weight, d_wavelength,
                                  static_cast<pp::FitRec*>(c->fit_rec.p), static_cast<const float2*>(c->fit_cs.p),
                                  n_angles, n_ph_gen, d_moments, d_fits, c->sm_count, s)))
    return c->cuda_fail(e, "fit_photon_dist");
  return PP_OK;
}

pp_status pp_measure_peaks(int device, double* fp32, double* mufu, double* iops) {
  if (!fp32 || !mufu || !iops) return PP_ERR_ARG;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    cudaGetLastError();
    return PP_ERR_ARG;
  }
  DeviceGuard guard(device);
  cudaDeviceProp prop;
  cudaGetDeviceProperties(&prop, device);
  cudaError_t e = pp::run_peaks(prop.multiProcessorCount, fp32, mufu, iops);
  return e ? PP_ERR_CUDA : PP_OK;
}

pp_status pp_measure_step_rate(int device, double* steps_per_s) {
  if (!steps_per_s) return PP_ERR_ARG;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    cudaGetLastError();
    return PP_ERR_ARG;
  }
  DeviceGuard guard(device);
  cudaDeviceProp prop;
  cudaGetDeviceProperties(&prop, device);
  cudaError_t e = pp::run_step_rate(prop.multiProcessorCount, steps_per_s);
  return e ? PP_ERR_CUDA : PP_OK;
}

// Autotuner: times the batched kernel over a grid of launch shapes on the
// given pairs and keeps the fastest per mode.  The cache file holds one line
// per (device name, mode): "name|mode|block|blocks_per_sm|chunk|photons_per_s".
pp_status pp_autotune(pp_ctx* c, const pp_pair* pairs, int64_t n_pairs, const pp_run_opts* opts,
                      const char* cache_path, pp_run_opts* best_out, double* best_rate) {
  pp::Range range_("pp_autotune");
  if (!c) return PP_ERR_ARG;
  pp_status st;
  {
    std::lock_guard<std::mutex> lk(c->mu);
    if ((st = validate_opts(c, opts))) return st;
    if ((st = validate_pairs(c, pairs, n_pairs, opts->mode))) return st;
  }
  pp_run_opts o_tune = *opts;
  if (any_cascade(pairs, n_pairs)) o_tune.flags |= PP_OPT_CASCADE;
  opts = &o_tune;
  const int m = opts->mode;
  if (cache_path) {
    std::ifstream f(cache_path);
    std::string line;
    while (std::getline(f, line)) {
      std::vector<std::string> tok;
      std::stringstream ss(line);
      std::string t;
      while (std::getline(ss, t, '|')) tok.push_back(t);
      if (tok.size() == 6 && tok[0] == c->device_name && std::atoi(tok[1].c_str()) == m) {
        std::lock_guard<std::mutex> lk(c->mu);
        c->tuned_block[m] = std::atoi(tok[2].c_str());
        c->tuned_bps[m] = std::atoi(tok[3].c_str());
        c->tuned_chunk[m] = std::atoi(tok[4].c_str());
        if (best_out) {
          *best_out = *opts;
          best_out->block_size = c->tuned_block[m];
          best_out->blocks_per_sm = c->tuned_bps[m];
          best_out->chunk_photons = c->tuned_chunk[m];
        }
        if (best_rate) *best_rate = std::atof(tok[5].c_str());
        return PP_OK;
      }
    }
  }
  double photons = 0;
  for (int64_t i = 0; i < n_pairs; ++i) photons += (double)pairs[i].n_photons;
  if (photons <= 0) return c->fail(PP_ERR_ARG, "pp_autotune: no photons to time");
  const int blocks[] = {128, 256};
  const int chunks[] = {1024, 4096, 16384};
  std::vector<pp_hit> hits(1 << 16);
  std::vector<double> stats((size_t)n_pairs * PP_STATS), hist((size_t)n_pairs * std::max(opts->hist_bins, 1));
  double best = -1.0;
  pp_run_opts bo = *opts;
  for (int b : blocks) {
    const int maxb = pp::batched_max_blocks_per_sm(m, b, (opts->flags & PP_OPT_CASCADE) != 0);
    for (int bps = 1; bps <= maxb; bps = (bps < maxb && bps * 2 > maxb) ? maxb : bps * 2) {
      for (int ch : chunks) {
        pp_run_opts o = *opts;
        o.block_size = b;
        o.blocks_per_sm = bps;
        o.chunk_photons = ch;
        o.flags |= PP_OPT_NO_HITS;
        int64_t nh = 0;
        const auto t0 = std::chrono::steady_clock::now();
        st = pp_propagate(c, pairs, n_pairs, &o, hits.data(), 0, &nh, stats.data(), hist.data());
        const auto t1 = std::chrono::steady_clock::now();
        if (st != PP_OK) return st;
        const double rate = photons / std::chrono::duration<double>(t1 - t0).count();
        if (rate > best) {
          best = rate;
          bo = o;
        }
      }
      if (bps == maxb) break;
    }
  }
  {
    std::lock_guard<std::mutex> lk(c->mu);
    c->tuned_block[m] = bo.block_size;
    c->tuned_bps[m] = bo.blocks_per_sm;
    c->tuned_chunk[m] = bo.chunk_photons;
    c->drop_graphs();
  }
  if (cache_path) {
    std::ofstream f(cache_path, std::ios::app);
    f << c->device_name << "|" << m << "|" << bo.block_size << "|" << bo.blocks_per_sm << "|" << bo.chunk_photons
      << "|" << best << "\n";
  }
  if (best_out) {
    *best_out = bo;
    best_out->flags = opts->flags;
  }
  if (best_rate) *best_rate = best;
  return PP_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Batched propagation with caller-owned work-queue scratch and no graph: the
// serving loop runs several batches at once, each with its own scratch.
namespace pp {
pp_status propagate_with_scratch(pp_ctx* c, const pp_pair* d_pairs, int64_t n_pairs, const pp_run_opts* opts,
                                 void* d_hits, int64_t cap, uint64_t* d_counters, double* d_stats,
                                 double* d_hist, unsigned long long* d_offsets, unsigned long long* d_queue,
                                 cudaStream_t stream) {
  if (!c) return PP_ERR_ARG;
  std::lock_guard<std::mutex> lk(c->mu);
  pp_status st = validate_opts(c, opts);
  if (st) return st;
  DeviceGuard guard(c->device);
  int grid, block;
  uint32_t chunk;
  resolve_launch(c, *opts, grid, block, chunk);
  pp::LaunchArgs a = base_args(c, opts);
  a.pairs = d_pairs;
  a.n_pairs = n_pairs;
  a.queue = d_queue;
  a.chunk_offsets = d_offsets;
  a.chunk = chunk;
  a.hits = static_cast<pp_hit*>(d_hits);
  a.hit_cap = (unsigned long long)cap;
  a.counters = reinterpret_cast<unsigned long long*>(d_counters);
  a.stats = d_stats;
  a.hist = opts->hist_bins > 0 ? d_hist : nullptr;
  const cudaError_t e = enqueue_batched(c, a, grid, block, stream);
  if (e) return c->cuda_fail(e, "batched launch");
  return PP_OK;
}

int ctx_device(const pp_ctx* c) { return c->device; }
int ctx_sm_count(const pp_ctx* c) { return c->sm_count; }
const pp_medium_desc* ctx_medium(const pp_ctx* c) { return &c->medium; }
pp_status ctx_fail(pp_ctx* c, pp_status s, const char* msg) { return c->fail(s, msg); }
pp_status ctx_cuda_fail(pp_ctx* c, cudaError_t e, const char* where) { return c->cuda_fail(e, where); }
std::mutex& ctx_mutex(pp_ctx* c) { return c->mu; }
cudaError_t ctx_llh_scratch(pp_ctx* c, size_t bytes, void** out) {
  bool grew = false;
  cudaError_t e = ensure(c->llh_chunks, bytes, &grew);
  *out = c->llh_chunks.p;
  return e;
}
}  // namespace pp

// ---------------------------------------------------------------------------
// Allocation-free batched propagation (pp_propagate_device_noalloc).
//
// The work-queue scratch is this file-scope device array: word 0 is the queue
// cursor, words 32.. the chunk offsets (n_pairs + 1 of them).  In host code
// the name g_noalloc_scratch is only a host-side stand-in for the symbol, not
// a device address: a kernel given it would fault or, where the GPU can reach
// host memory, silently use the wrong memory.  The device address is looked
// up with cudaGetSymbolAddress with the context's device current.  The first
// lookup on a device is the set-up (it may load the library's device code
// there); later lookups allocate nothing.  The lookup is repeated on every
// call rather than cached, so that after a device reset (cudaDeviceReset,
// CUDA.jl's device_reset!) the call uses the array of the new context
// instead of the old one's address.
namespace {
constexpr int kNoallocQueueWords = 32;
static __device__ __align__(256) unsigned long long g_noalloc_scratch[kNoallocQueueWords + PP_NOALLOC_MAX_PAIRS + 1];

// Device address of the scratch array on the current device.
cudaError_t noalloc_scratch(unsigned long long** out) {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess) return e;
  *out = static_cast<unsigned long long*>(p);
  return cudaSuccess;
}
}  // namespace

extern "C" pp_status pp_propagate_device_noalloc(pp_ctx* c, const pp_pair* d_pairs, int64_t n_pairs,
                                                 const pp_run_opts* opts, pp_hit* d_hits, int64_t cap,
                                                 uint64_t* d_counters, double* d_stats, double* d_hist,
                                                 void* stream) {
  pp::Range range_("pp_propagate_device_noalloc");
  if (!c) return PP_ERR_ARG;
  std::lock_guard<std::mutex> lk(c->mu);
  pp_status st = validate_opts(c, opts);
  if (st) return st;
  if (n_pairs > PP_NOALLOC_MAX_PAIRS)
    return c->fail(PP_ERR_ARG, "pp_propagate_device_noalloc: n_pairs exceeds PP_NOALLOC_MAX_PAIRS (65536); "
                               "split the batch or use pp_propagate_device");
  if (n_pairs < 0 || (n_pairs > 0 && !d_pairs) || !d_counters || !d_stats || (opts->hist_bins > 0 && !d_hist) ||
      cap < 0 || (cap > 0 && !d_hits))
    return c->fail(PP_ERR_ARG, "pp_propagate_device_noalloc: bad buffer arguments");
  if (!aligned(d_pairs, 16) || !aligned(d_hits, 16) || !aligned(d_counters, 8) || !aligned(d_stats, 8) ||
      !aligned(d_hist, 8))
    return c->fail(PP_ERR_ARG,
                   "pp_propagate_device_noalloc: pairs/hits need 16-byte, counters/stats/hist 8-byte alignment");
  DeviceGuard guard(c->device);
  unsigned long long* scratch = nullptr;
  cudaError_t e = noalloc_scratch(&scratch);
  if (e) return c->cuda_fail(e, "pp_propagate_device_noalloc: cudaGetSymbolAddress");
  int grid, block;
  uint32_t chunk;
  resolve_launch(c, *opts, grid, block, chunk);
  pp::LaunchArgs a = base_args(c, opts);
  a.pairs = d_pairs;
  a.n_pairs = n_pairs;
  a.queue = scratch;
  a.chunk_offsets = scratch + kNoallocQueueWords;
  a.chunk = chunk;
  a.hits = d_hits;
  a.hit_cap = (unsigned long long)cap;
  a.counters = reinterpret_cast<unsigned long long*>(d_counters);
  a.stats = d_stats;
  a.hist = opts->hist_bins > 0 ? d_hist : nullptr;
  // the scan kernel rewrites every offset and zeroes the cursor and counters
  if ((e = enqueue_batched(c, a, grid, block, static_cast<cudaStream_t>(stream))))
    return c->cuda_fail(e, "pp_propagate_device_noalloc");
  return PP_OK;
}
