// Continuous-batching serving loop (pp_server_*, include/photonprop_b200.h).
//
// One scheduler thread per server.  Requests wait in a FIFO; the scheduler
// admits the head requests while their hit buffers fit the HBM budget and a
// slot is free, packs them into one batch (one pair list, one launch of the
// batched kernel with the slot's own work-queue scratch) on the slot's
// stream, copies the results back on that stream and enqueues a host
// function that marks the slot finished.  A batch takes requests only while
// their reserved hits fit the slot's hit buffers (sized at creation), so a
// running server does not reallocate: a device free synchronises the device
// and pinning pages takes milliseconds, both under the server lock that
// submit() also takes.  Up to max_inflight slots run at
// once, so a request that arrives while batches are on the device is admitted
// as soon as a slot and memory free up, and its batch overlaps the running
// ones.  The host function only sets an atomic flag and notifies; it takes no
// lock (a device-synchronising CUDA call made under the server lock would
// otherwise wait for a host function that waits for the lock).  The scheduler
// also wakes every 500 us, so a missed notification costs at most that.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "pp_internal.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
  uint64_t id = 0;
  std::vector<pp_pair> pairs;
  int64_t hit_cap = 0;  // hit slots reserved in its batch
  int64_t reserve = 0;  // admission bytes
  Clock::time_point t_submit, t_done;
  bool done = false;
  pp_status status = PP_OK;
  std::vector<pp_hit32> hits;
  std::vector<double> stats, hist;
  double photons = 0;
};
using ReqPtr = std::shared_ptr<Request>;

// Buffers grow by doubling (at least 1 MiB) so that reallocation, whose free
// synchronises the device, stays rare in a running server.
inline size_t grown(size_t have, size_t need) {
  size_t n = std::max<size_t>(have, (size_t)1 << 20);
  while (n < need) n *= 2;
  return n;
}

struct DBuf {
  void* p = nullptr;
  size_t bytes = 0;
  cudaError_t ensure(size_t n) {
    if (n == 0) n = 16;
    if (bytes >= n) return cudaSuccess;
    n = grown(bytes, n);
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
    const cudaError_t e = cudaMalloc(&p, n);
    if (e == cudaSuccess) bytes = n;
    return e;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
};

struct HBuf {
  void* p = nullptr;
  size_t bytes = 0;
  cudaError_t ensure(size_t n) {
    if (n == 0) n = 16;
    if (bytes >= n) return cudaSuccess;
    n = grown(bytes, n);
    if (p) cudaFreeHost(p);
    p = nullptr;
    bytes = 0;
    const cudaError_t e = cudaHostAlloc(&p, n, cudaHostAllocDefault);
    if (e == cudaSuccess) bytes = n;
    return e;
  }
  void release() {
    if (p) cudaFreeHost(p);
    p = nullptr;
    bytes = 0;
  }
};

struct Slot {
  pp_server* server = nullptr;
  cudaStream_t stream = nullptr;
  bool busy = false;
  std::atomic<bool> finished{false};
  Clock::time_point t_done;
  std::vector<ReqPtr> reqs;
  std::vector<int64_t> pair_start;  // first batch pair of each request
  int64_t n_pairs = 0, hit_cap = 0, reserve = 0;
  DBuf d_pairs, d_offsets, d_queue, d_hits, d_counters, d_stats, d_hist;
  HBuf h_pairs, h_hits, h_counters, h_stats, h_hist;
};

// Expected hits of one pair for admission: the sphere's solid-angle share
// r^2 / (4 d^2) for an isotropic source; a Cherenkov track concentrates its
// light on a ring, where a sphere intercepts about r / (2 d) of it.
double expected_hits(const pp_pair& p) {
  double cx = p.pos[0], cy = p.pos[1], cz = p.pos[2];
  if (p.emitter == PP_EMITTER_CHERENKOV_CONE) {
    cx += 0.5 * p.track_len * p.dir[0];
    cy += 0.5 * p.track_len * p.dir[1];
    cz += 0.5 * p.track_len * p.dir[2];
  }
  const double dx = p.target[0] - cx, dy = p.target[1] - cy, dz = p.target[2] - cz;
  const double d = std::max(std::sqrt(dx * dx + dy * dy + dz * dz), (double)p.radius);
  const double r = p.radius;
  // cone and cascade emitters concentrate light near the Cherenkov angle: the cone bound for both
  const double f = p.emitter != PP_EMITTER_ISOTROPIC ? 0.5 * r / d : r * r / (4.0 * d * d);
  return (double)p.n_photons * std::min(1.0, f);
}

void CUDART_CB slot_done(void* arg);

}  // namespace

struct pp_server {
  pp_ctx* ctx = nullptr;
  pp_server_config cfg;
  int device = 0;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::thread worker;
  bool stop = false;
  std::deque<ReqPtr> waiting;
  std::unordered_map<uint64_t, ReqPtr> reqs;
  uint64_t next_id = 1;
  int64_t reserved = 0;
  std::vector<std::unique_ptr<Slot>> slots;
  pp_server_counters counters;
};

namespace {

void CUDART_CB slot_done(void* arg) {
  Slot* s = static_cast<Slot*>(arg);
  s->t_done = Clock::now();
  s->finished.store(true, std::memory_order_release);
  s->server->cv_work.notify_all();
}

void fail_requests(pp_server* S, std::vector<ReqPtr>& reqs, pp_status st) {
  const auto now = Clock::now();
  for (auto& r : reqs) {
    r->status = st;
    r->done = true;
    r->t_done = now;
    S->counters.completed += 1;
  }
  S->cv_done.notify_all();
}

// Splits a finished batch into its requests (called with the server lock).
void finish_slot(pp_server* S, Slot& s) {
  const int bins = S->cfg.opts.hist_bins;
  const unsigned long long* cnt = static_cast<const unsigned long long*>(s.h_counters.p);
  const int64_t stored = std::min<int64_t>((int64_t)cnt[0], s.hit_cap);
  const pp_hit32* hits = static_cast<const pp_hit32*>(s.h_hits.p);
  const double* stats = static_cast<const double*>(s.h_stats.p);
  const double* hist = static_cast<const double*>(s.h_hist.p);
  const size_t nr = s.reqs.size();
  for (size_t i = 0; i < nr; ++i) {
    Request& r = *s.reqs[i];
    const int64_t p0 = s.pair_start[i], n = (int64_t)r.pairs.size();
    r.stats.assign(stats + p0 * PP_STATS, stats + (p0 + n) * PP_STATS);
    if (bins > 0) r.hist.assign(hist + p0 * bins, hist + (p0 + n) * bins);
    r.hits.clear();
  }
  for (int64_t h = 0; h < stored; ++h) {  // bucket hits by request (pair ranges are sorted)
    const int64_t pair = hits[h].pair;
    const size_t i = (size_t)(std::upper_bound(s.pair_start.begin(), s.pair_start.end(), pair) - s.pair_start.begin()) - 1;
    pp_hit32 x = hits[h];
    x.pair = (uint32_t)(pair - s.pair_start[i]);
    s.reqs[i]->hits.push_back(x);
  }
  for (size_t i = 0; i < nr; ++i) {
    Request& r = *s.reqs[i];
    double true_hits = 0;
    for (size_t p = 0; p < r.pairs.size(); ++p) true_hits += r.stats[p * PP_STATS];
    r.status = ((double)r.hits.size() < true_hits) ? PP_ERR_OVERFLOW : PP_OK;
    r.t_done = s.t_done;
    r.done = true;
    S->counters.completed += 1;
    S->counters.photons += r.photons;
  }
  S->reserved -= s.reserve;
  S->counters.reserved_bytes = S->reserved;
  S->counters.in_flight_batches -= 1;
  s.reqs.clear();
  s.pair_start.clear();
  s.busy = false;
  s.finished.store(false, std::memory_order_relaxed);
  S->cv_done.notify_all();
}

// Packs the head of the queue into slot s and launches it (server lock held).
bool launch_slot(pp_server* S, Slot& s) {
  pp::Range range_("pp_server batch launch");
  std::vector<ReqPtr> take;
  int64_t pairs = 0, cap = 0, reserve = 0;
  // the slot's hit buffer as it is: a batch that would outgrow it waits for the
  // next slot, so that a running server does not reallocate (a free
  // synchronises the device, and pinning pages takes milliseconds)
  const int64_t have_hits = (int64_t)(std::min(s.d_hits.bytes, s.h_hits.bytes) / sizeof(pp_hit32));
  while (!S->waiting.empty()) {
    const ReqPtr& r = S->waiting.front();
    const int64_t n = (int64_t)r->pairs.size();
    if (!take.empty() && pairs + n > S->cfg.max_pairs_per_batch) break;
    if (!take.empty() && cap + r->hit_cap > have_hits) break;
    if (S->reserved + reserve + r->reserve > S->cfg.hbm_budget_bytes) break;  // wait for memory
    take.push_back(r);
    pairs += n;
    cap += r->hit_cap;
    reserve += r->reserve;
    S->waiting.pop_front();
  }
  if (take.empty()) return false;
  S->counters.waiting = (int64_t)S->waiting.size();
  const int bins = S->cfg.opts.hist_bins;
  cudaError_t e;
  if ((e = s.d_pairs.ensure((size_t)pairs * sizeof(pp_pair))) ||
      (e = s.d_offsets.ensure((size_t)(pairs + 1) * sizeof(unsigned long long))) || (e = s.d_queue.ensure(64)) ||
      (e = s.d_hits.ensure((size_t)cap * sizeof(pp_hit32))) || (e = s.d_counters.ensure(64)) ||
      (e = s.d_stats.ensure((size_t)pairs * PP_STATS * sizeof(double))) ||
      (e = s.d_hist.ensure((size_t)pairs * std::max(bins, 1) * sizeof(double))) ||
      (e = s.h_pairs.ensure((size_t)pairs * sizeof(pp_pair))) || (e = s.h_hits.ensure((size_t)cap * sizeof(pp_hit32))) ||
      (e = s.h_counters.ensure(64)) || (e = s.h_stats.ensure((size_t)pairs * PP_STATS * sizeof(double))) ||
      (e = s.h_hist.ensure((size_t)pairs * std::max(bins, 1) * sizeof(double)))) {
    cudaGetLastError();
    fail_requests(S, take, e == cudaErrorMemoryAllocation ? PP_ERR_OOM : PP_ERR_CUDA);
    return true;
  }
  s.pair_start.clear();
  pp_pair* hp = static_cast<pp_pair*>(s.h_pairs.p);
  int64_t off = 0;
  for (auto& r : take) {
    s.pair_start.push_back(off);
    std::memcpy(hp + off, r->pairs.data(), r->pairs.size() * sizeof(pp_pair));
    off += (int64_t)r->pairs.size();
  }
  pp_run_opts o = S->cfg.opts;
  o.flags |= PP_OPT_COMPACT_HITS;
  o.flags &= ~(uint32_t)PP_OPT_NO_HITS;
  for (int64_t i = 0; i < off; ++i)
    if (hp[i].emitter == PP_EMITTER_CASCADE) {
      o.flags |= PP_OPT_CASCADE;
      break;
    }
  const cudaStream_t st = s.stream;
  pp_status ps = PP_OK;
  if ((e = cudaMemcpyAsync(s.d_pairs.p, hp, (size_t)pairs * sizeof(pp_pair), cudaMemcpyHostToDevice, st)) ||
      (ps = pp::propagate_with_scratch(S->ctx, static_cast<const pp_pair*>(s.d_pairs.p), pairs, &o, s.d_hits.p, cap,
                                       static_cast<uint64_t*>(s.d_counters.p), static_cast<double*>(s.d_stats.p),
                                       static_cast<double*>(s.d_hist.p),
                                       static_cast<unsigned long long*>(s.d_offsets.p),
                                       static_cast<unsigned long long*>(s.d_queue.p), st)) ||
      (e = cudaMemcpyAsync(s.h_counters.p, s.d_counters.p, 32, cudaMemcpyDeviceToHost, st)) ||
      (e = cudaMemcpyAsync(s.h_stats.p, s.d_stats.p, (size_t)pairs * PP_STATS * sizeof(double),
                           cudaMemcpyDeviceToHost, st)) ||
      (bins > 0 && (e = cudaMemcpyAsync(s.h_hist.p, s.d_hist.p, (size_t)pairs * bins * sizeof(double),
                                        cudaMemcpyDeviceToHost, st))) ||
      (e = cudaMemcpyAsync(s.h_hits.p, s.d_hits.p, (size_t)cap * sizeof(pp_hit32), cudaMemcpyDeviceToHost, st)) ||
      (e = cudaLaunchHostFunc(st, slot_done, &s))) {
    cudaGetLastError();
    (void)e;
    fail_requests(S, take, ps ? ps : PP_ERR_CUDA);
    return true;
  }
  s.reqs = std::move(take);
  s.n_pairs = pairs;
  s.hit_cap = cap;
  s.reserve = reserve;
  s.busy = true;
  S->reserved += reserve;
  S->counters.reserved_bytes = S->reserved;
  S->counters.batches += 1;
  S->counters.pairs += pairs;
  S->counters.in_flight_batches += 1;
  return true;
}

void scheduler(pp_server* S) {
  cudaSetDevice(S->device);
  std::unique_lock<std::mutex> lk(S->mu);
  for (;;) {
    bool any_busy = false;
    for (auto& sp : S->slots) {
      Slot& s = *sp;
      if (s.busy && s.finished.load(std::memory_order_acquire)) finish_slot(S, s);
      any_busy |= s.busy;
    }
    if (S->stop && !any_busy) break;
    if (!S->stop) {
      for (auto& sp : S->slots) {
        if (S->waiting.empty()) break;
        if (!sp->busy && !launch_slot(S, *sp)) break;
      }
    }
    S->cv_work.wait_for(lk, std::chrono::microseconds(500));
  }
  std::vector<ReqPtr> rest(S->waiting.begin(), S->waiting.end());
  S->waiting.clear();
  fail_requests(S, rest, PP_ERR_STATE);
}

}  // namespace

extern "C" {

pp_status pp_server_create(pp_ctx* ctx, const pp_server_config* cfg, pp_server** out) {
  if (!ctx || !cfg || !out) return PP_ERR_ARG;
  *out = nullptr;
  pp_server_config c = *cfg;
  if (c.max_inflight <= 0) c.max_inflight = 2;
  if (c.max_inflight > 16) return PP_ERR_ARG;
  if (c.max_pairs_per_batch <= 0) c.max_pairs_per_batch = 4096;
  if (c.hbm_budget_bytes <= 0) c.hbm_budget_bytes = 40ll << 30;
  if (c.bytes_per_hit <= 0) c.bytes_per_hit = (int32_t)sizeof(pp_hit32);
  if (!(c.hit_safety > 0.f)) c.hit_safety = 4.f;
  if (c.max_queued <= 0) c.max_queued = 100000;
  if (c.opts.mode != PP_MODE_COMPAT && c.opts.mode != PP_MODE_PHYSICAL) return PP_ERR_ARG;
  pp_server* S = new pp_server();
  S->ctx = ctx;
  S->cfg = c;
  S->device = pp::ctx_device(ctx);
  std::memset(&S->counters, 0, sizeof S->counters);
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(S->device);
  for (int i = 0; i < c.max_inflight; ++i) {
    auto s = std::make_unique<Slot>();
    s->server = S;
    if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess) {
      cudaGetLastError();
      for (auto& x : S->slots) cudaStreamDestroy(x->stream);
      cudaSetDevice(prev);
      delete S;
      return PP_ERR_CUDA;
    }
    // size for a full batch up front (pairs, scratch, statistics, histograms)
    const size_t np = (size_t)c.max_pairs_per_batch, bins = (size_t)std::max(c.opts.hist_bins, 1);
    if (s->d_pairs.ensure(np * sizeof(pp_pair)) || s->d_offsets.ensure((np + 1) * 8) || s->d_queue.ensure(64) ||
        s->d_counters.ensure(64) || s->d_stats.ensure(np * PP_STATS * 8) || s->d_hist.ensure(np * bins * 8) ||
        s->h_pairs.ensure(np * sizeof(pp_pair)) || s->h_counters.ensure(64) || s->h_stats.ensure(np * PP_STATS * 8) ||
        s->h_hist.ensure(np * bins * 8) || s->d_hits.ensure((size_t)64 << 20) || s->h_hits.ensure((size_t)64 << 20))
      cudaGetLastError();  // a failed pre-allocation is retried at launch
    S->slots.push_back(std::move(s));
  }
  cudaSetDevice(prev);
  S->worker = std::thread(scheduler, S);
  *out = S;
  return PP_OK;
}

void pp_server_destroy(pp_server* S) {
  if (!S) return;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stop = true;
  }
  S->cv_work.notify_all();
  S->worker.join();
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(S->device);
  for (auto& s : S->slots) {
    cudaStreamSynchronize(s->stream);
    for (DBuf* b : {&s->d_pairs, &s->d_offsets, &s->d_queue, &s->d_hits, &s->d_counters, &s->d_stats, &s->d_hist})
      b->release();
    for (HBuf* b : {&s->h_pairs, &s->h_hits, &s->h_counters, &s->h_stats, &s->h_hist}) b->release();
    cudaStreamDestroy(s->stream);
  }
  cudaSetDevice(prev);
  delete S;
}

pp_status pp_server_submit(pp_server* S, const pp_pair* pairs, int32_t n_pairs, uint64_t* id) {
  if (!S || !id || n_pairs <= 0 || !pairs || n_pairs > S->cfg.max_pairs_per_batch) return PP_ERR_ARG;
  auto r = std::make_shared<Request>();
  r->pairs.assign(pairs, pairs + n_pairs);
  double hits = 0;
  for (int32_t i = 0; i < n_pairs; ++i) {
    const pp_pair& p = pairs[i];
    if (p.n_photons < 0 || p.n_photons > (1ll << 40) || !(p.radius > 0.f) ||
        (p.emitter != PP_EMITTER_ISOTROPIC && p.emitter != PP_EMITTER_CHERENKOV_CONE &&
         p.emitter != PP_EMITTER_CASCADE) ||
        (p.emitter != PP_EMITTER_ISOTROPIC && S->cfg.opts.mode == PP_MODE_COMPAT))
      return PP_ERR_ARG;
    hits += std::ceil(S->cfg.hit_safety * expected_hits(p)) + 64.0;
    r->photons += (double)p.n_photons;
  }
  r->hit_cap = (int64_t)hits;
  r->reserve = r->hit_cap * (int64_t)S->cfg.bytes_per_hit;
  if (r->reserve > S->cfg.hbm_budget_bytes) return PP_ERR_ARG;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    if (S->stop) return PP_ERR_STATE;
    if ((int64_t)S->waiting.size() >= S->cfg.max_queued) return PP_ERR_BUSY;
    r->id = S->next_id++;
    r->t_submit = Clock::now();
    S->reqs[r->id] = r;
    S->waiting.push_back(r);
    S->counters.submitted += 1;
    S->counters.waiting = (int64_t)S->waiting.size();
    *id = r->id;
  }
  S->cv_work.notify_all();
  return PP_OK;
}

pp_status pp_server_wait(pp_server* S, uint64_t id, double timeout_s) {
  if (!S) return PP_ERR_ARG;
  std::unique_lock<std::mutex> lk(S->mu);
  auto it = S->reqs.find(id);
  if (it == S->reqs.end()) return PP_ERR_ARG;
  ReqPtr r = it->second;
  const auto limit = std::chrono::duration<double>(std::max(timeout_s, 0.0));
  if (!S->cv_done.wait_for(lk, std::chrono::duration_cast<Clock::duration>(limit), [&] { return r->done; }))
    return PP_ERR_TIMEOUT;
  return PP_OK;
}

pp_status pp_server_result(pp_server* S, uint64_t id, pp_hit32* hits, int64_t cap, int64_t* n_hits, double* stats,
                           double* hist, double* latency_s) {
  if (!S || !n_hits || !stats) return PP_ERR_ARG;
  std::lock_guard<std::mutex> lk(S->mu);
  auto it = S->reqs.find(id);
  if (it == S->reqs.end()) return PP_ERR_ARG;
  Request& r = *it->second;
  if (!r.done) return PP_ERR_STATE;
  if (r.status != PP_OK && r.status != PP_ERR_OVERFLOW) {
    const pp_status st = r.status;
    S->reqs.erase(it);
    return st;
  }
  const int64_t n = std::min<int64_t>((int64_t)r.hits.size(), cap);
  if (hits && n > 0) std::memcpy(hits, r.hits.data(), (size_t)n * sizeof(pp_hit32));
  *n_hits = (int64_t)r.hits.size();
  std::memcpy(stats, r.stats.data(), r.stats.size() * sizeof(double));
  if (hist && !r.hist.empty()) std::memcpy(hist, r.hist.data(), r.hist.size() * sizeof(double));
  if (latency_s) *latency_s = std::chrono::duration<double>(r.t_done - r.t_submit).count();
  const pp_status st = ((int64_t)r.hits.size() > cap) ? PP_ERR_OVERFLOW : r.status;
  S->reqs.erase(it);
  return st;
}

pp_status pp_server_get_counters(pp_server* S, pp_server_counters* out) {
  if (!S || !out) return PP_ERR_ARG;
  std::lock_guard<std::mutex> lk(S->mu);
  *out = S->counters;
  return PP_OK;
}

}  // extern "C"
