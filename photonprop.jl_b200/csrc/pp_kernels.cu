// Kernels of the photon-propagation hot path (sm_100a).
//
//  batched_kernel  persistent: each warp pulls photon chunks of any pair from a
//                  device work queue and refills a lane as soon as its photon
//                  ends, so lanes never idle behind a long-lived photon and
//                  thousands of uneven pairs run in one launch.
//  plain_kernel    one pair per launch, one photon per thread at a time
//                  (grid-stride), the straightforward port of the reference's
//                  thread loop (src/photon_prop_cuda.jl:301-380).
//  stacks_kernel   cuda_propagate_photons! with the reference's output layout
//                  (per-block hit stacks, src/photon_prop_cuda.jl:262-386).
//  chunk_scan_kernel / finalize_kernel   work-queue set-up and FP64
//                  normalisation.
//  eval_kernel     device helpers on test inputs.
//  peak kernels    FP32 / MUFU / INT issue microbenchmarks for the roofline.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include "pp_device.cuh"
#include "pp_internal.h"

namespace ppd {

// ---------------------------------------------------------------------------
// Batched persistent kernel.
//
// Each warp owns a ring of kStage staged emissions in shared memory.  When
// its dead lanes outnumber the staged photons, all 32 lanes take the next
// photon indices from the warp's chunk (grabbing chunks from the device work
// queue) and compute 32 emissions together, converged; dead lanes then pick
// staged photons up with four 16-byte loads.  The step loop that follows
// is the same straight-line code for every lane.
constexpr int kStage = 64;  // >= 2 * 32 - 1 staged emissions per warp (power of two)

struct __align__(16) Staged {
  float px, py, pz, dx, dy, dz, neg_ln2_len, path;
  uint32_t id_lo, id_hi;
  int32_t pair;
  float radius;         // the pair's sphere radius, so that a refill reads
  uint32_t sc0, sc1;  // shared memory only, and the photon's step stream
  uint32_t pad[2];
};

// Compat mode hits often: a photon whose line meets the sphere beyond its
// step waits in place, pointing at it, until a step reaches it (3.6 % of the
// photons of make_photon_fits hit, against 4e-5 in physical mode).  There a
// hit lane stages its photon in shared memory and the warp records up to 32
// staged hits together, converged, instead of one or two lanes walking the
// hit path while the others wait.
constexpr unsigned kHitStage = 32;

// A warp's current photon chunk (warp-uniform): kept in shared memory, since
// only the warp's emission pass reads or advances it, so that the step loop
// holds no registers for it.
struct WarpChunk {
  unsigned long long base;  // first photon index of the chunk
  unsigned next, len;
  int pair;
  int done;  // the work queue is exhausted
};
struct StagedHit {
  float px, py, pz, dx, dy, dz, path;
  uint32_t id_lo, id_hi;
  int32_t pair;
};

// Register budget: 64 per thread (1024 threads per SM) for the basic
// emitters; the cascade variant's table lookups in the emission block spill
// at 64, so it gets 80 (768 threads per SM), which runs cone and isotropic
// pairs as fast as the basic variant does.
template <int MODE, int WARPS, int EM>
__global__ void __launch_bounds__(WARPS * 32, (EM == kEmCascade ? 768 : 1024) / (WARPS * 32))
    batched_kernel(const RunParams R) {
  __shared__ __align__(16) DevTables T;
  __shared__ Staged stage[WARPS][kStage];
  __shared__ WarpStats wstats[WARPS];
  __shared__ StagedHit hstage[MODE == kCompat ? WARPS : 1][kHitStage];
  __shared__ WarpChunk wchunk[WARPS];
  stage_tables(T, R.tables);
  if ((threadIdx.x & 31u) == 0) {
    WarpStats& w0 = wstats[threadIdx.x >> 5];
    w0.pair = -1;
    for (int k = 0; k < 6; ++k) w0.v[k] = 0.0;
    WarpChunk& q = wchunk[threadIdx.x >> 5];
    q.base = 0;
    q.next = q.len = 0;
    q.pair = 0;
    q.done = 0;
  }
  __syncthreads();

  const unsigned lane = threadIdx.x & 31u;
  const unsigned lt_mask = (1u << lane) - 1u;
  Staged* ring = stage[threadIdx.x >> 5];
  WarpStats* ws = &wstats[threadIdx.x >> 5];
  StagedHit* hst = hstage[MODE == kCompat ? (threadIdx.x >> 5) : 0];
  unsigned h_count = 0;  // staged hits (compat mode), warp-uniform
  const unsigned long long total_chunks = R.chunk_offsets[R.n_pairs];
  // records staged hits 0..n-1 (n warp-uniform), one per lane
  auto record_staged = [&](unsigned n) {
    if (lane < n) {
      const StagedHit& g = hst[lane];
      Photon p;
      p.px = g.px;
      p.py = g.py;
      p.pz = g.pz;
      p.dx = g.dx;
      p.dy = g.dy;
      p.dz = g.dz;
      p.path = g.path;
      p.neg_ln2_len = 0.f;
      p.id_lo = g.id_lo;
      p.ctr3 = g.id_hi;  // block 0: the index's top bits only
      p.sc0 = p.sc1 = 0u;
      const PairCtx pc = load_pair_ctx(R.pairs + g.pair, g.pair);
      const HitValues h = hit_values<MODE, EM>(T, R, R.pairs + g.pair, pc, p);
      record_hit_cached(R, ws, pc, p, h);
    }
    __syncwarp();
  };

  // warp-uniform state: the ring (the current chunk is in shared memory)
  WarpChunk* wq = &wchunk[threadIdx.x >> 5];
  unsigned r_head = 0, r_count = 0;

  // lane state
  bool alive = false;
  Photon s;
  s.id_lo = 0;
  s.ctr3 = 1u << 8;
  s.sc0 = s.sc1 = 0u;
  s.px = s.py = s.pz = s.dx = s.dy = s.path = s.neg_ln2_len = 0.f;
  s.dz = 1.f;
  // the lane's pair: radius and index (the seed, which only a hit's emission
  // replay needs, is read from the pair record then)
  PairCtx c;
  c.r = 0.f;
  c.seed_lo = c.seed_hi = 0u;
  c.index = 0;
  unsigned steps = 0;

  for (;;) {
    const unsigned need = __ballot_sync(kFull, !alive);
    const unsigned n_need = __popc(need);
    if (r_count < n_need && !wq->done) {
      unsigned long long c_base = wq->base;
      unsigned c_next = wq->next, c_len = wq->len;
      int c_pair = wq->pair;
      bool queue_done = false;
      // give every lane the next photon index of the queue
      bool have = false;
      unsigned long long pid = 0;
      int ppair = 0;
      unsigned filled = 0;
      while (filled < 32u) {
        if (c_next >= c_len) {
          unsigned long long cid = 0, start = 0, end = 0;
          int p = 0;
          if (lane == 0) {
            cid = atomicAdd(R.queue, 1ull);
            if (cid < total_chunks) {
              int lo = 0, hi = (int)R.n_pairs - 1;  // last pair whose first chunk <= cid
              while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (R.chunk_offsets[mid] <= cid) lo = mid; else hi = mid - 1;
              }
              p = lo;
              if (EM == kEmBasic && R.pairs[p].emitter == PP_EMITTER_CASCADE)
                atomicOr(R.counters + 2, 4ull);  // a cascade pair in a launch without PP_OPT_CASCADE
              start = (cid - R.chunk_offsets[p]) * (unsigned long long)R.chunk;
              end = min(start + (unsigned long long)R.chunk, (unsigned long long)R.pairs[p].n_photons);
            }
          }
          cid = __shfl_sync(kFull, cid, 0);
          if (cid >= total_chunks) {
            queue_done = true;
            break;
          }
          c_pair = __shfl_sync(kFull, p, 0);
          if (c_pair != ws->pair) {  // the warp's statistics cache follows its chunk
            if (lane == 0) {
              flush_warp_stats(R.stats, ws);
              ws->pair = c_pair;
            }
            __syncwarp();
          }
          c_base = __shfl_sync(kFull, start, 0);
          c_len = (unsigned)(__shfl_sync(kFull, end, 0) - c_base);
          c_next = 0;
        }
        const unsigned take = min(32u - filled, c_len - c_next);
        if (lane >= filled && lane < filled + take) {
          have = true;
          pid = c_base + (c_next + (lane - filled));
          ppair = c_pair;
        }
        c_next += take;
        filled += take;
      }
      if (lane == 0) {
        wq->base = c_base;
        wq->next = c_next;
        wq->len = c_len;
        wq->pair = c_pair;
        wq->done = queue_done;
      }
      if (have) {
        const pp_pair* P = R.pairs + ppair;
        const PairCtx pc = load_pair_ctx(P, ppair);
        Photon e;
        set_photon(e, pid);
        emit_event<MODE, EM>(T, R, P, pc, e);
        float4* dst = reinterpret_cast<float4*>(ring + ((r_head + r_count + lane) & (kStage - 1)));
        dst[0] = make_float4(e.px, e.py, e.pz, e.dx);
        dst[1] = make_float4(e.dy, e.dz, e.neg_ln2_len, e.path);
        dst[2] = make_float4(__uint_as_float((uint32_t)pid), __uint_as_float((uint32_t)(pid >> 32)),
                             __int_as_float(ppair), pc.r);
        dst[3] = make_float4(__uint_as_float(e.sc0), __uint_as_float(e.sc1), 0.f, 0.f);
      }
      r_count += filled;
      __syncwarp();
    }
    if (!alive) {
      const unsigned rank = __popc(need & lt_mask);
      if (rank < r_count) {
        const float4* src = reinterpret_cast<const float4*>(ring + ((r_head + rank) & (kStage - 1)));
        const float4 a = src[0], b = src[1], d = src[2], e = src[3];
        s.px = a.x;
        s.py = a.y;
        s.pz = a.z;
        s.dx = a.w;
        s.dy = b.x;
        s.dz = b.y;
        s.neg_ln2_len = b.z;
        s.path = b.w;
        s.id_lo = __float_as_uint(d.x);
        s.ctr3 = __float_as_uint(d.y) | (1u << 8);  // index bits 32..39, step 0
        c.index = __float_as_int(d.z);
        c.r = d.w;
        s.sc0 = __float_as_uint(e.x);
        s.sc1 = __float_as_uint(e.y);
        alive = true;
      }
    }
    const unsigned took = min(n_need, r_count);
    r_head += took;
    r_count -= took;
    __syncwarp();
    if (need == kFull && took == 0u) break;  // every lane was idle and none took a photon
    bool hit = false;
    if (alive) {
      ++steps;
      alive = step_event<MODE>(R, c, s, hit);
    }
    if (MODE == kCompat) {
      const unsigned hm = __ballot_sync(kFull, hit);
      if (hm) {
        const unsigned nh = __popc(hm);
        if (h_count + nh > kHitStage) {  // no room: record what is staged first
          record_staged(h_count);
          h_count = 0;
        }
        if (hit) {
          StagedHit& g = hst[h_count + __popc(hm & lt_mask)];
          g.px = s.px;
          g.py = s.py;
          g.pz = s.pz;
          g.dx = s.dx;
          g.dy = s.dy;
          g.dz = s.dz;
          g.path = s.path;
          g.id_lo = s.id_lo;
          g.id_hi = s.ctr3 & 0xFFu;
          g.pair = c.index;
        }
        h_count += nh;
        __syncwarp();
        if (h_count == kHitStage) {
          record_staged(kHitStage);
          h_count = 0;
        }
      }
    } else if (__any_sync(kFull, hit)) {
      if (hit) {
        const PairCtx pc = load_pair_ctx(R.pairs + c.index, c.index);
        const HitValues h = hit_values<MODE, EM>(T, R, R.pairs + c.index, pc, s);
        record_hit_cached(R, ws, pc, s, h);
      }
    }
  }
  __syncwarp();
  if (MODE == kCompat && h_count > 0u) record_staged(h_count);
  if (lane == 0) flush_warp_stats(R.stats, ws);
  // photon-step count for the roofline
  unsigned long long st = steps;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) st += __shfl_xor_sync(kFull, st, o);
  if (lane == 0) atomicAdd(R.counters + 1, st);
}

// ---------------------------------------------------------------------------
// Plain kernel: one pair, photons id = gtid + i * stride.
template <int MODE, int EM>
__global__ void __launch_bounds__(512) plain_kernel(const RunParams R, const pp_pair* __restrict__ pair_ptr,
                                                    int pair_index) {
  __shared__ __align__(16) DevTables T;
  stage_tables(T, R.tables);
  __syncthreads();
  const PairCtx c = load_pair_ctx(pair_ptr, pair_index);
  const unsigned long long n = (unsigned long long)pair_ptr->n_photons;
  const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
  unsigned steps = 0;
  for (unsigned long long id = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; id < n;
       id += stride) {
    Photon s;
    set_photon(s, id);
    s.dx = s.dy = 0.f;
    s.dz = 1.f;
    bool alive = true;
    while (alive) {
      bool hit = false;
      steps += (s.ctr3 >= (1u << 8));
      alive = photon_event<MODE, EM>(T, R, pair_ptr, c, s, hit);
      if (hit) {
        const HitValues h = hit_values<MODE, EM>(T, R, pair_ptr, c, s);
        record_hit(R, c, s, h, 0);
      }
    }
  }
  unsigned long long st = steps;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) st += __shfl_xor_sync(kFull, st, o);
  if ((threadIdx.x & 31u) == 0) atomicAdd(R.counters + 1, st);
}

// ---------------------------------------------------------------------------
// cuda_propagate_photons! layout (src/photon_prop_cuda.jl:262-386).  Photon
// ids: thread g simulates ids g + i * (blocks * threads), i < per_thread.
template <int MODE>
__global__ void __launch_bounds__(1024) stacks_kernel(const RunParams R, const pp_pair* __restrict__ pair_ptr,
                                                      float* __restrict__ out_pos, float* __restrict__ out_dir,
                                                      float* __restrict__ out_wl, float* __restrict__ out_dist,
                                                      int32_t* __restrict__ out_sp,
                                                      long long* __restrict__ out_nsim, int stack_len,
                                                      long long per_thread) {
  __shared__ __align__(16) DevTables T;
  __shared__ int cursor;
  stage_tables(T, R.tables);
  const int ix_offset = (int)blockIdx.x * stack_len + 1;  // 1-based, as in the reference
  if (threadIdx.x == 0) cursor = ix_offset;
  __syncthreads();
  const PairCtx c = load_pair_ctx(pair_ptr, 0);
  const int safe_margin = max(0, (int)blockDim.x - 32);
  const unsigned long long G = (unsigned long long)gridDim.x * blockDim.x;
  const unsigned long long g = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long n_sim = 0;
  unsigned steps = 0;
  for (long long i = 0; i < per_thread; ++i) {
    if (*(volatile int*)&cursor > ix_offset + stack_len - safe_margin) break;
    Photon s;
    set_photon(s, g + (unsigned long long)i * G);
    s.dx = s.dy = 0.f;
    s.dz = 1.f;
    bool alive = true;
    while (alive) {
      bool hit = false;
      steps += (s.ctr3 >= (1u << 8));
      alive = photon_event<MODE, kEmCascade>(T, R, pair_ptr, c, s, hit);
      if (hit) {
        const HitValues h = hit_values<MODE, kEmCascade>(T, R, pair_ptr, c, s);
        const int idx = atomicAdd(&cursor, 1);  // 1-based slot
        if (idx < ix_offset + stack_len) {
          const int j = idx - 1;
          out_pos[3 * j + 0] = h.px;
          out_pos[3 * j + 1] = h.py;
          out_pos[3 * j + 2] = h.pz;
          out_dir[3 * j + 0] = h.d0x;
          out_dir[3 * j + 1] = h.d0y;
          out_dir[3 * j + 2] = h.d0z;
          out_wl[j] = h.wl;
          out_dist[j] = h.dist;
          atomicMax(out_sp + blockIdx.x, idx);
        } else {
          atomicOr(R.counters + 2, 1ull);
        }
      }
    }
    ++n_sim;
  }
  atomicAdd(reinterpret_cast<unsigned long long*>(out_nsim), (unsigned long long)n_sim);
  atomicAdd(R.counters + 1, (unsigned long long)steps);
}

// ---------------------------------------------------------------------------
// Chunk offsets of the work queue: offsets[p] = sum_{q<p} ceil(N_q / chunk),
// offsets[n] = total.  One block; also resets the queue and counters.
__global__ void __launch_bounds__(1024) chunk_scan_kernel(const pp_pair* __restrict__ pairs, int64_t n,
                                                          uint32_t chunk,
                                                          unsigned long long* __restrict__ offsets,
                                                          unsigned long long* __restrict__ queue,
                                                          unsigned long long* __restrict__ counters) {
  __shared__ unsigned long long warp_sums[32];
  const int t = threadIdx.x;
  const int64_t per = (n + blockDim.x - 1) / blockDim.x;
  const int64_t b = (int64_t)t * per;
  const int64_t e = min(b + per, n);
  unsigned long long local = 0;
  for (int64_t i = b; i < e; ++i) {
    const long long np = pairs[i].n_photons;
    local += np > 0 ? ((unsigned long long)np + chunk - 1) / chunk : 0ull;
  }
  // exclusive block scan of `local`
  const unsigned lane = t & 31, warp = t >> 5;
  unsigned long long incl = local;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned long long v = __shfl_up_sync(kFull, incl, o);
    if ((int)lane >= o) incl += v;
  }
  if (lane == 31) warp_sums[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    unsigned long long w = (lane < (blockDim.x >> 5)) ? warp_sums[lane] : 0ull;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned long long v = __shfl_up_sync(kFull, w, o);
      if ((int)lane >= o) w += v;
    }
    warp_sums[lane] = w;  // inclusive over warps
  }
  __syncthreads();
  unsigned long long run = incl - local + (warp > 0 ? warp_sums[warp - 1] : 0ull);
  for (int64_t i = b; i < e; ++i) {
    offsets[i] = run;
    const long long np = pairs[i].n_photons;
    run += np > 0 ? ((unsigned long long)np + chunk - 1) / chunk : 0ull;
  }
  if (t == (int)blockDim.x - 1) offsets[n] = warp_sums[(blockDim.x >> 5) - 1];
  if (t == 0) {
    queue[0] = 0ull;
    counters[0] = 0ull;
    counters[1] = 0ull;
    counters[2] = 0ull;
    counters[3] = 0ull;
  }
}

__global__ void reset_counters_kernel(unsigned long long* __restrict__ counters) {
  if (threadIdx.x < 4) counters[threadIdx.x] = 0ull;
}

// stats[p][6] = photons; optionally hist[p][:] /= photons.
__global__ void finalize_kernel(const pp_pair* __restrict__ pairs, int64_t n_pairs, double* __restrict__ stats,
                                double* __restrict__ hist, int bins, int normalize) {
  const int64_t total = n_pairs * (int64_t)(bins > 0 ? bins : 1);
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t p = bins > 0 ? i / bins : i;
    const double n = (double)pairs[p].n_photons;
    if (bins <= 0 || i % bins == 0) stats[p * PP_STATS + 6] = n;
    if (normalize && bins > 0 && n > 0) hist[i] /= n;
  }
}

// ---------------------------------------------------------------------------
__global__ void eval_kernel(int op, const double* __restrict__ in, double* __restrict__ out, int64_t n,
                            const DevTables* __restrict__ tables) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const DevTables& T = *tables;
  switch (op) {
    case 0: {
      const double* a = in + 6 * i;
      uint32_t c[4] = {(uint32_t)a[0], (uint32_t)a[1], (uint32_t)a[2], (uint32_t)a[3]};
      philox4x32_10(c, (uint32_t)a[4], (uint32_t)a[5]);
      for (int j = 0; j < 4; ++j) out[4 * i + j] = (double)c[j];
      break;
    }
    case 1: out[i] = (double)u01((uint32_t)in[i]); break;
    case 12: {  // step block: (counter word 0, word 1, key) -> (w0, w1, u0, u1, u2)
      const double* a = in + 3 * i;
      uint32_t w0 = (uint32_t)a[0], w1 = (uint32_t)a[1];
      philox2x32_10(w0, w1, (uint32_t)a[2]);
      const Draw3 d = step_uniforms(w0, w1);
      double* o = out + 5 * i;
      o[0] = (double)w0;
      o[1] = (double)w1;
      o[2] = (double)d.u0;
      o[3] = (double)d.u1;
      o[4] = (double)d.u2;
      break;
    }
    case 2: {
      const float g = (float)in[2 * i];
      HG h;
      h.iso = (g == 0.f);
      h.two_g = 2.f * g;
      h.one_m_g = 1.f - g;
      h.a = 1.f - g * g;
      h.one_p_g2 = 1.f + g * g;
      h.inv_2g = h.iso ? 0.f : 1.f / (2.f * g);
      out[i] = (double)hg_costheta(h, (float)in[2 * i + 1]);
      break;
    }
    case 3: {
      const double* a = in + 6 * i;
      float x, y, z;
      rotate_to_axis((float)a[0], (float)a[1], (float)a[2], (float)a[3], (float)a[4], (float)a[5], x, y, z);
      out[3 * i] = x;
      out[3 * i + 1] = y;
      out[3 * i + 2] = z;
      break;
    }
    case 4: {
      const double* a = in + 7 * i;
      const float st = (float)a[6];
      out[3 * i] = fmaf(st, (float)a[3], (float)a[0]);
      out[3 * i + 1] = fmaf(st, (float)a[4], (float)a[1]);
      out[3 * i + 2] = fmaf(st, (float)a[5], (float)a[2]);
      break;
    }
    case 5: out[i] = (double)draw_wavelength(T, (float)in[i]); break;
    case 6: out[i] = (double)phase_index(T, 1.f / (float)in[i]); break;
    case 7: out[i] = (double)group_index(T, 1.f / (float)in[i]); break;
    case 8: out[i] = (double)scattering_length(T, (float)in[i]); break;
    case 9: out[i] = (double)interp_sorted((float)in[i], T.abs_wl, T.abs_len, T.n_abs); break;
    case 11: out[i] = (double)cascade_cos_theta(T, 1.f / (float)in[2 * i + 1], (float)in[2 * i]); break;
    case 10:
      out[i] = T.n_pmt > 0 ? (double)interp_sorted((float)in[i], T.pmt_wl, T.pmt_acc, T.n_pmt) : 1.0;
      break;
    default: out[i] = 0.0;
  }
}

// ---------------------------------------------------------------------------
// Issue-rate microbenchmarks: 8 independent dependent chains per thread.
__global__ void peak_fma_kernel(float* out, int iters, float a, float b) {
  float x[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) x[j] = (float)(threadIdx.x + j);
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int j = 0; j < 8; ++j) x[j] = fmaf(x[j], a, b);
  }
  float s = 0.f;
#pragma unroll
  for (int j = 0; j < 8; ++j) s += x[j];
  if (s == 1.2345f) out[0] = s;
}

__global__ void peak_mufu_kernel(float* out, int iters) {
  float x[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) x[j] = 0.5f + 0.01f * (float)(threadIdx.x & 7) + 0.001f * j;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int j = 0; j < 8; ++j) x[j] = ex2(x[j] * -0.5f);  // ex2 of a value in (0,1): stays in (0,1)
  }
  float s = 0.f;
#pragma unroll
  for (int j = 0; j < 8; ++j) s += x[j];
  if (s == 1.2345f) out[0] = s;
}

__global__ void peak_philox_kernel(unsigned* out, int iters) {
  // independent Philox4x32-10 blocks per thread: the integer work of one photon step
  uint32_t acc = 0;
  for (int i = 0; i < iters; ++i) {
    uint32_t c[4] = {threadIdx.x, blockIdx.x, (uint32_t)i, 0u};
    philox4x32_10(c, 0x12345678u, 0x9abcdef0u);
    acc ^= c[0] ^ c[1] ^ c[2] ^ c[3];
  }
  if (acc == 12345u) out[0] = acc;
}

// Speed of light of the physical step: every lane steps its own photon
// through step_event (one Philox2x32-10 block, the ray-sphere test, the move
// and the Henyey-Greenstein turn) with no emission, refill, hit record or
// loop bookkeeping, at the batched kernel's occupancy (256 threads, 4 CTAs
// per SM, at most 64 registers).  Its step rate bounds what the batched
// kernel can reach on this GPU under instruction-issue limits.  The photons
// start 100 m from a 0.21 m sphere with an unbounded path, so they keep
// moving; the results are kept live through a never-true store.
__global__ void __launch_bounds__(256, 4) peak_step_kernel(const RunParams R, int iters,
                                                           unsigned long long* __restrict__ out) {
  PairCtx c;
  c.r = 0.21f;
  c.seed_lo = c.seed_hi = 0u;
  c.index = 0;
  Photon s;
  s.sc0 = 0x9E3779B9u * (blockIdx.x + 1u) ^ threadIdx.x;
  s.sc1 = 0x2545F491u & 0x7FFFFFFu;
  const uint64_t id = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  s.id_lo = (uint32_t)id;
  s.px = 100.f + (float)(threadIdx.x & 31u);
  s.py = 50.f;
  s.pz = -30.f;
  s.dx = 0.6f;
  s.dy = 0.f;
  s.dz = 0.8f;
  s.path = 1e30f;
  s.neg_ln2_len = -kLn2 * 30.f;
  s.ctr3 = ctr_word(id, 1u);
  unsigned live = 0;
  for (int i = 0; i < iters; ++i) {
    bool hit = false;
    live += step_event<kPhysical>(R, c, s, hit) ? 1u : 0u;
  }
  if (s.px == 1.2345f && s.dz == 0.5f && live == 7u) out[1] = 1ull;
  if ((threadIdx.x & 31u) == 0) atomicAdd(out, 32ull * (unsigned long long)iters);
}

}  // namespace ppd

// ---------------------------------------------------------------------------
// Launch helpers (host).
namespace pp {

static __host__ ppd::RunParams to_params(const LaunchArgs& a) {
  ppd::RunParams R;
  R.pairs = a.pairs;
  R.n_pairs = a.n_pairs;
  R.chunk_offsets = a.chunk_offsets;
  R.queue = a.queue;
  R.chunk = a.chunk;
  R.pair_base = a.pair_base;
  R.hits = a.hits;
  R.hit_cap = a.hit_cap;
  R.counters = a.counters;
  R.stats = a.stats;
  R.hist = a.hist;
  R.tables = reinterpret_cast<const ppd::DevTables*>(a.tables);
  R.max_steps = a.opts.max_steps;
  R.ctr_limit = ((uint32_t)a.opts.max_steps + 1u) << 8;
  R.t_max = a.opts.t_max;
  R.hist_t0 = a.opts.hist_t0;
  R.inv_bin_width = a.opts.hist_bin_width > 0.f ? 1.f / a.opts.hist_bin_width : 0.f;
  R.hist_bins = a.opts.hist_bins;
  R.flags = a.opts.flags;
  const float g = a.opts.g;
  R.hg.iso = (g == 0.f);
  R.hg.two_g = 2.f * g;
  R.hg.one_m_g = 1.f - g;
  R.hg.a = 1.f - g * g;
  R.hg.one_p_g2 = 1.f + g * g;
  R.hg.inv_2g = R.hg.iso ? 0.f : 1.f / (2.f * g);
  return R;
}

size_t dev_tables_size() { return sizeof(ppd::DevTables); }

void fill_dev_tables(void* host_tables, const double coeffs[11], const float* knots, int n_knots,
                     const float* abs_wl, const float* abs_len, int n_abs, const float* pmt_wl,
                     const float* pmt_acc, int n_pmt) {
  ppd::DevTables* t = reinterpret_cast<ppd::DevTables*>(host_tables);
  memset(t, 0, sizeof(*t));
  t->a01 = (float)coeffs[0];
  t->a2 = (float)coeffs[1];
  t->a3 = (float)coeffs[2];
  t->a4 = (float)coeffs[3];
  t->g01 = (float)coeffs[0];
  t->g2 = (float)(2.0 * coeffs[1]);
  t->g3 = (float)(3.0 * coeffs[2]);
  t->g4 = (float)(4.0 * coeffs[3]);
  t->sca0 = (float)coeffs[4];
  t->sca1 = (float)coeffs[5];
  t->sca2 = (float)coeffs[6];
  t->n_knots = n_knots;
  for (int i = 0; i < n_knots; ++i) t->knots[i] = knots[i];
  t->n_abs = n_abs;
  for (int i = 0; i < n_abs; ++i) {
    t->abs_wl[i] = abs_wl[i];
    t->abs_len[i] = abs_len[i];
  }
  t->n_pmt = n_pmt;
  for (int i = 0; i < n_pmt; ++i) {
    t->pmt_wl[i] = pmt_wl[i];
    t->pmt_acc[i] = pmt_acc[i];
  }
}

void set_cascade_tables(void* host_tables, const float* d_casc, double gmin, double gmax) {
  ppd::DevTables* t = reinterpret_cast<ppd::DevTables*>(host_tables);
  t->casc = d_casc;
  t->casc_nf = kCascNF;
  t->casc_ni = kCascNI;
  t->casc_vmin = (float)kCascVMin;
  t->casc_inv_dv = (float)(kCascNF / (kCascVMax - kCascVMin));
  t->casc_gmin = (float)gmin;
  t->casc_inv_dg = (float)(kCascNI / (gmax - gmin));
}

void get_dev_knots(const void* host_tables, float* out, int* n) {
  const ppd::DevTables* t = reinterpret_cast<const ppd::DevTables*>(host_tables);
  *n = t->n_knots;
  for (int i = 0; i < t->n_knots; ++i) out[i] = t->knots[i];
}

cudaError_t launch_chunk_scan(const LaunchArgs& a, cudaStream_t s) {
  ppd::chunk_scan_kernel<<<1, 1024, 0, s>>>(a.pairs, a.n_pairs, a.chunk, a.chunk_offsets, a.queue, a.counters);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_reset_counters(unsigned long long* counters, cudaStream_t s) {
  ppd::reset_counters_kernel<<<1, 32, 0, s>>>(counters);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_batched(const LaunchArgs& a, int grid, int block, cudaStream_t s) {
  const ppd::RunParams R = to_params(a);
  const bool casc = a.opts.mode == PP_MODE_PHYSICAL && (a.opts.flags & PP_OPT_CASCADE);
  if (block == 128) {
    if (a.opts.mode == PP_MODE_COMPAT)
      ppd::batched_kernel<ppd::kCompat, 4, ppd::kEmBasic><<<grid, 128, 0, s>>>(R);
    else if (casc)
      ppd::batched_kernel<ppd::kPhysical, 4, ppd::kEmCascade><<<grid, 128, 0, s>>>(R);
    else
      ppd::batched_kernel<ppd::kPhysical, 4, ppd::kEmBasic><<<grid, 128, 0, s>>>(R);
  } else {
    if (a.opts.mode == PP_MODE_COMPAT)
      ppd::batched_kernel<ppd::kCompat, 8, ppd::kEmBasic><<<grid, 256, 0, s>>>(R);
    else if (casc)
      ppd::batched_kernel<ppd::kPhysical, 8, ppd::kEmCascade><<<grid, 256, 0, s>>>(R);
    else
      ppd::batched_kernel<ppd::kPhysical, 8, ppd::kEmBasic><<<grid, 256, 0, s>>>(R);
  }
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_plain(const LaunchArgs& a, const pp_pair* d_pair, int pair_index, int grid, int block,
                         cudaStream_t s) {
  const ppd::RunParams R = to_params(a);
  if (a.opts.mode == PP_MODE_COMPAT)
    ppd::plain_kernel<ppd::kCompat, ppd::kEmBasic><<<grid, block, 0, s>>>(R, d_pair, pair_index);
  else if (a.opts.flags & PP_OPT_CASCADE)
    ppd::plain_kernel<ppd::kPhysical, ppd::kEmCascade><<<grid, block, 0, s>>>(R, d_pair, pair_index);
  else
    ppd::plain_kernel<ppd::kPhysical, ppd::kEmBasic><<<grid, block, 0, s>>>(R, d_pair, pair_index);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_stacks(const LaunchArgs& a, const pp_pair* d_pair, float* pos, float* dir, float* wl,
                          float* dist, int32_t* sp, int64_t* nsim, int stack_len, int grid, int block,
                          long long per_thread, cudaStream_t s) {
  const ppd::RunParams R = to_params(a);
  if (a.opts.mode == PP_MODE_COMPAT)
    ppd::stacks_kernel<ppd::kCompat><<<grid, block, 0, s>>>(R, d_pair, pos, dir, wl, dist, sp,
                                                            reinterpret_cast<long long*>(nsim), stack_len,
                                                            per_thread);
  else
    ppd::stacks_kernel<ppd::kPhysical><<<grid, block, 0, s>>>(R, d_pair, pos, dir, wl, dist, sp,
                                                              reinterpret_cast<long long*>(nsim), stack_len,
                                                              per_thread);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_finalize(const pp_pair* pairs, int64_t n, double* stats, double* hist, int bins, int normalize,
                            int sm_count, cudaStream_t s) {
  const int64_t total = n * (int64_t)(bins > 0 ? bins : 1);
  int grid = (int)std::min<int64_t>((total + 255) / 256, (int64_t)sm_count * 8);
  if (grid < 1) grid = 1;
  ppd::finalize_kernel<<<grid, 256, 0, s>>>(pairs, n, stats, hist, bins, normalize);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_eval(int op, const double* in, double* out, int64_t n, const void* tables, cudaStream_t s) {
  const int grid = (int)((n + 127) / 128);
  ppd::eval_kernel<<<grid, 128, 0, s>>>(op, in, out, n, reinterpret_cast<const ppd::DevTables*>(tables));
  count_launches(1);
  return cudaGetLastError();
}

int batched_max_blocks_per_sm(int mode, int block, bool cascade) {
  int nb = 0;
  const bool c = mode == PP_MODE_PHYSICAL && cascade;
  if (block == 128) {
    if (mode == PP_MODE_COMPAT)
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, ppd::batched_kernel<ppd::kCompat, 4, ppd::kEmBasic>, 128, 0);
    else if (c)
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, ppd::batched_kernel<ppd::kPhysical, 4, ppd::kEmCascade>, 128, 0);
    else
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, ppd::batched_kernel<ppd::kPhysical, 4, ppd::kEmBasic>, 128, 0);
  } else {
    if (mode == PP_MODE_COMPAT)
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, ppd::batched_kernel<ppd::kCompat, 8, ppd::kEmBasic>, 256, 0);
    else if (c)
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, ppd::batched_kernel<ppd::kPhysical, 8, ppd::kEmCascade>, 256, 0);
    else
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, ppd::batched_kernel<ppd::kPhysical, 8, ppd::kEmBasic>, 256, 0);
  }
  return nb;
}

int plain_max_blocks_per_sm(int mode, int block) {
  int nb = 0;
  if (mode == PP_MODE_COMPAT)
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, ppd::plain_kernel<ppd::kCompat, ppd::kEmBasic>, block, 0);
  else
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, ppd::plain_kernel<ppd::kPhysical, ppd::kEmBasic>, block, 0);
  return nb;
}

cudaError_t run_peaks(int sm_count, double* fp32, double* mufu, double* iops) {
  float* dout = nullptr;
  cudaError_t e = cudaMalloc(&dout, 64);
  if (e != cudaSuccess) return e;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  const int block = 256, grid = sm_count * 8;
  const double threads = (double)grid * block;
  float ms = 0.f;
  // warm-up
  ppd::peak_fma_kernel<<<grid, block>>>(dout, 1000, 0.999f, 0.001f);
  ppd::peak_mufu_kernel<<<grid, block>>>(dout, 100);
  ppd::peak_philox_kernel<<<grid, block>>>(reinterpret_cast<unsigned*>(dout), 100);
  count_launches(3);
  const int it_f = 20000, it_m = 40000, it_i = 4000;
  cudaEventRecord(a);
  ppd::peak_fma_kernel<<<grid, block>>>(dout, it_f, 0.999f, 0.001f);
  cudaEventRecord(b);
  cudaEventSynchronize(b);
  cudaEventElapsedTime(&ms, a, b);
  *fp32 = threads * it_f * 8.0 / (ms * 1e-3);
  cudaEventRecord(a);
  ppd::peak_mufu_kernel<<<grid, block>>>(dout, it_m);
  cudaEventRecord(b);
  cudaEventSynchronize(b);
  cudaEventElapsedTime(&ms, a, b);
  *mufu = threads * it_m * 8.0 / (ms * 1e-3);
  cudaEventRecord(a);
  ppd::peak_philox_kernel<<<grid, block>>>(reinterpret_cast<unsigned*>(dout), it_i);
  cudaEventRecord(b);
  cudaEventSynchronize(b);
  cudaEventElapsedTime(&ms, a, b);
  *iops = threads * it_i / (ms * 1e-3);  // Philox blocks per second
  count_launches(3);
  e = cudaGetLastError();
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(dout);
  return e;
}

cudaError_t run_step_rate(int sm_count, double* steps_per_s) {
  unsigned long long* dout = nullptr;
  cudaError_t e = cudaMalloc(&dout, 16);
  if (e != cudaSuccess) return e;
  cudaMemset(dout, 0, 16);
  LaunchArgs a{};
  a.opts.mode = PP_MODE_PHYSICAL;
  a.opts.max_steps = 1000;
  a.opts.g = 0.95f;
  a.opts.t_max = 1000.f;
  ppd::RunParams R = to_params(a);
  R.ctr_limit = 0xFFFFFFFFu;
  cudaEvent_t t0, t1;
  cudaEventCreate(&t0);
  cudaEventCreate(&t1);
  const int grid = sm_count * 4, block = 256, iters = 20000;
  ppd::peak_step_kernel<<<grid, block>>>(R, 500, dout);  // warm-up
  cudaEventRecord(t0);
  ppd::peak_step_kernel<<<grid, block>>>(R, iters, dout);
  cudaEventRecord(t1);
  cudaEventSynchronize(t1);
  count_launches(2);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, t0, t1);
  *steps_per_s = (double)grid * block * iters / (ms * 1e-3);
  e = cudaGetLastError();
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  cudaFree(dout);
  return e;
}

}  // namespace pp
