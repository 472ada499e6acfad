// Event likelihood on the device: per (hypothesis, module) the extended
// log-likelihood of the module's hit times under a Poisson count and a
// mixture of per-source arrival-time densities (the likelihood of
// example_full.jl:338-449: poisson_dist_per_module, shape_mixture_per_module,
// extended_llh_per_module), FP64.
//
// A module's hits are cut into chunks of one hit per thread; blocks take
// (chunk, hypothesis) items from a grid-stride loop (busy modules spread
// over many blocks, empty ones cost one chunk).  A block sums the module's
// expected photons, stages one term per (source, mixture component) in shared memory
//   c = ln(q w) - lnGamma(alpha) - alpha ln(theta),  alpha - 1,  1 / theta,  shift
// and each thread takes hits: ln f(x) = logsumexp over the terms of
// c + (alpha - 1) ln(x - shift) - (x - shift) / theta, accumulated online
// (running maximum and scaled sum).  Sources beyond one shared-memory tile
// are staged tile by tile for every chunk of hits.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "pp_internal.h"

namespace {

constexpr int kThreads = 256;
constexpr int kTile = 512;  // sources per shared-memory tile

struct Term {
  double c1, am1, c2, bm1, inv_theta, shift;
};

__device__ __forceinline__ double block_sum(double v, double* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x < 32) {
    t = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (threadIdx.x == 0) red[0] = t;
  }
  __syncthreads();
  return red[0];
}

__device__ __forceinline__ void lse_add(double v, double& m, double& s) {
  if (v == -INFINITY) return;
  if (v > m) {
    s = s * exp(m - v) + 1.0;
    m = v;
  } else {
    s += exp(v - m);
  }
}

// chunk_start[k] = first chunk of module k (one chunk per kThreads hits, at
// least one per module); chunk_start[M] = all chunks.  One block.
__global__ void __launch_bounds__(1024) llh_chunk_scan_kernel(const int64_t* __restrict__ offsets, int64_t M,
                                                              int64_t* __restrict__ chunk_start) {
  __shared__ int64_t warp_tot[32];
  __shared__ int64_t carry;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int64_t base = 0; base < M; base += blockDim.x) {
    const int64_t i = base + threadIdx.x;
    const int64_t n = i < M ? offsets[i + 1] - offsets[i] : 0;
    const int64_t v = i < M ? max((int64_t)1, (n + kThreads - 1) / kThreads) : 0;
    int64_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int64_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) warp_tot[warp] = x;
    __syncthreads();
    if (warp == 0) {
      const int nw = blockDim.x >> 5;
      int64_t t = lane < nw ? warp_tot[lane] : 0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int64_t y = __shfl_up_sync(0xffffffffu, t, o);
        if (lane >= o) t += y;
      }
      if (lane < nw) warp_tot[lane] = t;
    }
    __syncthreads();
    const int64_t excl = carry + (warp > 0 ? warp_tot[warp - 1] : 0) + x - v;
    if (i < M) chunk_start[i] = excl;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry = excl + v;
    __syncthreads();
  }
  if (threadIdx.x == 0) chunk_start[M] = carry;
}

__global__ void __launch_bounds__(kThreads) llh_kernel(int mode, int64_t S, int64_t M,
                                                       const double* __restrict__ params,
                                                       const double* __restrict__ photons,
                                                       const int64_t* __restrict__ offsets,
                                                       const double* __restrict__ times,
                                                       const int64_t* __restrict__ chunk_start,
                                                       double* __restrict__ llh) {
  __shared__ Term terms[kTile];
  __shared__ double red[32];
  const int64_t h = blockIdx.y;
  const int64_t total = chunk_start[M];
  for (int64_t g = blockIdx.x; g < total; g += gridDim.x) {
    int64_t lo = 0, hi = M - 1;  // the module whose chunks hold g
    while (lo < hi) {
      const int64_t mid = (lo + hi + 1) >> 1;
      if (chunk_start[mid] <= g) lo = mid; else hi = mid - 1;
    }
    const int64_t k = lo, chunk = g - chunk_start[k];
    const double* P = params + (h * M + k) * S * PP_LLH_PARAMS;
    const double* N = photons ? photons + h * S : nullptr;
    double mu = 0.0, sa = 0.0;
    for (int64_t j = threadIdx.x; j < S; j += blockDim.x) {
      const double a = P[j * PP_LLH_PARAMS];
      mu += a * (N ? N[j] : 1.0);
      sa += a;
    }
    mu = block_sum(mu, red);
    sa = block_sum(sa, red);
    const int64_t h0 = offsets[k], n = offsets[k + 1] - h0;
    const double norm = mode == PP_LLH_REFERENCE ? sa : mu;
    double acc = 0.0;
    {
      const int64_t base = chunk * (int64_t)blockDim.x;
      const bool has = base + threadIdx.x < n;
      const double x = has ? times[h0 + base + threadIdx.x] : 0.0;
      double m = -INFINITY, s = 0.0;
      for (int64_t t0 = 0; t0 < S; t0 += kTile) {
        const int cnt = (int)min((int64_t)kTile, S - t0);
        __syncthreads();
        for (int j = threadIdx.x; j < cnt; j += blockDim.x) {
          const double* q = P + (t0 + j) * PP_LLH_PARAMS;
          const double a = q[0], w = q[1], a1 = q[2], a2 = q[3], th = q[4];
          const double wt = (mode == PP_LLH_REFERENCE ? a : a * (N ? N[t0 + j] : 1.0)) / norm;
          const double lth = log(th);
          Term t;
          t.c1 = (wt * w > 0.0 && a1 > 0.0) ? log(wt * w) - lgamma(a1) - a1 * lth : -INFINITY;
          t.c2 = (wt * (1.0 - w) > 0.0 && a2 > 0.0) ? log(wt * (1.0 - w)) - lgamma(a2) - a2 * lth : -INFINITY;
          t.am1 = a1 - 1.0;
          t.bm1 = a2 - 1.0;
          t.inv_theta = 1.0 / th;
          t.shift = q[5];
          terms[j] = t;
        }
        __syncthreads();
        if (has) {
          for (int j = 0; j < cnt; ++j) {
            const Term t = terms[j];
            const double y = x - t.shift;
            if (!(y > 0.0)) continue;
            const double ly = log(y), e = y * t.inv_theta;
            lse_add(t.c1 + t.am1 * ly - e, m, s);
            lse_add(t.c2 + t.bm1 * ly - e, m, s);
          }
        }
      }
      if (has) acc += s > 0.0 ? m + log(s) : -INFINITY;
    }
    acc = block_sum(acc, red);
    if (threadIdx.x == 0) {
      const double nn = (double)n;
      const double pois = chunk > 0 ? 0.0 : (n > 0 ? nn * log(mu) - mu - lgamma(nn + 1.0) : -mu);
      atomicAdd(llh + h * M + k, pois + (n > 0 ? acc : 0.0));
    }
    __syncthreads();
  }
}

}  // namespace

extern "C" pp_status pp_event_llh_device(pp_ctx* c, int32_t mode, int64_t n_hyp, int64_t n_sources,
                                         int64_t n_modules, const double* d_params, const double* d_photons,
                                         const int64_t* d_offsets, const double* d_times, double* d_llh,
                                         void* stream) {
  pp::Range range_("pp_event_llh_device");
  if (!c) return PP_ERR_ARG;
  std::lock_guard<std::mutex> lk(pp::ctx_mutex(c));
  if (mode != PP_LLH_REFERENCE && mode != PP_LLH_SHIFTED) return pp::ctx_fail(c, PP_ERR_ARG, "unknown llh mode");
  if (n_hyp < 0 || n_sources < 1 || n_modules < 0 || n_hyp > 65535 || n_modules > (int64_t)INT32_MAX)
    return pp::ctx_fail(c, PP_ERR_ARG, "need n_sources >= 1, 0 <= n_hyp <= 65535, n_modules >= 0");
  if (n_hyp * n_modules == 0) return PP_OK;
  if (!d_params || !d_offsets || !d_times || !d_llh) return pp::ctx_fail(c, PP_ERR_ARG, "NULL buffer");
  int dev = pp::ctx_device(c), prev = -1;
  cudaGetDevice(&prev);
  if (prev != dev) cudaSetDevice(dev);
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  void* scratch = nullptr;
  cudaError_t e = pp::ctx_llh_scratch(c, (size_t)(n_modules + 1) * sizeof(int64_t), &scratch);
  if (!e) e = cudaMemsetAsync(d_llh, 0, (size_t)n_hyp * n_modules * sizeof(double), s);
  if (!e) {
    int64_t* cs = static_cast<int64_t*>(scratch);
    llh_chunk_scan_kernel<<<1, 1024, 0, s>>>(d_offsets, n_modules, cs);
    pp::count_launches(1);
    int sms = pp::ctx_sm_count(c);
    const int64_t items = (int64_t)sms * 8;  // blocks per hypothesis: grid-stride over the chunks
    dim3 grid((unsigned)std::min<int64_t>(items, std::max<int64_t>(n_modules, 1) * 4), (unsigned)n_hyp);
    llh_kernel<<<grid, kThreads, 0, s>>>(mode, n_sources, n_modules, d_params, d_photons, d_offsets, d_times, cs,
                                         d_llh);
    pp::count_launches(1);
    e = cudaGetLastError();
  }
  if (prev >= 0 && prev != dev) cudaSetDevice(prev);
  if (e) return pp::ctx_cuda_fail(c, e, "event llh");
  return PP_OK;
}
