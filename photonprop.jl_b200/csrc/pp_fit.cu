// Fit stage on the device: Cherenkov reweighting of hits and weighted Gamma
// maximum-likelihood fits per (pair, observation angle), the caller of the
// hot path in the reference (get_dir_reweight / fit_photon_dist /
// make_photon_fits, src/modelling.jl:46-111; cherenkov_ang_dist,
// src/emission.jl:32-44).
//
// Pipeline on one stream, no host round trip:
//   fit_count_kernel    hits per pair (stored hits only)
//   fit_scan_kernel     exclusive scan in place -> each pair's first record slot
//   fit_scatter_kernel  one 32-byte FitRec per hit, grouped by pair: the
//                       per-hit parts of the weight (cos/sin of the emission
//                       polar angle, 1/n, hit weight / (2 int(n))), tres, ln tres
//   fit_moments_kernel  one thread per observation angle walks a segment of
//                       records staged in shared memory, accumulates the four
//                       FP64 moments and flushes them when the pair changes
//   fit_gamma_kernel    Gamma MLE per (pair, angle) from the moments
// fit_columns_kernel builds the records straight from a hit table given as
// FP64 columns (fit_photon_dist over a DataFrame).
//
// The weighted Gamma MLE is the generalised Newton iteration of T. Minka,
// "Estimating a Gamma distribution" (2002), which is how Distributions.jl
// 0.25.62 fits Gamma(x, w) in the reference (fit_mle, src/modelling.jl:75):
// with mx = sum w x / sum w and ml = sum w ln x / sum w,
//   1/a' = 1/a + (ml - ln mx + ln a - psi(a)) / (a^2 (1/a - psi'(a))),
// started at a = (3 - s + sqrt((s - 3)^2 + 24 s)) / (12 s), s = ln mx - ml;
// theta = mx / a.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "pp_device.cuh"
#include "pp_internal.h"
#include "pp_special.cuh"

namespace ppd {

constexpr int kFitSeg = 2048;   // records per block segment of the moments kernel
constexpr int kFitTile = 256;   // records per shared-memory tile

__global__ void fit_count_kernel(const pp_hit* __restrict__ hits, const unsigned long long* __restrict__ counters,
                                 unsigned long long cap, int64_t n_pairs, unsigned long long* __restrict__ counts) {
  const unsigned long long n = min(counters[0], cap);
  for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (unsigned long long)gridDim.x * blockDim.x) {
    const uint32_t p = __ldg(&hits[i].pair);
    if ((int64_t)p >= n_pairs) continue;
    // one atomic per pair per warp: hits of one pair sit together in the buffer
    const unsigned grp = __match_any_sync(__activemask(), p);
    if ((threadIdx.x & 31u) == (unsigned)(__ffs(grp) - 1)) atomicAdd(counts + p, (unsigned long long)__popc(grp));
  }
}

// One block, in place: counts[i] becomes sum_{j < i} counts[j], the first
// record slot of pair i (the scatter's cursor).
__global__ void __launch_bounds__(1024) fit_scan_kernel(unsigned long long* __restrict__ counts, int64_t n) {
  __shared__ unsigned long long warp_tot[32];
  __shared__ unsigned long long carry;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int64_t base = 0; base < n; base += blockDim.x) {
    const int64_t i = base + threadIdx.x;
    const unsigned long long v = i < n ? counts[i] : 0ull;
    unsigned long long x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) warp_tot[warp] = x;
    __syncthreads();
    if (warp == 0) {
      const int nw = blockDim.x >> 5;
      unsigned long long t = lane < nw ? warp_tot[lane] : 0ull;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long y = __shfl_up_sync(0xffffffffu, t, o);
        if (lane >= o) t += y;
      }
      if (lane < nw) warp_tot[lane] = t;  // inclusive prefix of the warp totals
    }
    __syncthreads();
    const unsigned long long excl = carry + (warp > 0 ? warp_tot[warp - 1] : 0ull) + x - v;
    if (i < n) counts[i] = excl;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry = excl + v;
    __syncthreads();
  }
}

__device__ __forceinline__ float ang_norm(const pp::FitConsts& K, float n) {
  // 2 x LinearInterpolation(1.1:0.01:1.5, integral)(n); NaN outside like the reference's BoundsError
  const float x = (n - (float)pp::kAngIntN0) * K.inv_dn;
  if (!(x >= -1e-4f) || !(x <= (float)(pp::kAngIntN - 1) + 1e-4f)) return __int_as_float(0x7fc00000);
  int i = (int)floorf(x);
  i = min(max(i, 0), pp::kAngIntN - 2);
  const float f = x - (float)i;
  return 2.f * fmaf(K.normf[i + 1] - K.normf[i], f, K.normf[i]);
}

// The fit takes tres > 0 (the reference masks tres >= 0, src/modelling.jl:73,
// but a residual of exactly 0, which FP32 rounding makes common for photons
// that fly straight at the sphere, has ln 0 = -inf and no Gamma likelihood).
__device__ __forceinline__ void write_rec(pp::FitRec* r, float ct, float st, float c0, float wn, float tres, int pair) {
  const bool pos = tres > 0.f;
  const float lnt = pos ? logf(tres) : 0.f;
  float4* d = reinterpret_cast<float4*>(r);
  d[0] = make_float4(ct, st, c0, wn);
  d[1] = make_float4(tres, lnt, __int_as_float(pair), __int_as_float(pos ? 1 : 0));
}

__global__ void fit_scatter_kernel(const pp_hit* __restrict__ hits, const unsigned long long* __restrict__ counters,
                                   unsigned long long cap, const pp_pair* __restrict__ pairs, int64_t n_pairs,
                                   int mode, const DevTables* __restrict__ T, const pp::FitConsts K,
                                   unsigned long long* __restrict__ cursor, pp::FitRec* __restrict__ rec) {
  const unsigned long long n = min(counters[0], cap);
  for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (unsigned long long)gridDim.x * blockDim.x) {
    const float4* h = reinterpret_cast<const float4*>(hits + i);
    const float4 h0 = __ldg(h), h1 = __ldg(h + 1), h2 = __ldg(h + 2), h3 = __ldg(h + 3);
    const uint32_t p = __float_as_uint(h3.y);
    if ((int64_t)p >= n_pairs) continue;
    const float4* P = reinterpret_cast<const float4*>(pairs + p);
    const float4 pt = __ldg(P), dl = __ldg(P + 1), tg = __ldg(P + 2);
    // emission polar angle about the pair's axis (e_z when the axis is unset)
    const float a2 = fmaf(dl.x, dl.x, fmaf(dl.y, dl.y, dl.z * dl.z));
    float ct = a2 > 0.f ? fmaf(h1.x, dl.x, fmaf(h1.y, dl.y, h1.z * dl.z)) * rsqrtf(a2) : h1.z;
    ct = fminf(fmaxf(ct, -1.f), 1.f);
    const float st = sqrtf(fmaxf(0.f, fmaf(-ct, ct, 1.f)));
    const float wl = h2.w;
    const float n_ph = phase_index(*T, 1.f / wl);
    const float wn = h1.w / ang_norm(K, n_ph);
    const float dx = tg.x - pt.x, dy = tg.y - pt.y, dz = tg.z - pt.z;
    const float d = sqrtf(fmaf(dx, dx, fmaf(dy, dy, dz * dz)));
    const float tgeo = (d - tg.w) * (mode == kCompat ? K.n800_phase : K.n800_group) / kCVac;
    const float tres = h0.w - (mode == kCompat ? 0.f : pt.w) - tgeo;
    const unsigned grp = __match_any_sync(__activemask(), p);
    const unsigned lane = threadIdx.x & 31u;
    const int lead = __ffs(grp) - 1;
    unsigned long long base = 0;
    if ((int)lane == lead) base = atomicAdd(cursor + p, (unsigned long long)__popc(grp));
    base = __shfl_sync(grp, base, lead);
    write_rec(rec + base + __popc(grp & ((1u << lane) - 1u)), ct, st, 1.f / n_ph, wn, tres, (int)p);
  }
}

__global__ void fit_columns_kernel(int64_t n, const double* __restrict__ tres, const double* __restrict__ theta,
                                   const double* __restrict__ ref_ix, const double* __restrict__ abs_w,
                                   const double* __restrict__ wl, const DevTables* __restrict__ T,
                                   const pp::FitConsts K, pp::FitRec* __restrict__ rec) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double th = theta[i];
    const double nr = ref_ix[i];
    const float pmt = T->n_pmt > 0 ? interp_sorted((float)wl[i], T->pmt_wl, T->pmt_acc, T->n_pmt) : 1.f;
    const float w = (float)abs_w[i] * pmt;
    write_rec(rec + i, (float)cos(th), (float)sin(th), (float)(1.0 / nr), w / ang_norm(K, (float)nr),
              (float)tres[i], 0);
  }
}

// grid (segments, angle tiles); one thread per angle.
__global__ void __launch_bounds__(128) fit_moments_kernel(const pp::FitRec* __restrict__ rec,
                                                          const unsigned long long* __restrict__ n_ptr,
                                                          unsigned long long n_fixed, unsigned long long cap,
                                                          const float2* __restrict__ cs, int n_angles,
                                                          const pp::FitConsts K, double* __restrict__ moments) {
  __shared__ float4 tile[kFitTile][2];
  const unsigned long long n = n_ptr ? min(*n_ptr, cap) : n_fixed;
  const unsigned long long seg0 = (unsigned long long)blockIdx.x * kFitSeg;
  if (seg0 >= n) return;
  const unsigned long long seg1 = min(seg0 + (unsigned long long)kFitSeg, n);
  const int a = blockIdx.y * blockDim.x + threadIdx.x;
  const bool valid = a < n_angles;
  const float2 c = valid ? cs[a] : make_float2(1.f, 0.f);
  double m0 = 0.0, m1 = 0.0, m2 = 0.0, m3 = 0.0;
  int cur = -1;
  const float4* src = reinterpret_cast<const float4*>(rec);
  for (unsigned long long t0 = seg0; t0 < seg1; t0 += kFitTile) {
    const int cnt = (int)min((unsigned long long)kFitTile, seg1 - t0);
    __syncthreads();
    for (int j = threadIdx.x; j < 2 * cnt; j += blockDim.x) tile[j >> 1][j & 1] = src[2 * t0 + j];
    __syncthreads();
    for (int j = 0; j < cnt; ++j) {
      const float4 r0 = tile[j][0], r1 = tile[j][1];
      const int pair = __float_as_int(r1.z);
      if (pair != cur) {
        if (cur >= 0 && valid) {
          double* m = moments + ((int64_t)cur * n_angles + a) * PP_FIT_MOMENTS;
          atomicAdd(m + 0, m0);
          atomicAdd(m + 1, m1);
          atomicAdd(m + 2, m2);
          atomicAdd(m + 3, m3);
        }
        cur = pair;
        m0 = m1 = m2 = m3 = 0.0;
      }
      // cherenkov_ang_dist(cos(theta0 - a), n) x hit weight / (2 int(n))
      const float x = fmaf(r0.x, c.x, r0.y * c.y);
      const float pw = ex2(K.c * lg2(fabsf(x - r0.z)));
      const double w = (double)(fmaf(K.a, ex2(K.b_l2 * pw), K.d) * r0.w);
      m0 += w;
      if (__float_as_int(r1.w)) {
        m1 += w;
        m2 = fma(w, (double)r1.x, m2);
        m3 = fma(w, (double)r1.y, m3);
      }
    }
  }
  if (cur >= 0 && valid) {
    double* m = moments + ((int64_t)cur * n_angles + a) * PP_FIT_MOMENTS;
    atomicAdd(m + 0, m0);
    atomicAdd(m + 1, m1);
    atomicAdd(m + 2, m2);
    atomicAdd(m + 3, m3);
  }
}

__global__ void fit_gamma_kernel(const double* __restrict__ moments, int64_t rows, int n_angles,
                                 const pp_pair* __restrict__ pairs, int64_t n_gen, double* __restrict__ fits) {
  const int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= rows) return;
  const double* m = moments + row * PP_FIT_MOMENTS;
  const int64_t N = pairs ? pairs[row / n_angles].n_photons : n_gen;
  const double nan = __longlong_as_double(0x7ff8000000000000ll);
  double alpha = nan, theta = nan;
  if (m[1] > 0.0) {
    const double mx = m[2] / m[1];
    const double ml = m[3] / m[1];
    const double lmx = log(mx);
    const double s = lmx - ml;
    if (s > 0.0 && isfinite(s) && mx > 0.0) {
      double a = (3.0 - s + sqrt((s - 3.0) * (s - 3.0) + 24.0 * s)) / (12.0 * s);
      for (int it = 0; it < 100; ++it) {
        const double ia = 1.0 / a;
        const double z = ia + (ml - lmx + log(a) - ppsf::digamma_d(a)) / (a * a * (ia - ppsf::trigamma_d(a)));
        const double an = 1.0 / z;
        const bool done = fabs(an - a) <= 1e-14 * a;
        a = an;
        if (done || !(a > 0.0)) break;
      }
      if (a > 0.0 && isfinite(a)) {
        alpha = a;
        theta = mx / a;
      }
    }
  }
  fits[row * PP_FIT_OUT + 0] = alpha;
  fits[row * PP_FIT_OUT + 1] = theta;
  fits[row * PP_FIT_OUT + 2] = N > 0 ? m[0] / (double)N : nan;
}

}  // namespace ppd

namespace pp {

namespace {
int grid_for(int64_t n, int block, int sm_count) {
  const int64_t want = (n + block - 1) / block;
  return (int)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)sm_count * 8));
}

cudaError_t add_moments(const FitConsts& K, const FitRec* rec, const unsigned long long* n_ptr,
                        unsigned long long n_fixed, unsigned long long cap, const float2* cs, int n_angles,
                        double* moments, cudaStream_t s) {
  const unsigned long long span = n_ptr ? cap : n_fixed;
  if (span == 0) return cudaSuccess;
  const int block = std::min(128, ((n_angles + 31) / 32) * 32);
  dim3 grid((unsigned)((span + ppd::kFitSeg - 1) / ppd::kFitSeg), (unsigned)((n_angles + block - 1) / block));
  ppd::fit_moments_kernel<<<grid, block, 0, s>>>(rec, n_ptr, n_fixed, cap, cs, n_angles, K, moments);
  count_launches(1);
  return cudaGetLastError();
}
}  // namespace

void fill_fit_consts(FitConsts* K, double n800_phase, double n800_group) {
  K->a = (float)kAngA;
  K->b_l2 = (float)(kAngB / std::log(2.0));  // exp(b v) = 2^(b log2(e) v)
  K->c = (float)kAngC;
  K->d = (float)kAngD;
  K->n800_phase = (float)n800_phase;
  K->n800_group = (float)n800_group;
  K->inv_dn = (float)(1.0 / kAngIntDn);
  double t[kAngIntN];
  cherenkov_ang_dist_int_table(t);
  for (int i = 0; i < kAngIntN; ++i) K->normf[i] = (float)t[i];
}

cudaError_t launch_fit_gamma(const double* moments, int64_t n_pairs, int n_angles, const pp_pair* pairs,
                             int64_t n_gen, double* fits, cudaStream_t s) {
  const int64_t rows = n_pairs * n_angles;
  if (rows == 0) return cudaSuccess;
  ppd::fit_gamma_kernel<<<(unsigned)((rows + 127) / 128), 128, 0, s>>>(moments, rows, n_angles, pairs, n_gen, fits);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_fit_moments_hits(const FitConsts& K, const void* tables, const pp_pair* pairs, int64_t n_pairs,
                                    int mode, const pp_hit* hits, unsigned long long cap,
                                    const unsigned long long* counters, unsigned long long* counts, FitRec* rec,
                                    const float2* cs, int n_angles, double* moments, int sm_count, cudaStream_t s) {
  cudaError_t e;
  if (n_pairs == 0 || cap == 0) return cudaSuccess;
  if ((e = cudaMemsetAsync(counts, 0, (size_t)n_pairs * sizeof(unsigned long long), s))) return e;
  const int g = grid_for((int64_t)cap, 256, sm_count);
  ppd::fit_count_kernel<<<g, 256, 0, s>>>(hits, counters, cap, n_pairs, counts);
  count_launches(1);
  if ((e = cudaGetLastError())) return e;
  ppd::fit_scan_kernel<<<1, 1024, 0, s>>>(counts, n_pairs);
  count_launches(1);
  if ((e = cudaGetLastError())) return e;
  ppd::fit_scatter_kernel<<<g, 256, 0, s>>>(hits, counters, cap, pairs, n_pairs, mode,
                                            static_cast<const ppd::DevTables*>(tables), K, counts, rec);
  count_launches(1);
  if ((e = cudaGetLastError())) return e;
  return add_moments(K, rec, counters, 0, cap, cs, n_angles, moments, s);
}

cudaError_t launch_fit_columns(const FitConsts& K, const void* tables, int64_t n, const double* tres,
                               const double* theta, const double* ref_ix, const double* abs_w, const double* wl,
                               FitRec* rec, const float2* cs, int n_angles, int64_t n_gen, double* moments,
                               double* fits, int sm_count, cudaStream_t s) {
  cudaError_t e;
  if ((e = cudaMemsetAsync(moments, 0, (size_t)n_angles * PP_FIT_MOMENTS * sizeof(double), s))) return e;
  if (n > 0) {
    ppd::fit_columns_kernel<<<grid_for(n, 256, sm_count), 256, 0, s>>>(
        n, tres, theta, ref_ix, abs_w, wl, static_cast<const ppd::DevTables*>(tables), K, rec);
    count_launches(1);
    if ((e = cudaGetLastError())) return e;
    if ((e = add_moments(K, rec, nullptr, (unsigned long long)n, (unsigned long long)n, cs, n_angles, moments, s)))
      return e;
  }
  return launch_fit_gamma(moments, 1, n_angles, nullptr, n_gen, fits, s);
}

}  // namespace pp
