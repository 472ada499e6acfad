// Light yield of electromagnetic cascades: particles -> Cherenkov light
// sources (src/lightyield.jl), on the host in FP64 and, for many particles
// at once, on the device.
//
//   longitudinal_profile   b ((t b)^(a-1) e^(-t b) / Gamma(a)),
//                          t = z / L_rad, a = alpha + beta log10(E)
//                          (src/lightyield.jl:116-140, parameters :35-37)
//   cherenkov_track_length alpha E^beta cm (src/lightyield.jl:190-198, :46-69)
//   fractional_contrib_long the profile's share of each grid interval,
//                          50-point Gauss-Legendre (src/lightyield.jl:143-169)
//   particle_to_elongated_lightsource one source per interval at its midpoint
//                          with round(frank_tamm_norm x track length x share)
//                          photons (src/lightyield.jl:219-285)
// L_rad = X0 / density x 1000 cm with X0 in g/cm^2 and the density in kg/m^3
// (src/lightyield.jl:121-122).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <vector>

#include "pp_internal.h"

namespace {

struct LongPars {
  double alpha, beta, b;
};
struct TrackPars {
  double alpha, beta, alpha_dev, beta_dev;
};

// src/lightyield.jl:35-37 and :46-69
bool params_of(int ptype, LongPars* lp, TrackPars* tp) {
  switch (ptype) {
    case PP_PARTICLE_EMINUS:
      *lp = {2.01849, 1.45469, 0.63207};
      *tp = {532.07078881, 1.00000211, 5.78170887, 0.5};
      return true;
    case PP_PARTICLE_EPLUS:
      *lp = {2.00035, 1.45501, 0.63008};
      *tp = {532.11320598, 0.99999254, 5.73419669, 0.5};
      return true;
    case PP_PARTICLE_GAMMA:
      *lp = {2.83923, 1.34031, 0.64526};
      *tp = {532.08540905, 0.99999877, 5.78170887, 5.66586567};
      return true;
    default:
      return false;
  }
}

// DIPPR105 water density, DDB parameters (src/medium.jl:60-78).
constexpr double kDA = 0.14395, kDB = 0.0112, kDC = 649.727, kDD = 0.05107;

double density(const pp_medium_desc* m, int mode) {
  const double T = m->temperature;
  if (mode == PP_LY_REFERENCE) return kDA / std::pow(kDB, std::pow(1.0 + (1.0 - T) / kDC, kDD));
  return kDA / std::pow(kDB, 1.0 + std::pow(1.0 - (T + 273.15) / kDC, kDD));
}

double rad_length_cm(const pp_medium_desc* m, int mode) { return m->radiation_length / density(m, mode) * 1000.0; }

double profile(const LongPars& p, double lrad, double e, double z_cm) {
  const double t = z_cm / lrad;
  const double a = p.alpha + p.beta * std::log10(e);
  return p.b * (std::pow(t * p.b, a - 1.0) * std::exp(-(t * p.b)) / std::tgamma(a));
}

double gl_integral(const LongPars& p, double lrad, double e, double lo, double hi, const double* x, const double* w) {
  const double half = (hi - lo) / 2.0, mid = (hi + lo) / 2.0;
  double s = 0.0;
  for (int i = 0; i < 50; ++i) s += w[i] * profile(p, lrad, e, half * x[i] + mid) * half;
  return s;
}

int64_t grid_points(double lo, double hi, double step) {
  if (!(step > 0.0) || !(hi >= lo)) return 0;
  return (int64_t)std::floor((hi - lo) / step * (1.0 + 1e-12) + 1e-9) + 1;
}

constexpr double kCVacD = 0.299792458;  // m/ns

struct LyParams {
  double x[50], w[50];
  double lrad;  // cm
  double ft_norm;  // photons per cm
  double len_min, step;
  int64_t n_grid;
  int32_t mode, emitter;
};

__device__ double d_profile(double alpha, double beta, double b, double lrad, double e, double z_cm) {
  const double t = z_cm / lrad;
  const double a = alpha + beta * log10(e);
  return b * (pow(t * b, a - 1.0) * exp(-(t * b)) / tgamma(a));
}

__device__ double d_gl(const LyParams& P, double alpha, double beta, double b, double e, double lo, double hi) {
  const double half = (hi - lo) / 2.0, mid = (hi + lo) / 2.0;
  double s = 0.0;
  for (int i = 0; i < 50; ++i) s += P.w[i] * d_profile(alpha, beta, b, P.lrad, e, half * P.x[i] + mid) * half;
  return s;
}

// One thread per (particle, interval).
__global__ void sources_kernel(const pp_particle* __restrict__ parts, int64_t n_particles, const LyParams P,
                               pp_pair* __restrict__ out) {
  const int64_t n_int = P.n_grid - 1;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_particles * n_int) return;
  const int64_t pi = i / n_int, k = i % n_int;
  const pp_particle q = parts[pi];
  double alpha, beta, b, ta, tb;
  if (q.type == PP_PARTICLE_EPLUS) {
    alpha = 2.00035; beta = 1.45501; b = 0.63008; ta = 532.11320598; tb = 0.99999254;
  } else if (q.type == PP_PARTICLE_GAMMA) {
    alpha = 2.83923; beta = 1.34031; b = 0.64526; ta = 532.08540905; tb = 0.99999877;
  } else {  // PP_PARTICLE_EMINUS; another type gives emitter -1, which propagation rejects
    alpha = 2.01849; beta = 1.45469; b = 0.63207; ta = 532.07078881; tb = 1.00000211;
  }
  const bool known = q.type == PP_PARTICLE_EMINUS || q.type == PP_PARTICLE_EPLUS || q.type == PP_PARTICLE_GAMMA;
  const double e = (double)q.energy;
  const double g0 = P.len_min, g1 = P.len_min + (double)(P.n_grid - 1) * P.step;
  const double lo = P.len_min + (double)k * P.step, hi = P.len_min + (double)(k + 1) * P.step;
  const double to_cm = P.mode == PP_LY_REFERENCE ? 1.0 : 100.0;
  const double norm = d_gl(P, alpha, beta, b, e, g0 * to_cm, g1 * to_cm);
  const double share = d_gl(P, alpha, beta, b, e, lo * to_cm, hi * to_cm) / norm;
  const double total = P.ft_norm * (ta * pow(e, tb));
  const double mid = 0.5 * (lo + hi);  // metres along the particle
  pp_pair s;
  s.dir[0] = q.dir[0];
  s.dir[1] = q.dir[1];
  s.dir[2] = q.dir[2];
  double start = mid;
  if (P.emitter == PP_EMITTER_CHERENKOV_CONE) {
    start = lo;
    s.track_len = (float)(hi - lo);
  } else {
    s.track_len = 0.f;
  }
  s.pos[0] = (float)((double)q.pos[0] + start * (double)q.dir[0]);
  s.pos[1] = (float)((double)q.pos[1] + start * (double)q.dir[1]);
  s.pos[2] = (float)((double)q.pos[2] + start * (double)q.dir[2]);
  s.t0 = (float)((double)q.time + start / kCVacD);
  s.target[0] = s.target[1] = s.target[2] = 0.f;
  s.radius = 0.f;
  s.n_photons = known ? __double2ll_rn(total * share) : 0;  // round half to even, as Julia's round
  s.seed = 0;
  s.emitter = known ? P.emitter : -1;
  s.reserved[0] = s.reserved[1] = s.reserved[2] = 0;
  out[i] = s;
}

__global__ void cross_kernel(const pp_pair* __restrict__ src, int64_t n_s, const float4* __restrict__ tg, int64_t n_t,
                             uint64_t seed, pp_pair* __restrict__ out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_s * n_t) return;
  pp_pair p = src[i / n_t];
  const float4 t = tg[i % n_t];
  p.target[0] = t.x;
  p.target[1] = t.y;
  p.target[2] = t.z;
  p.radius = t.w;
  // splitmix64 of (seed, index), the same per-pair seed as pp_pair_seed
  uint64_t z = seed + 0x9E3779B97F4A7C15ull * ((uint64_t)i + 1ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  p.seed = z ^ (z >> 31);
  out[i] = p;
}

}  // namespace

extern "C" {

double pp_medium_density(const pp_medium_desc* m, int32_t mode) {
  if (!m || (mode != PP_LY_REFERENCE && mode != PP_LY_METRES)) return NAN;
  return density(m, mode);
}

double pp_longitudinal_profile(const pp_medium_desc* m, int32_t mode, int32_t ptype, double e, double z_cm) {
  LongPars lp;
  TrackPars tp;
  if (!m || !params_of(ptype, &lp, &tp) || (mode != PP_LY_REFERENCE && mode != PP_LY_METRES)) return NAN;
  return profile(lp, rad_length_cm(m, mode), e, z_cm);
}

double pp_cherenkov_track_length(int32_t ptype, double e) {
  LongPars lp;
  TrackPars tp;
  if (!params_of(ptype, &lp, &tp)) return NAN;
  return tp.alpha * std::pow(e, tp.beta);
}

double pp_cherenkov_track_length_dev(int32_t ptype, double e) {
  LongPars lp;
  TrackPars tp;
  if (!params_of(ptype, &lp, &tp)) return NAN;
  return tp.alpha_dev * std::pow(e, tp.beta_dev);
}

double pp_frank_tamm_norm(const pp_medium_desc* m, double wl_min, double wl_max) {
  if (!m || !(wl_max > wl_min) || !(wl_min > 0.0)) return NAN;
  return pp::frank_tamm_norm_cm(m, wl_min, wl_max);
}

pp_status pp_fractional_contrib_long(const pp_medium_desc* m, int32_t mode, int32_t ptype, double e,
                                     const double* z, int64_t n, double* out) {
  LongPars lp;
  TrackPars tp;
  if (!m || !params_of(ptype, &lp, &tp) || (mode != PP_LY_REFERENCE && mode != PP_LY_METRES) || n < 1 || !z ||
      !out)
    return PP_ERR_ARG;
  double x[50], w[50];
  pp::gl_nodes(50, x, w);
  const double lrad = rad_length_cm(m, mode);
  double lo = z[0], hi = z[0];
  for (int64_t i = 0; i < n; ++i) {
    lo = std::min(lo, z[i]);
    hi = std::max(hi, z[i]);
  }
  const double norm = gl_integral(lp, lrad, e, lo, hi, x, w);
  out[0] = 0.0;
  for (int64_t i = 0; i + 1 < n; ++i) out[i + 1] = gl_integral(lp, lrad, e, z[i], z[i + 1], x, w) / norm;
  return PP_OK;
}

pp_status pp_particles_to_sources_device(pp_ctx* c, const pp_particle* d_parts, int64_t n_particles,
                                         double len_min, double len_max, double precision, int32_t mode,
                                         double wl_min, double wl_max, int32_t emitter, pp_pair* d_sources,
                                         int64_t capacity, int64_t* n_grid, void* stream) {
  if (!c) return PP_ERR_ARG;
  std::lock_guard<std::mutex> lk(pp::ctx_mutex(c));
  if (mode != PP_LY_REFERENCE && mode != PP_LY_METRES)
    return pp::ctx_fail(c, PP_ERR_ARG, "unknown light-yield length mode");
  if (emitter != PP_EMITTER_ISOTROPIC && emitter != PP_EMITTER_CHERENKOV_CONE && emitter != PP_EMITTER_CASCADE)
    return pp::ctx_fail(c, PP_ERR_ARG, "unknown emitter");
  if (!(wl_max > wl_min) || !(wl_min > 0.0)) return pp::ctx_fail(c, PP_ERR_ARG, "bad wavelength range");
  const int64_t ng = grid_points(len_min, len_max, precision);
  if (ng < 2) return pp::ctx_fail(c, PP_ERR_ARG, "the grid len_min:precision:len_max needs at least two points");
  if (n_grid) *n_grid = ng;
  if (n_particles < 0 || (n_particles > 0 && (!d_parts || !d_sources)))
    return pp::ctx_fail(c, PP_ERR_ARG, "bad particle or source buffers");
  if (n_particles * (ng - 1) > capacity) return pp::ctx_fail(c, PP_ERR_ARG, "source capacity too small");
  if (n_particles == 0) return PP_OK;
  LyParams P;
  pp::gl_nodes(50, P.x, P.w);
  P.lrad = rad_length_cm(pp::ctx_medium(c), mode);
  P.ft_norm = pp::frank_tamm_norm_cm(pp::ctx_medium(c), wl_min, wl_max);
  P.len_min = len_min;
  P.step = precision;
  P.n_grid = ng;
  P.mode = mode;
  P.emitter = emitter;
  int dev = pp::ctx_device(c), prev = -1;
  cudaGetDevice(&prev);
  if (prev != dev) cudaSetDevice(dev);
  const int64_t total = n_particles * (ng - 1);
  sources_kernel<<<(unsigned)((total + 127) / 128), 128, 0, static_cast<cudaStream_t>(stream)>>>(d_parts, n_particles,
                                                                                                  P, d_sources);
  pp::count_launches(1);
  cudaError_t e = cudaGetLastError();
  if (prev >= 0 && prev != dev) cudaSetDevice(prev);
  if (e) return pp::ctx_cuda_fail(c, e, "particles_to_sources");
  return PP_OK;
}

pp_status pp_cross_pairs_device(pp_ctx* c, const pp_pair* d_sources, int64_t n_s, const float* d_targets, int64_t n_t,
                                uint64_t seed, pp_pair* d_pairs, void* stream) {
  if (!c) return PP_ERR_ARG;
  std::lock_guard<std::mutex> lk(pp::ctx_mutex(c));
  if (n_s < 0 || n_t < 0 || (n_s * n_t > 0 && (!d_sources || !d_targets || !d_pairs)))
    return pp::ctx_fail(c, PP_ERR_ARG, "bad cross-pair arguments");
  if (((uintptr_t)d_targets & 15) || ((uintptr_t)d_pairs & 15) || ((uintptr_t)d_sources & 15))
    return pp::ctx_fail(c, PP_ERR_ARG, "sources, targets and pairs need 16-byte alignment");
  const int64_t total = n_s * n_t;
  if (total == 0) return PP_OK;
  int dev = pp::ctx_device(c), prev = -1;
  cudaGetDevice(&prev);
  if (prev != dev) cudaSetDevice(dev);
  cross_kernel<<<(unsigned)((total + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      d_sources, n_s, reinterpret_cast<const float4*>(d_targets), n_t, seed, d_pairs);
  pp::count_launches(1);
  cudaError_t e = cudaGetLastError();
  if (prev >= 0 && prev != dev) cudaSetDevice(prev);
  if (e) return pp::ctx_cuda_fail(c, e, "cross_pairs");
  return PP_OK;
}

}  // extern "C"
