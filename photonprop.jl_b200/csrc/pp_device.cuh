// Device-side physics of the photon-propagation hot path (sm_100a).
//
// One photon lives in registers: position, direction, path length, step
// counter and two precomputed per-photon constants.  Its random numbers are
// Philox4x32-10 blocks addressed by (photon index, block) under the pair's
// seed, so nothing about the RNG is stored: block 0 holds the emission draws,
// block k+1 the draws of step k, and the emission values (wavelength,
// emission direction, emission time) are recomputed at a hit instead of
// being kept live through the step loop.
//
// Transcendentals use the approximate MUFU instructions through inline PTX
// (lg2/ex2/rcp/sqrt/sin/cos .approx); the rare hit path uses the accurate
// libm functions.  Reference arithmetic followed:
//   uniform / sph_to_cart / isotropic init  src/photon_prop_cuda.jl:26-56
//   HG cos(theta)                           src/photon_prop_cuda.jl:31-38
//   wavelength draw                         src/photon_prop_cuda.jl:73-75, src/utils.jl:37-60
//   rotate_to_axis / update_direction       src/photon_prop_cuda.jl:171-241
//   step, ray-sphere test, position update  src/photon_prop_cuda.jl:244-259,319-361
//   scattering length                       src/medium.jl:201-214
//   refractive index                        src/medium.jl:125-158
//   absorption length                       src/medium.jl:243-251
#pragma once

#include <cstdint>

#include "photonprop_b200.h"

namespace ppd {

constexpr float kCVac = 0.299792458f;   // m/ns
constexpr float kTwoPi = 6.28318530717958647692f;
constexpr float kPi = 3.14159265358979323846f;
constexpr float kLn2 = 0.69314718055994530942f;
constexpr float kLog2_550 = 9.10328780806166633225f;  // log2(550 nm), the scattering reference
constexpr unsigned kFull = 0xffffffffu;

enum { kCompat = PP_MODE_COMPAT, kPhysical = PP_MODE_PHYSICAL };

// ---- MUFU wrappers (PTX ISA .approx forms) -------------------------------
__device__ __forceinline__ float lg2(float x) {
  float r;
  asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ float ex2(float x) {
  float r;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ float rcp(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ float sqrt_a(float x) {
  float r;
  asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ float sin_a(float x) {
  float r;
  asm("sin.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ float cos_a(float x) {
  float r;
  asm("cos.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// ---- Philox4x32-10 (Salmon et al., SC'11) ---------------------------------
__host__ __device__ __forceinline__ void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint64_t p0 = (uint64_t)c[0] * 0xD2511F53u;
    const uint64_t p1 = (uint64_t)c[2] * 0xCD9E8D57u;
    const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c[1] ^ k0;
    const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c[3] ^ k1;
    c[0] = n0;
    c[1] = (uint32_t)p1;
    c[2] = n2;
    c[3] = (uint32_t)p0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
}

struct Draw4 {
  float u0, u1, u2, u3;
};

// ((w >> 9) + 1/2) * 2^-23, exact in FP32: 1.m - (1 - 2^-24).
__device__ __forceinline__ float u01(uint32_t w) {
  return __uint_as_float(0x3F800000u | (w >> 9)) - __uint_as_float(0x3F7FFFFFu);
}

__device__ __forceinline__ Draw4 draw_block(uint64_t photon, uint32_t block, uint32_t k0, uint32_t k1) {
  uint32_t c[4] = {(uint32_t)photon, (uint32_t)(photon >> 32), block, 0u};
  philox4x32_10(c, k0, k1);
  return Draw4{u01(c[0]), u01(c[1]), u01(c[2]), u01(c[3])};
}

// ---- resident tables (one copy per context, staged into shared memory) ----
struct DevTables {
  float a01, a2, a3, a4;   // phase index n = a01 + x(a2 + x(a3 + x a4)), x = 1/nm
  float g01, g2, g3, g4;   // group index a01 + x(2a2 + x(3a3 + x 4a4))
  float sca0, sca1, sca2;  // 0.0017, 1.34 c_small, 0.312 c_large
  int32_t n_knots;
  int32_t n_abs;
  int32_t n_pmt;
  int32_t pad0, pad1;
  float knots[PP_MAX_KNOTS];
  float abs_wl[PP_MAX_ABS];
  float abs_len[PP_MAX_ABS];
  float pmt_wl[PP_MAX_PMT];
  float pmt_acc[PP_MAX_PMT];
};
static_assert(sizeof(DevTables) % 16 == 0, "DevTables is copied as 16-byte words");

__device__ __forceinline__ void stage_tables(DevTables& s, const DevTables* __restrict__ g) {
  const int4* src = reinterpret_cast<const int4*>(g);
  int4* dst = reinterpret_cast<int4*>(&s);
  for (int i = threadIdx.x; i < (int)(sizeof(DevTables) / 16); i += blockDim.x) dst[i] = src[i];
}

__device__ __forceinline__ float phase_index(const DevTables& T, float x) {
  return fmaf(x, fmaf(x, fmaf(x, T.a4, T.a3), T.a2), T.a01);
}
__device__ __forceinline__ float group_index(const DevTables& T, float x) {
  return fmaf(x, fmaf(x, fmaf(x, T.g4, T.g3), T.g2), T.g01);
}
// 1 / (0.0017 y^4.3 + 1.34 c_s y^1.7 + 0.312 c_l y^0.3), y = 550 / wl.
__device__ __forceinline__ float scattering_length(const DevTables& T, float wl) {
  const float ly = kLog2_550 - lg2(wl);
  const float c = fmaf(T.sca0, ex2(4.3f * ly), fmaf(T.sca1, ex2(1.7f * ly), T.sca2 * ex2(0.3f * ly)));
  return rcp(c);
}

// fast_linear_interp(x, xs, ys) with the lower index clamped (src/utils.jl:10-34).
__device__ __forceinline__ float interp_sorted(float x, const float* xs, const float* ys, int n) {
  x = fminf(fmaxf(x, xs[0]), xs[n - 1]);
  int lo = 0, hi = n - 1;  // first index with xs[i] >= x, clamped to [1, n-1]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (xs[mid] < x) lo = mid; else hi = mid;
  }
  if (hi < 1) hi = 1;
  lo = hi - 1;
  const float along = (x - xs[lo]) / (xs[hi] - xs[lo]);
  return fmaf(ys[hi] - ys[lo], along, ys[lo]);
}

// fast_linear_interp(u, knots, 0, 1) for u in (0, 1) (src/utils.jl:37-60).
__device__ __forceinline__ float draw_wavelength(const DevTables& T, float u) {
  if (T.n_knots == 1) return T.knots[0];
  const float x = u * (float)(T.n_knots - 1);
  int i = (int)x;
  i = min(i, T.n_knots - 2);
  const float f = x - (float)i;
  return fmaf(T.knots[i + 1] - T.knots[i], f, T.knots[i]);
}

// cos(theta) of Henyey-Greenstein scattering (src/photon_prop_cuda.jl:31-38)
// with the launch constants of g folded: 1 - g + 2g u = 1 + g(2u - 1).
struct HG {
  float two_g, one_m_g, a, one_p_g2, inv_2g;
  int iso;
};
__device__ __forceinline__ float hg_costheta(const HG& h, float u) {
  if (h.iso) return fmaf(2.f, u, -1.f);
  const float t = h.a * rcp(fmaf(h.two_g, u, h.one_m_g));
  const float c = fmaf(-t, t, h.one_p_g2) * h.inv_2g;
  return fminf(fmaxf(c, -1.f), 1.f);
}

// Rotation that takes e_z to the unit vector o, applied to n (the Rodrigues
// form of rotate_to_axis, src/photon_prop_cuda.jl:171-219), written without
// sin(theta): the (1 - cos)/sin^2 factor is 1/(1 + o_z) on the upper
// hemisphere and (1 - o_z)/(o_x^2 + o_y^2) on the lower one, both well
// conditioned in FP32; o = -e_z maps n to (n_x, -n_y, -n_z) as in the
// reference.  One MUFU (rcp) instead of the reference's sqrt, 2 divides and
// rsqrt; the result is renormalised with one Newton step instead of rsqrt.
__device__ __forceinline__ void rotate_to_axis(float ox, float oy, float oz, float nx, float ny,
                                               float nz, float& rx, float& ry, float& rz) {
  const float q = fmaf(ox, ny, -oy * nx);
  const float s2 = fmaf(ox, ox, oy * oy);
  const bool up = oz >= 0.f;
  const float den = up ? 1.f + oz : s2;
  const float num = up ? 1.f : 1.f - oz;
  const float t = q * num * rcp(den);
  float x = fmaf(nx, oz, fmaf(ox, nz, -oy * t));
  float y = fmaf(ny, oz, fmaf(oy, nz, ox * t));
  float z = fmaf(nz, oz, -fmaf(ox, nx, oy * ny));
  if (den == 0.f) {
    x = nx;
    y = -ny;
    z = -nz;
  }
  const float f = fmaf(-0.5f, fmaf(x, x, fmaf(y, y, z * z)), 1.5f);
  rx = x * f;
  ry = y * f;
  rz = z * f;
}

struct Emission {
  float px, py, pz;
  float dx, dy, dz;
  float wl;
  float t_emit;
};

// Emission of one photon from block 0 of its stream (src/photon_prop_cuda.jl:52-56,
// 67-75, 308-316; the Cherenkov cone has no reference code: a point uniform
// along the track, angle acos(1/n(wl)) about the track axis, time t0 + s/c).
template <int MODE>
__device__ __forceinline__ Emission emit_photon(const DevTables& T, const pp_pair& P, uint64_t photon,
                                                uint32_t k0, uint32_t k1) {
  const Draw4 d = draw_block(photon, 0u, k0, k1);
  Emission e;
  e.wl = draw_wavelength(T, d.u0);
  // phi = 2 pi u2; evaluated as phi - pi in [-pi, pi) and negated.
  const float ph = fmaf(kTwoPi, d.u2, -kPi);
  const float sphi = -sin_a(ph), cphi = -cos_a(ph);
  if (P.emitter == PP_EMITTER_ISOTROPIC) {
    float st, ct;
    if (MODE == kCompat) {  // theta = uniform(-1, 1) radians (reference quirk)
      const float th = fmaf(2.f, d.u1, -1.f);
      st = sin_a(th);
      ct = cos_a(th);
    } else {
      ct = fmaf(2.f, d.u1, -1.f);
      st = sqrt_a(fmaxf(0.f, fmaf(-ct, ct, 1.f)));
    }
    e.dx = cphi * st;
    e.dy = sphi * st;
    e.dz = ct;
    e.px = P.pos[0];
    e.py = P.pos[1];
    e.pz = P.pos[2];
    e.t_emit = P.t0;
  } else {
    const float ct = rcp(phase_index(T, rcp(e.wl)));
    const float st = sqrt_a(fmaxf(0.f, fmaf(-ct, ct, 1.f)));
    rotate_to_axis(P.dir[0], P.dir[1], P.dir[2], cphi * st, sphi * st, ct, e.dx, e.dy, e.dz);
    const float s = d.u1 * P.track_len;
    e.px = fmaf(s, P.dir[0], P.pos[0]);
    e.py = fmaf(s, P.dir[1], P.pos[1]);
    e.pz = fmaf(s, P.dir[2], P.pos[2]);
    e.t_emit = fmaf(s, 1.f / kCVac, P.t0);
  }
  return e;
}

// Per-launch constants.
struct RunParams {
  const pp_pair* __restrict__ pairs;
  int64_t n_pairs;
  const unsigned long long* __restrict__ chunk_offsets;  // [n_pairs + 1]
  unsigned long long* __restrict__ queue;                // [0]: next chunk
  uint32_t chunk;
  uint32_t pair_base;  // added to the pair index written into hits
  pp_hit* __restrict__ hits;
  unsigned long long hit_cap;
  unsigned long long* __restrict__ counters;  // [0] hits, [1] steps, [2] status bits
  double* __restrict__ stats;                 // [n_pairs x PP_STATS]
  double* __restrict__ hist;                  // [n_pairs x hist_bins]
  const DevTables* __restrict__ tables;
  int32_t max_steps;
  float t_max;
  float hist_t0;
  float inv_bin_width;
  int32_t hist_bins;
  uint32_t flags;
  HG hg;
};

// Registers of one live photon.
struct Photon {
  float px, py, pz;
  float dx, dy, dz;
  float dist;
  float neg_ln2_len;  // -ln2 * scattering length: step = lg2(u) * this
  float max_dist;     // physical mode: path length at t_max
  int32_t k;          // steps taken
  uint64_t id;
};

struct PairCtx {
  float tx, ty, tz, r2;
  uint32_t k0, k1;
  int32_t index;
};

__device__ __forceinline__ PairCtx load_pair_ctx(const pp_pair& P, int index) {
  PairCtx c;
  c.tx = P.target[0];
  c.ty = P.target[1];
  c.tz = P.target[2];
  c.r2 = P.radius * P.radius;
  c.k0 = (uint32_t)P.seed;
  c.k1 = (uint32_t)(P.seed >> 32);
  c.index = index;
  return c;
}

template <int MODE>
__device__ __forceinline__ void start_photon(const DevTables& T, const pp_pair& P, const PairCtx& c,
                                             const RunParams& R, uint64_t id, Photon& s) {
  const Emission e = emit_photon<MODE>(T, P, id, c.k0, c.k1);
  s.px = e.px;
  s.py = e.py;
  s.pz = e.pz;
  s.dx = e.dx;
  s.dy = e.dy;
  s.dz = e.dz;
  s.dist = 0.f;
  s.k = 0;
  s.id = id;
  s.neg_ln2_len = -kLn2 * scattering_length(T, e.wl);
  if (MODE == kPhysical) {
    s.max_dist = (R.t_max - e.t_emit) * kCVac * rcp(group_index(T, rcp(e.wl)));
  } else {
    s.max_dist = 3.0e38f;
  }
}

// One step of src/photon_prop_cuda.jl:320-376.  Returns false when the photon
// ends; *hit is set when it ends on the sphere (position and path length
// then point at the hit).
template <int MODE>
__device__ __forceinline__ bool step_photon(const RunParams& R, const PairCtx& c, Photon& s, bool& hit) {
  s.k += 1;
  const Draw4 d = draw_block(s.id, (uint32_t)s.k, c.k0, c.k1);
  const float step = lg2(d.u0) * s.neg_ln2_len;
  const float ex = s.px - c.tx, ey = s.py - c.ty, ez = s.pz - c.tz;
  const float a = fmaf(s.dz, ez, fmaf(s.dy, ey, s.dx * ex));
  const float pp = fmaf(ez, ez, fmaf(ey, ey, ex * ex));
  const float b = fmaf(a, a, c.r2 - pp);
  bool alive = true;
  bool move = true;
  if (b >= 0.f) {
    const float dd = -a - sqrt_a(b);
    if (dd > 0.f && dd < step) {
      move = false;
      alive = false;
      if (MODE == kCompat || s.dist + dd <= s.max_dist) {
        hit = true;
        s.px = fmaf(dd, s.dx, s.px);
        s.py = fmaf(dd, s.dy, s.py);
        s.pz = fmaf(dd, s.dz, s.pz);
        s.dist += dd;
      }
    } else if (MODE == kCompat) {
      move = false;  // the line meets the sphere outside this step: no move (reference)
    }
  }
  if (move) {
    if (MODE == kPhysical && s.dist + step > s.max_dist) {
      alive = false;
    } else {
      s.px = fmaf(step, s.dx, s.px);
      s.py = fmaf(step, s.dy, s.py);
      s.pz = fmaf(step, s.dz, s.pz);
      s.dist += step;
      const float ct = hg_costheta(R.hg, d.u1);
      const float st = sqrt_a(fmaxf(0.f, fmaf(-ct, ct, 1.f)));
      const float ph = fmaf(kTwoPi, d.u2, -kPi);
      const float nx = -cos_a(ph) * st, ny = -sin_a(ph) * st;
      rotate_to_axis(s.dx, s.dy, s.dz, nx, ny, ct, s.dx, s.dy, s.dz);
    }
  }
  if (s.k >= R.max_steps) alive = false;
  return alive;
}

// Everything a hit record needs (src/photon_prop_cuda.jl:622,634-641).
struct HitValues {
  float time, weight, wl;
  float d0x, d0y, d0z;
};

template <int MODE>
__device__ __forceinline__ HitValues hit_values(const DevTables& T, const RunParams& R, const pp_pair& P,
                                                const PairCtx& c, const Photon& s) {
  const Emission e = emit_photon<MODE>(T, P, s.id, c.k0, c.k1);
  HitValues h;
  h.wl = e.wl;
  h.d0x = e.dx;
  h.d0y = e.dy;
  h.d0z = e.dz;
  const float x = 1.f / e.wl;
  if (MODE == kCompat) {
    h.time = s.dist * phase_index(T, x) / kCVac;  // phase velocity (reference)
  } else {
    h.time = e.t_emit + s.dist * group_index(T, x) / kCVac;
  }
  float w = expf(-s.dist / interp_sorted(e.wl, T.abs_wl, T.abs_len, T.n_abs));
  if ((R.flags & PP_OPT_PMT_WEIGHT) && T.n_pmt > 0) w *= interp_sorted(e.wl, T.pmt_wl, T.pmt_acc, T.n_pmt);
  h.weight = w;
  return h;
}

// Per-pair FP64 accumulation, histogram and warp-aggregated hit write-back.
__device__ __forceinline__ void record_hit(const RunParams& R, const PairCtx& c, const Photon& s,
                                           const HitValues& h, int stats_row) {
  double* st = R.stats + (int64_t)stats_row * PP_STATS;
  const double w = (double)h.weight;
  const double t = (double)h.time;
  atomicAdd(st + 0, 1.0);
  atomicAdd(st + 1, w);
  atomicAdd(st + 2, w * w);
  atomicAdd(st + 3, w * t);
  atomicAdd(st + 4, w * t * t);
  atomicAdd(st + 5, w * (double)logf(h.time));
  if (R.hist_bins > 0) {
    const float fb = floorf((h.time - R.hist_t0) * R.inv_bin_width);
    if (fb >= 0.f && fb < (float)R.hist_bins)
      atomicAdd(R.hist + (int64_t)stats_row * R.hist_bins + (int)fb, w);
  }
  // warp-aggregated slot reservation among the lanes that hit in this step
  const unsigned m = __activemask();
  const int leader = __ffs(m) - 1;
  const unsigned lane = threadIdx.x & 31u;
  const unsigned rank = __popc(m & ((1u << lane) - 1u));
  unsigned long long base = 0;
  if ((int)lane == leader) base = atomicAdd(R.counters + 0, (unsigned long long)__popc(m));
  base = __shfl_sync(m, base, leader);
  if (R.flags & PP_OPT_NO_HITS) return;
  const unsigned long long idx = base + rank;
  if (idx < R.hit_cap) {
    float4* dst = reinterpret_cast<float4*>(R.hits + idx);
    dst[0] = make_float4(s.px, s.py, s.pz, h.time);
    dst[1] = make_float4(h.d0x, h.d0y, h.d0z, h.weight);
    dst[2] = make_float4(s.dx, s.dy, s.dz, h.wl);
    dst[3] = make_float4(s.dist, __uint_as_float((uint32_t)c.index + R.pair_base),
                         __uint_as_float((uint32_t)s.id), __uint_as_float((uint32_t)(s.id >> 32)));
  } else {
    atomicOr(R.counters + 2, 1ull);
  }
}

}  // namespace ppd
