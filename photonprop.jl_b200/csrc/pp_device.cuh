// Device-side physics of the photon-propagation hot path (sm_100a).
//
// One photon lives in registers: position, direction, path length, step
// counter and two precomputed per-photon constants.  Its random numbers are
// Philox4x32-10 blocks under a fixed library key with the counter
// (seed lo, seed hi, photon lo, photon hi | block << 8): the pair's 64-bit
// seed, a photon index below 2^40 and a block below 2^24.  Nothing about the
// RNG is stored: block 0 holds the emission draws, block k+1 the draws of
// step k, and the emission values (wavelength, emission direction, emission
// time) are recomputed at a hit instead of being kept live through the step
// loop.  With the key fixed, the ten round keys are immediates.
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
__device__ __forceinline__ float rsqrt_a(float x) {
  float r;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
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
// Each round's products are written as a 32-bit high half (__umulhi) and a
// 32-bit low product rather than as one 64-bit product: the same numbers,
// but on sm_100a the 64-bit form cost two extra integer adds per round on the
// half-rate ALU pipe (ncu opcode counts of the bare step); this form ran the
// bare step 16 % and the batched kernel 10 % faster.
__host__ __device__ __forceinline__ void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
#ifdef __CUDA_ARCH__
    const uint32_t h0 = __umulhi(c[0], 0xD2511F53u), l0 = c[0] * 0xD2511F53u;
    const uint32_t h1 = __umulhi(c[2], 0xCD9E8D57u), l1 = c[2] * 0xCD9E8D57u;
#else
    const uint64_t p0 = (uint64_t)c[0] * 0xD2511F53u, p1 = (uint64_t)c[2] * 0xCD9E8D57u;
    const uint32_t h0 = (uint32_t)(p0 >> 32), l0 = (uint32_t)p0, h1 = (uint32_t)(p1 >> 32), l1 = (uint32_t)p1;
#endif
    const uint32_t n0 = h1 ^ c[1] ^ k0;
    const uint32_t n2 = h0 ^ c[3] ^ k1;
    c[0] = n0;
    c[1] = l1;
    c[2] = n2;
    c[3] = l0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
}

// Philox2x32-10 (same paper): one multiplier and one key word.  A block gives
// 64 bits for two 32x32 products per round, against 128 bits for four in a
// Philox4x32 block; a step needs 63 bits.  Under a fixed key (the steps') the
// round keys are immediates.
__host__ __device__ __forceinline__ void philox2x32_10(uint32_t& c0, uint32_t& c1, uint32_t k) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
#ifdef __CUDA_ARCH__
    const uint32_t h = __umulhi(c0, 0xD256D193u), l = c0 * 0xD256D193u;
#else
    const uint64_t p = (uint64_t)c0 * 0xD256D193u;
    const uint32_t h = (uint32_t)(p >> 32), l = (uint32_t)p;
#endif
    c0 = h ^ k ^ c1;
    c1 = l;
    k += 0x9E3779B9u;
  }
}

struct Draw3 {
  float u0, u1, u2;
};

// ((w >> 9) + 1/2) * 2^-23, exact in FP32: 1.m - (1 - 2^-24).  The mantissa
// bits (w >> 9) are placed with one integer multiply-add, hi(w * 2^23) +
// bits(1.0f), which runs on the FMA pipe instead of a shift and an OR on the
// half-rate ALU pipe.
__device__ __forceinline__ float u01(uint32_t w) {
  uint32_t m;
  asm("mad.hi.u32 %0, %1, %2, %3;" : "=r"(m) : "r"(w), "r"(1u << 23), "r"(0x3F800000u));
  return __uint_as_float(m) - __uint_as_float(0x3F7FFFFFu);
}

constexpr uint32_t kKey0 = 0x243F6A88u;  // fixed Philox4x32 key of the emission blocks (hex digits of pi)
constexpr uint32_t kKey1 = 0x85A308D3u;
constexpr uint32_t kStepKey = 0x13198A2Eu;  // fixed Philox2x32 key of the step blocks (the digits that follow)

// Photon index bits 32..39 and a step's block number (step k: k + 1) above
// them: word 3 of the emission counter (block 0) and word 1 of the step
// counter.
__device__ __forceinline__ uint32_t ctr_word(uint64_t photon, uint32_t block) {
  return (uint32_t)(photon >> 32) | (block << 8);
}

// Emission block of a photon: Philox4x32-10 under the fixed key with counter
// (seed lo, seed hi, photon lo, photon hi).  Words 0..2 give the emission's
// uniforms (their top 23 bits); word 3 and the low 9 bits of words 0..2 name
// the photon's step stream: step k is the Philox2x32-10 block under the
// fixed step key at counter (word 3, base + ctr_word(photon, k + 1)), where
// base packs those 27 low bits.
__device__ __forceinline__ uint4 emission_block(uint32_t seed_lo, uint32_t seed_hi, uint64_t photon) {
  uint32_t c[4] = {seed_lo, seed_hi, (uint32_t)photon, ctr_word(photon, 0u)};
  philox4x32_10(c, kKey0, kKey1);
  return make_uint4(c[0], c[1], c[2], c[3]);
}
__device__ __forceinline__ Draw3 emission_uniforms(const uint4& w) { return Draw3{u01(w.x), u01(w.y), u01(w.z)}; }
__device__ __forceinline__ uint32_t step_base(const uint4& w) {
  return (w.x & 0x1FFu) | ((w.y & 0x1FFu) << 9) | ((w.z & 0x1FFu) << 18);
}

// A step's three uniforms from its Philox2x32 block (w0, w1): bits 63..43,
// 42..22 and 21..1 of w0:w1, each placed in mantissa bits 22..2 of 1.m with
// bit 1 set, so that 1.m - 1 = (k + 1/2) 2^-21 exactly.
// The first and third fields are shifted into place by integer multiply-adds
// (FMA pipe) rather than shifts (the half-rate ALU pipe): the same bits.
__device__ __forceinline__ Draw3 step_uniforms(uint32_t w0, uint32_t w1) {
  uint32_t b0, b2;
  asm("mad.hi.u32 %0, %1, %2, %3;" : "=r"(b0) : "r"(w0 & 0xFFFFF800u), "r"(1u << 23), "r"(0x3F800002u));
  asm("mad.lo.u32 %0, %1, %2, %3;" : "=r"(b2) : "r"(w1 & 0x003FFFFEu), "r"(2u), "r"(0x3F800002u));
  const uint32_t m1 = __funnelshift_r(w1, w0, 20) & 0x7FFFFCu;
  return Draw3{__uint_as_float(b0) - 1.f, __uint_as_float(m1 | 0x3F800002u) - 1.f, __uint_as_float(b2) - 1.f};
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
  // cascade emitter: device tables (forward G, then inverse v) and their grids
  const float* casc;
  float casc_vmin, casc_inv_dv, casc_gmin, casc_inv_dg;
  int32_t casc_nf, casc_ni;
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

// cos(theta) of the cascade emitter: inverse-CDF sample of
// a exp(b |x - c0|^c) + d on [-1, 1], c0 = 1/n (cherenkov_ang_dist,
// src/emission.jl:32-44), from the tables of G(v) = integral of the profile.
__device__ __forceinline__ float casc_lerp(const float* __restrict__ t, int cells, float x) {
  x = fminf(fmaxf(x, 0.f), (float)cells);
  const int i = min((int)x, cells - 1);
  const float a = __ldg(t + i), b = __ldg(t + i + 1);
  return fmaf(x - (float)i, b - a, a);
}
__device__ __forceinline__ float cascade_cos_theta(const DevTables& T, float c0, float u) {
  const float gl = casc_lerp(T.casc, T.casc_nf, (-1.f - c0 - T.casc_vmin) * T.casc_inv_dv);
  const float gh = casc_lerp(T.casc, T.casc_nf, (1.f - c0 - T.casc_vmin) * T.casc_inv_dv);
  const float v = casc_lerp(T.casc + T.casc_nf + 1, T.casc_ni, (fmaf(u, gh - gl, gl) - T.casc_gmin) * T.casc_inv_dg);
  return fminf(fmaxf(v + c0, -1.f), 1.f);
}

// cos(theta) of Henyey-Greenstein scattering (src/photon_prop_cuda.jl:31-38)
// with the launch constants of g folded: 1 - g + 2g u = 1 + g(2u - 1).  The
// reference clamps the result to [-1, 1]; for u in (0, 1) the formula leaves
// that interval by at most a rounding, which sin_from_cos absorbs (it clamps
// 1 - c^2 at 0) and the rotation's renormalisation removes, so the clamp's
// two min/max instructions (on the busiest pipe, the integer/compare ALU)
// are left out of the step.
struct HG {
  float two_g, one_m_g, a, one_p_g2, inv_2g;
  int iso;
};
// g == 0 (isotropic, where the formula divides by zero) is a select rather
// than a branch: the formula then gives 0 (inv_2g is 0), which is dropped.
__device__ __forceinline__ float hg_costheta(const HG& h, float u) {
  const float t = h.a * rcp(fmaf(h.two_g, u, h.one_m_g));
  const float c = fmaf(-t, t, h.one_p_g2) * h.inv_2g;
  return h.iso ? fmaf(2.f, u, -1.f) : c;
}

// Rotation that takes e_z to the unit vector o, applied to n (the Rodrigues
// form of rotate_to_axis, src/photon_prop_cuda.jl:171-219), written without
// sin(theta): the (1 - cos)/sin^2 factor is 1/(1 + o_z) on the upper
// hemisphere and (1 - o_z)/(o_x^2 + o_y^2) on the lower one, both well
// conditioned in FP32; o = -e_z maps n to (n_x, -n_y, -n_z) as in the
// reference.  One MUFU (rcp) instead of the reference's sqrt, 2 divides and
// rsqrt; the result is renormalised with one Newton step instead of rsqrt.
// kExactNegZ keeps the reference's result at o = -e_z exactly; a step's
// turn leaves it out (a photon's direction there is -e_z exactly with
// probability zero, and either sign of n_x is an equally likely azimuth),
// which takes a compare and a select off the step's critical path.
template <bool kExactNegZ = true>
__device__ __forceinline__ void rotate_to_axis(float ox, float oy, float oz, float nx, float ny,
                                               float nz, float& rx, float& ry, float& rz) {
  const float q = fmaf(ox, ny, -oy * nx);
  const float s2 = fmaf(ox, ox, oy * oy);
  const bool up = oz >= 0.f;
  const float den = up ? 1.f + oz : s2 + 1e-30f;  // finite at o = -e_z, where q = 0
  const float num = up ? 1.f : 1.f - oz;
  const float t = q * num * rcp(den);
  const float z = fmaf(nz, oz, -fmaf(ox, nx, oy * ny));
  if constexpr (kExactNegZ) {
    float x = fmaf(nx, oz, fmaf(ox, nz, -oy * t));
    const float y = fmaf(ny, oz, fmaf(oy, nz, ox * t));
    // o = -e_z exactly: the formula gives (-n_x, -n_y, -n_z), the reference (n_x, -n_y, -n_z)
    if (!up && s2 == 0.f) x = nx;
    const float f = fmaf(-0.5f, fmaf(x, x, fmaf(y, y, z * z)), 1.5f);
    rx = x * f;
    ry = y * f;
    rz = z * f;
  } else {
    // the compat-mode step's turn: the (x, y) rows and the renormalisation on
    // sm_100's packed FP32 instructions (round to nearest, so the same bits
    // as the scalar form above); the emission keeps the scalar form, which
    // the batched kernel's 64-register loop runs faster
    const float2 xy = __ffma2_rn(make_float2(nx, ny), make_float2(oz, oz),
                                 __ffma2_rn(make_float2(ox, oy), make_float2(nz, nz),
                                            __fmul2_rn(make_float2(-oy, ox), make_float2(t, t))));
    const float f = fmaf(-0.5f, fmaf(xy.x, xy.x, fmaf(xy.y, xy.y, z * z)), 1.5f);
    const float2 rxy = __fmul2_rn(xy, make_float2(f, f));
    rx = rxy.x;
    ry = rxy.y;
    rz = z * f;
  }
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
  uint32_t ctr_limit;  // (max_steps + 1) << 8: a photon whose next counter word reaches it has ended
  float t_max;
  float hist_t0;
  float inv_bin_width;
  int32_t hist_bins;
  uint32_t flags;
  HG hg;
};

// Registers of one live photon.  The position is kept relative to the
// target sphere's centre (the ray-sphere test needs nothing else; the hit
// record adds the centre back), and the path as what the step logic
// compares: in physical mode the path left before t_max, in compat mode
// (no time window) the path travelled.
struct Photon {
  float px, py, pz;   // position - sphere centre
  float dx, dy, dz;
  float path;         // physical: path left before t_max; compat: path travelled
  float neg_ln2_len;  // -ln2 * scattering length: step = lg2(u) * this
  uint32_t ctr3;      // Philox counter word of the next event: block (= steps + 1) << 8 | photon bits 32..39
  uint32_t sc0;       // the step stream (from the emission block): counter word 0
  uint32_t sc1;       // and the base added to ctr3 for counter word 1
  uint32_t id_lo;     // photon index bits 0..31 (bits 32..39 are the low byte of ctr3)
};

// The photon's index: bits 0..31 in id_lo, 32..39 in the low byte of ctr3
// (which keeps them for every block), so the index costs one register.
__device__ __forceinline__ uint64_t photon_index(const Photon& s) {
  return ((uint64_t)(s.ctr3 & 0xFFu) << 32) | s.id_lo;
}
// Sets the photon's index with its counter at block 0 (emission pending).
__device__ __forceinline__ void set_photon(Photon& s, uint64_t id) {
  s.id_lo = (uint32_t)id;
  s.ctr3 = ctr_word(id, 0u);
}

struct PairCtx {
  float r;  // sphere radius
  uint32_t seed_lo, seed_hi;
  int32_t index;
};

__device__ __forceinline__ PairCtx load_pair_ctx(const pp_pair* __restrict__ P, int index) {
  const uint2 sd = __ldg(reinterpret_cast<const uint2*>(P) + 7);  // seed
  PairCtx c;
  c.r = __ldg(reinterpret_cast<const float*>(P) + 11);  // radius
  c.seed_lo = sd.x;
  c.seed_hi = sd.y;
  c.index = index;
  return c;
}

__device__ __forceinline__ float3 pair_target(const pp_pair* __restrict__ P) {
  const float4 t = __ldg(reinterpret_cast<const float4*>(P) + 2);  // target, radius
  return make_float3(t.x, t.y, t.z);
}

// Where and how a photon is emitted, from block 0 of its stream
// (src/photon_prop_cuda.jl:52-56, 67-75, 308-316).  The emission direction
// is written as a polar angle about an axis, like a scattering: isotropic
// emission is polar angle acos(2 u1 - 1) about e_z; the Cherenkov cone (no
// reference code) is acos(1/n(wl)) about the track, from a point uniform
// along the track at time t0 + s/c.  The reference-compatible isotropic
// draw takes theta = 2 u1 - 1 radians (a reference quirk) and so carries its
// own sin(theta).
struct EmissionFrame {
  float px, py, pz, t_emit, wl;
  float ox, oy, oz;  // polar axis
  float cpol, spol;  // spol valid only if has_spol
  bool has_spol;
  bool axis_ez;  // isotropic: the axis is e_z
};

// EM selects the emitters a kernel variant samples: 0 isotropic and cone
// (a cascade pair is then emitted on the cone; the batched kernel flags it),
// kEmCascade also the cascade profile, whose table lookups would otherwise
// cost every variant registers.
enum { kEmBasic = 0, kEmCascade = 1 };

template <int MODE, int EM = kEmBasic>
__device__ __forceinline__ EmissionFrame emission_frame(const DevTables& T, const pp_pair* __restrict__ P,
                                                        const Draw3& d) {
  const float4 pt = __ldg(reinterpret_cast<const float4*>(P));      // pos, t0
  const float4 dl = __ldg(reinterpret_cast<const float4*>(P) + 1);  // dir, track_len
  const int emitter = __ldg(reinterpret_cast<const int*>(P) + 16);
  EmissionFrame f;
  f.wl = draw_wavelength(T, d.u0);
  f.px = pt.x;
  f.py = pt.y;
  f.pz = pt.z;
  f.t_emit = pt.w;
  f.has_spol = false;
  f.spol = 0.f;
  f.axis_ez = emitter == PP_EMITTER_ISOTROPIC;
  if (emitter == PP_EMITTER_ISOTROPIC) {
    f.ox = 0.f;
    f.oy = 0.f;
    f.oz = 1.f;
    if (MODE == kCompat) {
      const float th = fmaf(2.f, d.u1, -1.f);
      f.cpol = cos_a(th);
      f.spol = sin_a(th);
      f.has_spol = true;
    } else {
      f.cpol = fmaf(2.f, d.u1, -1.f);
    }
  } else {  // Cherenkov cone (a track), or the cascade profile (a point)
    f.ox = dl.x;
    f.oy = dl.y;
    f.oz = dl.z;
    const float c0 = rcp(phase_index(T, rcp(f.wl)));
    f.cpol = c0;
    float s = d.u1 * dl.w;
    if (EM == kEmCascade && emitter == PP_EMITTER_CASCADE) {
      f.cpol = cascade_cos_theta(T, c0, d.u1);
      s = 0.f;
    }
    f.px = fmaf(s, f.ox, f.px);
    f.py = fmaf(s, f.oy, f.py);
    f.pz = fmaf(s, f.oz, f.pz);
    f.t_emit = fmaf(s, 1.f / kCVac, f.t_emit);
  }
  return f;
}

// Unit vector at polar cos cpol (sin spol) and azimuth 2 pi u about the axis o
// (update_direction, src/photon_prop_cuda.jl:223-241).  The azimuth is
// evaluated as 2 pi u - pi in [-pi, pi) and the sine/cosine negated.
template <bool kExactNegZ = true>
__device__ __forceinline__ void polar_direction(float ox, float oy, float oz, float cpol, float spol, float u,
                                                float& rx, float& ry, float& rz) {
  const float ph = fmaf(kTwoPi, u, -kPi);
  const float nx = -cos_a(ph) * spol, ny = -sin_a(ph) * spol;
  rotate_to_axis<kExactNegZ>(ox, oy, oz, nx, ny, cpol, rx, ry, rz);
}

__device__ __forceinline__ float sin_from_cos(float c) { return sqrt_a(fmaxf(0.f, fmaf(-c, c, 1.f))); }

// Physical-mode scattering turn: the new direction at polar cos cpol (sin
// spol) and azimuth 2 pi u about the old direction (ux, uy, uz), in the frame
// whose first axis is the old direction's meridian (the frame of the
// Monte-Carlo codes for light in turbid media, e.g. Wang, Jacques and Zheng,
// Comput. Methods Programs Biomed. 47 (1995) 131):
//   x' = (ux uz a - uy b) / s + ux c,  y' = (uy uz a + ux b) / s + uy c,
//   z' = -a s + uz c,  with s = sqrt(ux^2 + uy^2), (a, b, c) the local vector.
// The azimuth is uniform, so the choice of frame about the old direction
// does not change the physics; this one takes 14 FP32 operations and one
// rsqrt against the Rodrigues form's 22 and an rcp, and needs no branch
// between hemispheres (s = 0 exactly, a direction of exactly +-e_z, does not
// arise from these draws).  No renormalisation: |r|^2 = (a^2 + c^2) |u|^2 + b^2,
// so a norm error of the old direction enters damped by a^2 + c^2 <= 1 and
// the FP32 error stays bounded at a few times one step's rounding instead of
// accumulating over a photon's steps.
__device__ __forceinline__ void scatter_turn(float ux, float uy, float uz, float cpol, float spol, float u,
                                             float& rx, float& ry, float& rz) {
  const float ph = fmaf(kTwoPi, u, -kPi);
  const float2 ab = __fmul2_rn(make_float2(-cos_a(ph), -sin_a(ph)), make_float2(spol, spol));
  const float a = ab.x, b = ab.y;
  const float s2 = fmaf(ux, ux, uy * uy);
  const float rs = rsqrt_a(s2);
  const float p = uz * a;
  const float X = fmaf(ux, p, -uy * b);
  const float Y = fmaf(uy, p, ux * b);
  const float2 rxy = __ffma2_rn(make_float2(X, Y), make_float2(rs, rs),
                                __fmul2_rn(make_float2(ux, uy), make_float2(cpol, cpol)));
  rx = rxy.x;
  ry = rxy.y;
  rz = fmaf(-a, s2 * rs, uz * cpol);
}

// Emission direction of a frame: the isotropic axis is e_z, about which the
// polar vector needs no rotation; the cone axis is the track.
__device__ __forceinline__ void emission_direction(const EmissionFrame& f, float u, float& rx, float& ry,
                                                   float& rz) {
  const float spol = f.has_spol ? f.spol : sin_from_cos(f.cpol);
  if (f.axis_ez) {
    const float ph = fmaf(kTwoPi, u, -kPi);
    rx = -cos_a(ph) * spol;
    ry = -sin_a(ph) * spol;
    rz = f.cpol;
  } else {
    polar_direction(f.ox, f.oy, f.oz, f.cpol, spol, u, rx, ry, rz);
  }
}

// Path a photon emitted in frame f can travel before t_max at the group
// velocity c / n_g(wl): the emission and the hit record evaluate this one
// expression, so the hit's path travelled is this minus the path left.
__device__ __forceinline__ float path_at_tmax(const DevTables& T, const RunParams& R, const EmissionFrame& f) {
  return (R.t_max - f.t_emit) * kCVac * rcp(group_index(T, rcp(f.wl)));
}

// Emission of photon photon_index(s) (its emission block): position, direction, the
// per-wavelength constants and the step stream; afterwards the next event
// is step 0 (step block 1).
template <int MODE, int EM = kEmBasic>
__device__ __forceinline__ void emit_event(const DevTables& T, const RunParams& R, const pp_pair* __restrict__ P,
                                           const PairCtx& c, Photon& s) {
  const uint64_t id = photon_index(s);
  const uint4 w = emission_block(c.seed_lo, c.seed_hi, id);
  const Draw3 d = emission_uniforms(w);
  const EmissionFrame f = emission_frame<MODE, EM>(T, P, d);
  const float3 tg = pair_target(P);
  s.px = f.px - tg.x;
  s.py = f.py - tg.y;
  s.pz = f.pz - tg.z;
  s.path = (MODE == kPhysical) ? path_at_tmax(T, R, f) : 0.f;
  s.neg_ln2_len = -kLn2 * scattering_length(T, f.wl);
  emission_direction(f, d.u2, s.dx, s.dy, s.dz);
  s.sc0 = w.w;
  s.sc1 = step_base(w);
  s.ctr3 = ctr_word(id, 1u);
}

// Step k (block k + 1 of the photon's Philox2x32 stream) of
// src/photon_prop_cuda.jl:320-376: step length,
// ray-sphere test, move, Henyey-Greenstein turn.  Returns false when the
// photon ends; *hit is set when it ends on the sphere (position and path
// length then at the hit).
template <int MODE>
__device__ __forceinline__ bool step_event(const RunParams& R, const PairCtx& c, Photon& s, bool& hit) {
  uint32_t w0 = s.sc0, w1 = s.sc1 + s.ctr3;
  philox2x32_10(w0, w1, kStepKey);
  const Draw3 d = step_uniforms(w0, w1);
  const float step = lg2(d.u0) * s.neg_ln2_len;
  const float ex = s.px, ey = s.py, ez = s.pz;  // photon - sphere centre
  const float a = fmaf(s.dz, ez, fmaf(s.dy, ey, s.dx * ex));
  // b = a^2 - |e|^2 + r^2 (src/photon_prop_cuda.jl:340) evaluated as r^2 - |e - a d|^2:
  // the same number, but without cancelling two large squares, which in FP32
  // costs millimetres at grazing incidence on a sphere tens of metres away
  // (x, y) pairs on sm_100's packed FP32 instructions (round to nearest: the
  // scalar results bit for bit, in half the issue slots)
  const float2 qxy = __ffma2_rn(make_float2(-a, -a), make_float2(s.dx, s.dy), make_float2(ex, ey));
  const float qx = qxy.x, qy = qxy.y, qz = fmaf(-a, s.dz, ez);
  const float q = fmaf(qz, qz, fmaf(qy, qy, qx * qx));
  const float b = fmaf(c.r, c.r, -q);
  const float pp = fmaf(a, a, q);  // |e|^2
  // branch-free decisions: the line meets the sphere (b >= 0) at dd ahead
  // (b < 0 makes dd NaN, which no decision reads: line is false)
  const float dd = -a - sqrt_a(b);
  const bool line = b >= 0.f;
  const bool geo = line && dd > 0.f && dd < step;  // reaches the sphere within this step
  bool alive, move;
  if (MODE == kCompat) {
    hit = geo;
    move = !line;  // the line meets the sphere outside this step: no move (reference)
    alive = !geo;
  } else {
    hit = geo && dd <= s.path;  // arrives inside the time window
    // A photon farther from the sphere than the path it has left before t_max
    // can never arrive in time (any path to the sphere is at least the straight
    // distance): it ends now.  Exact, with a margin for FP32 rounding; it
    // spares the steps of photons drifting away from their target.
    const float reach = fmaf(s.path, 1.0001f, c.r + 0.05f);
    move = !geo && step <= s.path && pp <= reach * reach;
    alive = move;
  }
  const float len = hit ? dd : (move ? step : 0.f);
  const float2 pxy = __ffma2_rn(make_float2(len, len), make_float2(s.dx, s.dy), make_float2(s.px, s.py));
  s.px = pxy.x;
  s.py = pxy.y;
  s.pz = fmaf(len, s.dz, s.pz);
  s.path += (MODE == kPhysical) ? -len : len;
  const float cpol = hg_costheta(R.hg, d.u1);
  float rx, ry, rz;
  if (MODE == kPhysical) {
    scatter_turn(s.dx, s.dy, s.dz, cpol, sin_from_cos(cpol), d.u2, rx, ry, rz);
  } else {
    polar_direction<false>(s.dx, s.dy, s.dz, cpol, sin_from_cos(cpol), d.u2, rx, ry, rz);
  }
  s.dx = move ? rx : s.dx;
  s.dy = move ? ry : s.dy;
  s.dz = move ? rz : s.dz;
  s.ctr3 += 1u << 8;
  return alive && s.ctr3 < R.ctr_limit;  // at most max_steps steps
}

// Emission (block 0) or step event of one photon.
template <int MODE, int EM = kEmBasic>
__device__ __forceinline__ bool photon_event(const DevTables& T, const RunParams& R, const pp_pair* __restrict__ P,
                                             const PairCtx& c, Photon& s, bool& hit) {
  if (s.ctr3 < (1u << 8)) {
    emit_event<MODE, EM>(T, R, P, c, s);
    return true;
  }
  return step_event<MODE>(R, c, s, hit);
}

// Everything a hit record needs (src/photon_prop_cuda.jl:622,634-641); the
// emission is replayed from block 0 with the same arithmetic as its event.
struct HitValues {
  float time, weight, wl;
  float d0x, d0y, d0z;
  float px, py, pz;  // hit position (absolute)
  float dist;        // path travelled
};

template <int MODE, int EM = kEmBasic>
__device__ __forceinline__ HitValues hit_values(const DevTables& T, const RunParams& R, const pp_pair* __restrict__ P,
                                                const PairCtx& c, const Photon& s) {
  const Draw3 d = emission_uniforms(emission_block(c.seed_lo, c.seed_hi, photon_index(s)));
  const EmissionFrame f = emission_frame<MODE, EM>(T, P, d);
  HitValues h;
  h.wl = f.wl;
  emission_direction(f, d.u2, h.d0x, h.d0y, h.d0z);
  const float3 tg = pair_target(P);
  h.px = s.px + tg.x;
  h.py = s.py + tg.y;
  h.pz = s.pz + tg.z;
  h.dist = (MODE == kPhysical) ? path_at_tmax(T, R, f) - s.path : s.path;
  const float x = 1.f / f.wl;
  if (MODE == kCompat) {
    h.time = h.dist * phase_index(T, x) / kCVac;  // phase velocity (reference)
  } else {
    h.time = f.t_emit + h.dist * group_index(T, x) / kCVac;
  }
  float w = expf(-h.dist / interp_sorted(f.wl, T.abs_wl, T.abs_len, T.n_abs));
  if ((R.flags & PP_OPT_PMT_WEIGHT) && T.n_pmt > 0) w *= interp_sorted(f.wl, T.pmt_wl, T.pmt_acc, T.n_pmt);
  h.weight = w;
  return h;
}

// One hit's histogram bin (FP64 atomic).
__device__ __forceinline__ void histogram_hit(const RunParams& R, const HitValues& h, int stats_row) {
  if (R.hist_bins > 0) {
    const float fb = floorf((h.time - R.hist_t0) * R.inv_bin_width);
    if (fb >= 0.f && fb < (float)R.hist_bins)
      atomicAdd(R.hist + (int64_t)stats_row * R.hist_bins + (int)fb, (double)h.weight);
  }
}

// Writes hit record idx (or flags the overflow).
__device__ __forceinline__ void write_hit(const RunParams& R, const PairCtx& c, const Photon& s, const HitValues& h,
                                          unsigned long long idx) {
  if (R.flags & PP_OPT_NO_HITS) return;
  if (idx < R.hit_cap) {
    if (R.flags & PP_OPT_COMPACT_HITS) {
      float4* dst = reinterpret_cast<float4*>(reinterpret_cast<pp_hit32*>(R.hits) + idx);
      dst[0] = make_float4(h.px, h.py, h.pz, h.time);
      dst[1] = make_float4(h.weight, h.wl, __uint_as_float(s.id_lo),
                           __uint_as_float((uint32_t)c.index + R.pair_base));
    } else {
      float4* dst = reinterpret_cast<float4*>(R.hits + idx);
      dst[0] = make_float4(h.px, h.py, h.pz, h.time);
      dst[1] = make_float4(h.d0x, h.d0y, h.d0z, h.weight);
      dst[2] = make_float4(s.dx, s.dy, s.dz, h.wl);
      dst[3] = make_float4(h.dist, __uint_as_float((uint32_t)c.index + R.pair_base),
                           __uint_as_float(s.id_lo), __uint_as_float(s.ctr3 & 0xFFu));
    }
  } else {
    atomicOr(R.counters + 2, 1ull);
  }
}

// Per-pair FP64 accumulation, histogram and warp-aggregated hit write-back,
// called by the lanes that hit (any convergence).
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
  histogram_hit(R, h, stats_row);
  // warp-aggregated slot reservation among the lanes that hit in this step
  const unsigned m = __activemask();
  const int leader = __ffs(m) - 1;
  const unsigned lane = threadIdx.x & 31u;
  const unsigned rank = __popc(m & ((1u << lane) - 1u));
  unsigned long long base = 0;
  if ((int)lane == leader) base = atomicAdd(R.counters + 0, (unsigned long long)__popc(m));
  base = __shfl_sync(m, base, leader);
  write_hit(R, c, s, h, base + rank);
}

// A warp's running sums for the pair of its current photon chunk (shared
// memory): hits of that pair add here and the warp adds the sums to the
// pair's FP64 statistics when it moves to another pair, so a hit-dense pair
// does not serialise every hit on its six global addresses.
struct WarpStats {
  double v[6];
  int32_t pair;
  int32_t pad;
};

__device__ __forceinline__ void flush_warp_stats(double* stats, WarpStats* ws) {
  if (ws->pair >= 0 && ws->v[0] != 0.0) {
    double* st = stats + (int64_t)ws->pair * PP_STATS;
#pragma unroll
    for (int k = 0; k < 6; ++k) atomicAdd(st + k, ws->v[k]);
  }
#pragma unroll
  for (int k = 0; k < 6; ++k) ws->v[k] = 0.0;
}

// record_hit with the warp's statistics cache: lanes whose pair is the
// cached one add to it (shared-memory atomics), others to the global sums.
__device__ __forceinline__ void record_hit_cached(const RunParams& R, WarpStats* ws, const PairCtx& c,
                                                  const Photon& s, const HitValues& h) {
  const double w = (double)h.weight;
  const double t = (double)h.time;
  double* st = c.index == ws->pair ? ws->v : R.stats + (int64_t)c.index * PP_STATS;
  atomicAdd(st + 0, 1.0);
  atomicAdd(st + 1, w);
  atomicAdd(st + 2, w * w);
  atomicAdd(st + 3, w * t);
  atomicAdd(st + 4, w * t * t);
  atomicAdd(st + 5, w * (double)logf(h.time));
  histogram_hit(R, h, c.index);
  const unsigned m = __activemask();
  const int leader = __ffs(m) - 1;
  const unsigned lane = threadIdx.x & 31u;
  unsigned long long base = 0;
  if ((int)lane == leader) base = atomicAdd(R.counters + 0, (unsigned long long)__popc(m));
  base = __shfl_sync(m, base, leader);
  write_hit(R, c, s, h, base + __popc(m & ((1u << lane) - 1u)));
}

}  // namespace ppd
