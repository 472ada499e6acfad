/*
 * FP64 CPU oracle for the photon-propagation hot path of PhotonProp.jl.
 * TEST INFRASTRUCTURE ONLY (see pp_oracle.h): the checker, never the product.
 *
 * Each function cites the reference file:line it restates.  Where the
 * reference has no code (cone emission, group-velocity time, time window) the
 * physical-mode definition below is the one the CUDA kernels implement:
 *   - isotropic emission draws cos(theta) uniformly in [-1, 1];
 *   - Cherenkov-cone emission: a point uniform along the track, emission angle
 *     acos(1/n(lambda)) around the track axis, emission time t0 + s/c;
 *   - arrival time t = t_emit + dist * n_group(lambda) / c;
 *   - a scattering turns the direction in the frame of its meridian
 *     (orc_scatter_turn; the reference's rotate_to_axis frame in compat mode);
 *   - a photon ends when its next position would lie beyond the time window
 *     t_max, when it hits the sphere, or after max_steps steps.
 * Random numbers (Salmon et al., SC'11).  Emission: Philox4x32-10 under the
 * fixed key (0x243F6A88, 0x85A308D3) with counter (seed lo, seed hi,
 * photon lo, photon hi) for a photon index below 2^40; its words w0..w2 give
 * the emission draws (wavelength, polar angle or track position, azimuth) as
 * 23-bit uniforms.  Steps: the photon's own Philox2x32-10 stream under the
 * fixed step key 0x13198A2E, with counter (w3, base + (photon hi |
 * (k + 1) << 8)) for step k, where base packs the low 9 bits of w0, w1, w2
 * into 27 bits; its 64 output bits give three 21-bit uniforms (step length,
 * HG cos(theta), azimuth).
 */
#include "pp_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_C_VAC 0.299792458
#define ORC_KEY0 0x243F6A88u /* fixed Philox key */
#define ORC_KEY1 0x85A308D3u
#define ORC_STEP_KEY 0x13198A2Eu /* fixed Philox2x32 key of the step blocks */
#define ORC_TWO_PI 6.283185307179586

/* Philox4x32-10, Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
 * easy as 1, 2, 3", SC'11: multipliers 0xD2511F53/0xCD9E8D57, Weyl key
 * increments 0x9E3779B9/0xBB67AE85. */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
  uint32_t k0 = key[0], k1 = key[1];
  for (int r = 0; r < 10; ++r) {
    if (r) {
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
    uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
    uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
    c0 = n0;
    c1 = (uint32_t)p1;
    c2 = n2;
    c3 = (uint32_t)p0;
  }
  out[0] = c0;
  out[1] = c1;
  out[2] = c2;
  out[3] = c3;
}

/* Philox2x32-10 (same paper): multiplier 0xD256D193, Weyl key increment
 * 0x9E3779B9. */
void orc_philox2x32_10(const uint32_t ctr[2], uint32_t key, uint32_t out[2]) {
  uint32_t c0 = ctr[0], c1 = ctr[1], k = key;
  for (int r = 0; r < 10; ++r) {
    if (r) k += 0x9E3779B9u;
    uint64_t p = (uint64_t)0xD256D193u * c0;
    uint32_t n0 = (uint32_t)(p >> 32) ^ c1 ^ k;
    c0 = n0;
    c1 = (uint32_t)p;
  }
  out[0] = c0;
  out[1] = c1;
}

/* The three 21-bit uniforms of a step from the 64 bits (w0, w1) of its
 * Philox2x32 block: bits 63..43, 42..22 and 21..1 of w0:w1, each as
 * (k + 1/2) * 2^-21 (exact in FP32). */
void orc_step_uniforms(const uint32_t w[2], double u[3]) {
  const uint64_t b = ((uint64_t)w[0] << 32) | w[1];
  for (int i = 0; i < 3; ++i) u[i] = ((double)((b >> (43 - 21 * i)) & 0x1FFFFFu) + 0.5) * (1.0 / 2097152.0);
}

/* The step stream of a photon from its emission block: counter word 0 is
 * w3, counter word 1 a base (the low 9 bits of w0, w1 and w2) plus the
 * photon's top index bits and block number. */
void orc_step_stream(const uint32_t w[4], uint32_t* word0, uint32_t* base) {
  *word0 = w[3];
  *base = (w[0] & 0x1FFu) | ((w[1] & 0x1FFu) << 9) | ((w[2] & 0x1FFu) << 18);
}

/* 23-bit uniform in the open interval (0, 1): ((w >> 9) + 1/2) * 2^-23.
 * The value is exactly representable in FP32, so the FP32 kernels see the
 * same number. */
double orc_uniform(uint32_t w) { return ((double)(w >> 9) + 0.5) * (1.0 / 8388608.0); }

/* cuda_hg_scattering_func, src/photon_prop_cuda.jl:31-38 (g == 0 falls back to
 * isotropic scattering, where the reference formula divides by zero). */
double orc_hg_costheta(double g, double u) {
  if (g == 0.0) return 2.0 * u - 1.0;
  double t = fma(-g, g, 1.0) / fma(g, fma(2.0, u, -1.0), 1.0);
  double c = 1.0 / (2.0 * g) * (fma(g, g, 1.0) - t * t);
  if (c < -1.0) c = -1.0;
  if (c > 1.0) c = 1.0;
  return c;
}

/* rotate_to_axis, src/photon_prop_cuda.jl:171-219: rotate new_dir by the
 * rotation that takes e_z to old_dir (Rodrigues), then renormalise. */
void orc_rotate_to_axis(const double o[3], const double n[3], double out[3]) {
  if (fabs(o[2]) == 1.0) {
    double s = o[2] > 0 ? 1.0 : -1.0;
    out[0] = n[0];
    out[1] = s * n[1];
    out[2] = s * n[2];
    return;
  }
  double st = sqrt(fma(-o[2], o[2], 1.0));
  double ax1 = -o[1] / st, ax2 = o[0] / st;
  double kappa = (ax1 * n[0] + ax2 * n[1]) * (1.0 - o[2]);
  double nd3s = n[2] * st;
  double x = fma(n[0], o[2], fma(ax2, nd3s, ax1 * kappa));
  double y = fma(n[1], o[2], fma(-ax1, nd3s, ax2 * kappa));
  double z = fma(n[2], o[2], st * fma(ax1, n[1], -ax2 * n[0]));
  double r = 1.0 / sqrt(x * x + y * y + z * z);
  out[0] = x * r;
  out[1] = y * r;
  out[2] = z * r;
}

/* Physical-mode scattering turn (no reference code: the reference turns with
 * rotate_to_axis in both modes): the local vector n = (a, b, c) placed in
 * the frame whose first axis is the old direction u's meridian,
 *   x = (ux uz a - uy b) / s + ux c, y = (uy uz a + ux b) / s + uy c,
 *   z = -a s + uz c, s = sqrt(ux^2 + uy^2).
 * The azimuth is uniform, so this is the same scattering distribution as the
 * Rodrigues frame; the CUDA kernels use this frame in physical mode. */
void orc_scatter_turn(const double u[3], const double n[3], double out[3]) {
  const double s2 = u[0] * u[0] + u[1] * u[1];
  const double rs = 1.0 / sqrt(s2);
  const double p = u[2] * n[0];
  const double X = u[0] * p - u[1] * n[1];
  const double Y = u[1] * p + u[0] * n[1];
  out[0] = X * rs + u[0] * n[2];
  out[1] = Y * rs + u[1] * n[2];
  out[2] = -n[0] * s2 * rs + u[2] * n[2];
}

/* update_position, src/photon_prop_cuda.jl:255-259. */
void orc_update_position(const double p[3], const double d[3], double step, double out[3]) {
  for (int j = 0; j < 3; ++j) out[j] = fma(step, d[j], p[j]);
}

/* fast_linear_interp(x, xs, ys), src/utils.jl:10-34 (lower index clamped). */
double orc_interp_sorted(double x, const double* xs, const double* ys, int n) {
  if (x < xs[0]) x = xs[0];
  if (x > xs[n - 1]) x = xs[n - 1];
  int hi = 0;
  while (hi < n && xs[hi] < x) ++hi; /* searchsortedfirst */
  if (hi < 1) hi = 1;
  if (hi > n - 1) hi = n - 1;
  int lo = hi - 1;
  double along = (x - xs[lo]) / (xs[hi] - xs[lo]);
  return ys[lo] + (ys[hi] - ys[lo]) * along;
}

/* fast_linear_interp(x, knots, lower, upper), src/utils.jl:37-60. */
double orc_interp_equidistant(double x, const double* k, int n, double lo, double hi) {
  if (x < lo) x = lo;
  if (x > hi) x = hi;
  double step = (hi - lo) / (double)(n - 1);
  double along = (x - lo) / step;
  double fl = floor(along);
  int i = (int)fl;
  if (i >= n - 1) return k[n - 1];
  double frac = along - fl;
  return k[i] + (k[i + 1] - k[i]) * frac;
}

/* get_refractive_index_fry, src/medium.jl:125-158. */
double orc_refractive_index(const orc_tables* t, double wl) {
  double x = 1.0 / wl;
  return t->a01 + x * (t->a2 + x * (t->a3 + x * t->a4));
}

/* n - lambda dn/dlambda of the same polynomial (no reference counterpart). */
double orc_group_index(const orc_tables* t, double wl) {
  double x = 1.0 / wl;
  return t->a01 + x * (2.0 * t->a2 + x * (3.0 * t->a3 + x * 4.0 * t->a4));
}

/* get_sca_len_part_conc, src/medium.jl:201-214. */
double orc_scattering_length(const orc_tables* t, double wl) {
  double x = 550.0 / wl;
  double c = 0.0017 * pow(x, 4.3) + 1.34 * t->c_small * pow(x, 1.7) + 0.312 * t->c_large * pow(x, 0.3);
  return 1.0 / c;
}

typedef struct {
  orc_hit* h;
  int64_t n, cap;
} hitbuf;

static void hb_push(hitbuf* b, const orc_hit* h) {
  if (b->n == b->cap) {
    b->cap = b->cap ? 2 * b->cap : 256;
    b->h = (orc_hit*)realloc(b->h, (size_t)b->cap * sizeof(orc_hit));
  }
  b->h[b->n++] = *h;
}

/* Emission block of a photon: its three uniforms and the step stream. */
static void emission_block(uint64_t seed, int64_t photon, double u[3], uint32_t* sc0, uint32_t* sc1) {
  uint32_t key[2] = {ORC_KEY0, ORC_KEY1};
  uint32_t ctr[4] = {(uint32_t)seed, (uint32_t)(seed >> 32), (uint32_t)(uint64_t)photon,
                     (uint32_t)((uint64_t)photon >> 32)};
  uint32_t w[4];
  orc_philox4x32_10(ctr, key, w);
  for (int i = 0; i < 3; ++i) u[i] = orc_uniform(w[i]);
  orc_step_stream(w, sc0, sc1);
}

/* Uniforms of step k of a photon. */
static void step_block(uint32_t sc0, uint32_t sc1, int64_t photon, int k, double u[3]) {
  uint32_t ctr[2] = {sc0, sc1 + ((uint32_t)((uint64_t)photon >> 32) | ((uint32_t)(k + 1) << 8))};
  uint32_t w[2];
  orc_philox2x32_10(ctr, ORC_STEP_KEY, w);
  orc_step_uniforms(w, u);
}

/* cos(theta) of the cascade emitter: inverse CDF of the EM-cascade profile
 * cherenkov_ang_dist (src/emission.jl:32-44) at 1/n = c0 through the
 * tables (linear interpolation). */
static double lerp_tab(const double* t, int cells, double x) {
  if (x < 0.0) x = 0.0;
  if (x > cells) x = cells;
  int i = (int)x;
  if (i > cells - 1) i = cells - 1;
  return t[i] + (x - i) * (t[i + 1] - t[i]);
}

static double cascade_cos_theta(const orc_tables* T, double c0, double u) {
  const double gl = lerp_tab(T->casc_fwd, T->casc_nf, (-1.0 - c0 - T->casc_vmin) / T->casc_dv);
  const double gh = lerp_tab(T->casc_fwd, T->casc_nf, (1.0 - c0 - T->casc_vmin) / T->casc_dv);
  const double v = lerp_tab(T->casc_inv, T->casc_ni, (gl + u * (gh - gl) - T->casc_gmin) / T->casc_dg);
  const double x = v + c0;
  return x < -1.0 ? -1.0 : (x > 1.0 ? 1.0 : x);
}

/* One photon: the per-photon body of cuda_propagate_photons!,
 * src/photon_prop_cuda.jl:301-380, plus the host finish of
 * propagate_distance (:622, :634-638) done per hit. */
static int simulate_photon(const orc_tables* T, const orc_pair* P, int64_t pair_idx, int64_t ph,
                           const orc_opts* O, orc_hit* out, int64_t* steps) {
  const int compat = (O->mode == 0);
  double u[3];
  uint32_t sc0, sc1;
  emission_block(P->seed, ph, u, &sc0, &sc1);
  /* initialize_wavelength, src/photon_prop_cuda.jl:73-75 */
  double wl = (T->n_knots == 1) ? T->knots[0] : orc_interp_equidistant(u[0], T->knots, T->n_knots, 0.0, 1.0);
  double phi = ORC_TWO_PI * u[2]; /* uniform(0, 2pi), :54 */
  double sp = sin(phi), cp = cos(phi);
  double dir[3], pos[3], t_emit = P->t0;
  if (P->emitter == 0) {
    double st, ct;
    if (compat) { /* theta = uniform(-1, 1) radians (reference quirk), :52-56 */
      double th = -1.0 + u[1] * 2.0;
      st = sin(th);
      ct = cos(th);
    } else {
      ct = -1.0 + u[1] * 2.0;
      st = sqrt(fmax(0.0, fma(-ct, ct, 1.0)));
    }
    dir[0] = cp * st; /* sph_to_cart, :41-50 */
    dir[1] = sp * st;
    dir[2] = ct;
    pos[0] = P->pos[0];
    pos[1] = P->pos[1];
    pos[2] = P->pos[2];
  } else if (P->emitter == 2) {
    double ct = cascade_cos_theta(T, 1.0 / orc_refractive_index(T, wl), u[1]);
    double st = sqrt(fmax(0.0, fma(-ct, ct, 1.0)));
    double loc[3] = {cp * st, sp * st, ct};
    orc_rotate_to_axis(P->dir, loc, dir);
    for (int j = 0; j < 3; ++j) pos[j] = P->pos[j];
  } else {
    double ct = 1.0 / orc_refractive_index(T, wl);
    double st = sqrt(fmax(0.0, fma(-ct, ct, 1.0)));
    double loc[3] = {cp * st, sp * st, ct};
    orc_rotate_to_axis(P->dir, loc, dir);
    double s = u[1] * P->track_len;
    for (int j = 0; j < 3; ++j) pos[j] = P->pos[j] + s * P->dir[j];
    t_emit = P->t0 + s / ORC_C_VAC;
  }
  double dir0[3] = {dir[0], dir[1], dir[2]};
  double sca_len = orc_scattering_length(T, wl); /* :316 */
  double max_dist = compat ? INFINITY : (O->t_max - t_emit) * ORC_C_VAC / orc_group_index(T, wl);
  double dist = 0.0;
  double rsq = P->radius * P->radius;
  for (int k = 0; k < O->max_steps; ++k) {
    ++*steps;
    step_block(sc0, sc1, ph, k, u);
    double step = -log(u[0]) * sca_len; /* :322-323 */
    double a = 0.0, pp = 0.0;           /* :330-337 */
    for (int j = 0; j < 3; ++j) {
      double dp = pos[j] - P->target[j];
      a += dir[j] * dp;
      pp += dp * dp;
    }
    double b = fma(a, a, -pp + rsq); /* :340 */
    int hit = 0;
    double d = 0.0;
    if (b >= 0.0) {
      d = -a - sqrt(b); /* :348 */
      if (d > 0.0 && d < step) {
        if (!compat && dist + d > max_dist) return 0; /* arrives after the window */
        hit = 1;
      } else if (compat) {
        continue; /* line meets the sphere outside this step: no move (reference, :345-357) */
      }
    }
    if (hit) {
      double np[3];
      orc_update_position(pos, dir, d, np);
      dist += d;
      double n_idx = compat ? orc_refractive_index(T, wl) : orc_group_index(T, wl);
      double t = (compat ? 0.0 : t_emit) + dist * n_idx / ORC_C_VAC; /* :634-638 */
      double w = exp(-dist / orc_interp_sorted(wl, T->abs_wl, T->abs_len, T->n_abs)); /* :622 */
      if (O->flags & 1u) w *= orc_interp_sorted(wl, T->pmt_wl, T->pmt_acc, T->n_pmt);
      for (int j = 0; j < 3; ++j) {
        out->pos[j] = np[j];
        out->dir0[j] = dir0[j];
        out->dir[j] = dir[j];
      }
      out->time = t;
      out->weight = w;
      out->wavelength = wl;
      out->dist = dist;
      out->pair = pair_idx;
      out->photon = ph;
      out->step = k;
      out->pad = 0;
      return 1;
    }
    if (!compat && dist + step > max_dist) return 0;
    double np[3];
    orc_update_position(pos, dir, step, np); /* :358 */
    pos[0] = np[0];
    pos[1] = np[1];
    pos[2] = np[2];
    dist += step;
    /* update_direction, :223-241 */
    double cs = orc_hg_costheta(O->g, u[1]);
    double ss = sqrt(fmax(0.0, fma(-cs, cs, 1.0)));
    double ph2 = ORC_TWO_PI * u[2];
    double loc[3] = {cos(ph2) * ss, sin(ph2) * ss, cs};
    double nd[3];
    if (compat)
      orc_rotate_to_axis(dir, loc, nd);
    else
      orc_scatter_turn(dir, loc, nd);
    dir[0] = nd[0];
    dir[1] = nd[1];
    dir[2] = nd[2];
  }
  return 0;
}

static int cmp_hit(const void* a, const void* b) {
  const orc_hit* x = (const orc_hit*)a;
  const orc_hit* y = (const orc_hit*)b;
  if (x->pair != y->pair) return x->pair < y->pair ? -1 : 1;
  if (x->photon != y->photon) return x->photon < y->photon ? -1 : 1;
  return 0;
}

/* Work items of the flat (pair, photon) index space: chunks of ORC_CHUNK
 * photons of one pair, so every host thread has work at any photon count. */
#define ORC_CHUNK 256

int64_t orc_propagate(const orc_tables* t, const orc_pair* pairs, int64_t n_pairs, const orc_opts* o,
                      int64_t photon_limit, orc_hit* hits, int64_t hit_cap, double* stats, double* hist,
                      int n_threads, int64_t* steps_out, int* threads_used) {
  int nt = n_threads > 0 ? n_threads : 1;
#ifdef _OPENMP
  if (n_threads <= 0) nt = omp_get_max_threads();
#endif
  hitbuf* bufs = (hitbuf*)calloc((size_t)nt, sizeof(hitbuf));
  int64_t* steps = (int64_t*)calloc((size_t)nt, sizeof(int64_t));
  /* chunk offsets: pair p owns chunks [off[p], off[p + 1]) */
  int64_t* coff = (int64_t*)malloc((size_t)(n_pairs + 1) * sizeof(int64_t));
  coff[0] = 0;
  for (int64_t p = 0; p < n_pairs; ++p) {
    int64_t n = pairs[p].n_photons;
    if (photon_limit >= 0 && n > photon_limit) n = photon_limit;
    if (n < 0) n = 0;
    coff[p + 1] = coff[p] + (n + ORC_CHUNK - 1) / ORC_CHUNK;
  }
  const int64_t n_chunks = coff[n_pairs];
  int used = 1;
#pragma omp parallel num_threads(nt)
  {
    int tid = 0;
#ifdef _OPENMP
    tid = omp_get_thread_num();
#pragma omp single
    used = omp_get_num_threads();
#endif
#pragma omp for schedule(dynamic, 1)
    for (int64_t c = 0; c < n_chunks; ++c) {
      int64_t lo = 0, hi = n_pairs - 1; /* last pair whose first chunk <= c */
      while (lo < hi) {
        const int64_t mid = (lo + hi + 1) / 2;
        if (coff[mid] <= c) lo = mid; else hi = mid - 1;
      }
      const int64_t p = lo;
      int64_t n = pairs[p].n_photons;
      if (photon_limit >= 0 && n > photon_limit) n = photon_limit;
      const int64_t b = (c - coff[p]) * ORC_CHUNK;
      const int64_t e = b + ORC_CHUNK < n ? b + ORC_CHUNK : n;
      for (int64_t ph = b; ph < e; ++ph) {
        orc_hit h;
        if (simulate_photon(t, &pairs[p], p, ph, o, &h, &steps[tid])) hb_push(&bufs[tid], &h);
      }
    }
  }
  free(coff);
  if (threads_used) *threads_used = used;
  int64_t total = 0, total_steps = 0;
  for (int i = 0; i < nt; ++i) {
    total += bufs[i].n;
    total_steps += steps[i];
  }
  orc_hit* all = (orc_hit*)malloc((size_t)(total ? total : 1) * sizeof(orc_hit));
  int64_t off = 0;
  for (int i = 0; i < nt; ++i) {
    if (bufs[i].n) memcpy(all + off, bufs[i].h, (size_t)bufs[i].n * sizeof(orc_hit));
    off += bufs[i].n;
    free(bufs[i].h);
  }
  free(bufs);
  free(steps);
  qsort(all, (size_t)total, sizeof(orc_hit), cmp_hit);
  if (stats) memset(stats, 0, (size_t)n_pairs * ORC_STATS * sizeof(double));
  if (hist && o->hist_bins > 0) memset(hist, 0, (size_t)n_pairs * (size_t)o->hist_bins * sizeof(double));
  for (int64_t i = 0; i < total; ++i) {
    const orc_hit* h = &all[i];
    if (stats) {
      double* s = stats + h->pair * ORC_STATS;
      s[0] += 1.0;
      s[1] += h->weight;
      s[2] += h->weight * h->weight;
      s[3] += h->weight * h->time;
      s[4] += h->weight * h->time * h->time;
      s[5] += h->weight * log(h->time);
    }
    if (hist && o->hist_bins > 0) {
      double f = floor((h->time - o->hist_t0) / o->hist_bin_width);
      if (f >= 0.0 && f < (double)o->hist_bins) hist[h->pair * o->hist_bins + (int64_t)f] += h->weight;
    }
    if (hits && i < hit_cap) hits[i] = *h;
  }
  for (int64_t p = 0; p < n_pairs; ++p) {
    int64_t n = pairs[p].n_photons;
    if (photon_limit >= 0 && n > photon_limit) n = photon_limit;
    if (stats) stats[p * ORC_STATS + 6] = (double)n;
    if (hist && o->hist_bins > 0 && (o->flags & 2u) && n > 0)
      for (int b = 0; b < o->hist_bins; ++b) hist[p * o->hist_bins + b] /= (double)n;
  }
  free(all);
  if (steps_out) *steps_out = total_steps;
  return total;
}

/* Replays one photon (any 64-bit index): 1 and *hit filled if it is detected. */
int orc_simulate_one(const orc_tables* t, const orc_pair* pair, int64_t pair_idx, int64_t photon,
                     const orc_opts* o, orc_hit* hit) {
  int64_t steps = 0;
  return simulate_photon(t, pair, pair_idx, photon, o, hit, &steps);
}
