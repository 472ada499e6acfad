/*
 * FP64 CPU oracle for the photon-propagation hot path of PhotonProp.jl.
 *
 * TEST INFRASTRUCTURE ONLY: a restatement of the reference kernel
 * cuda_propagate_photons! (src/photon_prop_cuda.jl:262-386) and its helpers,
 * replaying the same Philox random numbers as the CUDA kernels (a photon's
 * emission block is Philox4x32-10, its steps its own Philox2x32-10 stream).  Only
 * the tests, the smoke check and the CPU-baseline leg of bench.py load it, and
 * only as the checker.  Nothing in the product links it.
 *
 * Parity status: the helper functions are pinned by the known-answer tests of
 * src/tests/test_photon_prob.jl and both Philox forms by the Random123 known-answer
 * vectors; end-to-end hit statistics are "parity unpinned" against the
 * reference itself (the reference is Julia/CUDA.jl and cannot run here, and
 * its device RNG stream is not reproducible).
 */
#ifndef PP_ORACLE_H
#define PP_ORACLE_H
#include <stdint.h>

#define ORC_MAX_KNOTS 64
#define ORC_MAX_ABS 32
#define ORC_MAX_PMT 256

typedef struct {
  double a01, a2, a3, a4;  /* Quan-Fry: n = a01 + x(a2 + x(a3 + x a4)), x = 1/nm */
  double c_small, c_large; /* particle concentrations, ppm */
  int32_t n_knots;         /* spectrum inverse-CDF knots; 1 = monochromatic */
  int32_t n_abs;
  int32_t n_pmt;
  int32_t pad;
  double knots[ORC_MAX_KNOTS];
  double abs_wl[ORC_MAX_ABS], abs_len[ORC_MAX_ABS];
  double pmt_wl[ORC_MAX_PMT], pmt_acc[ORC_MAX_PMT];
  /* cascade emitter (emitter 2): G of the angular profile on casc_nf + 1
   * points from casc_vmin, step casc_dv; v at casc_ni + 1 levels of G from
   * casc_gmin, step casc_dg (NULL: no cascade emitter) */
  const double* casc_fwd;
  const double* casc_inv;
  double casc_vmin, casc_dv, casc_gmin, casc_dg;
  int32_t casc_nf, casc_ni;
} orc_tables;

typedef struct {
  double pos[3];
  double t0;
  double dir[3];
  double track_len;
  double target[3];
  double radius;
  int64_t n_photons;
  uint64_t seed;
  int32_t emitter; /* 0 isotropic point, 1 Cherenkov-cone line, 2 cascade-profile point */
  int32_t pad;
} orc_pair;

typedef struct {
  int32_t mode; /* 0 reference-compatible, 1 physical */
  int32_t max_steps;
  double g;
  double t_max;
  double hist_t0;
  double hist_bin_width;
  int32_t hist_bins;
  uint32_t flags; /* bit0: PMT weight, bit1: normalise histogram */
} orc_opts;

typedef struct {
  double pos[3];
  double time;
  double dir0[3];
  double weight;
  double dir[3];
  double wavelength;
  double dist;
  int64_t pair;
  int64_t photon;
  int32_t step;
  int32_t pad;
} orc_hit;

#define ORC_STATS 8

void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
void orc_philox2x32_10(const uint32_t ctr[2], uint32_t key, uint32_t out[2]);
void orc_step_uniforms(const uint32_t w[2], double u[3]);
void orc_scatter_turn(const double u[3], const double n[3], double out[3]);
void orc_step_stream(const uint32_t w[4], uint32_t* word0, uint32_t* base);
double orc_uniform(uint32_t w);
double orc_hg_costheta(double g, double u);
void orc_rotate_to_axis(const double old_dir[3], const double new_dir[3], double out[3]);
void orc_update_position(const double pos[3], const double dir[3], double step, double out[3]);
double orc_interp_sorted(double x, const double* xs, const double* ys, int n);
double orc_interp_equidistant(double x, const double* knots, int n, double lo, double hi);
double orc_refractive_index(const orc_tables* t, double wl);
double orc_group_index(const orc_tables* t, double wl);
double orc_scattering_length(const orc_tables* t, double wl);

/* Propagates min(n_photons, photon_limit) photons of every pair (photon_limit
 * < 0: all).  Hits are returned sorted by (pair, photon); stats is
 * [n_pairs x ORC_STATS], hist [n_pairs x hist_bins].  Returns the total number
 * of hits (which may exceed hit_cap; only hit_cap are copied).  The work is
 * one flat index space of 256-photon chunks over all pairs (OpenMP, dynamic
 * schedule), so all n_threads threads (0: OpenMP's default) work at any photon
 * count; *threads_used (may be NULL) receives the team size that ran. */
int64_t orc_propagate(const orc_tables* t, const orc_pair* pairs, int64_t n_pairs,
                      const orc_opts* o, int64_t photon_limit, orc_hit* hits,
                      int64_t hit_cap, double* stats, double* hist, int n_threads,
                      int64_t* steps_out, int* threads_used);

/* Replays one photon of a pair; returns 1 and fills *hit when it is detected. */
int orc_simulate_one(const orc_tables* t, const orc_pair* pair, int64_t pair_idx, int64_t photon,
                     const orc_opts* o, orc_hit* hit);

#endif
