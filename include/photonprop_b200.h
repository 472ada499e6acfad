/*
 * photonprop_b200 — B200-native (sm_100a) photon propagation for PhotonProp.jl.
 *
 * C ABI of libphotonprop_b200.so.  Plain C types only (no CUDA, no torch in
 * the signatures) so that Julia can bind every entry point with `ccall` and
 * isbits mirror structs; the Python host package binds it with ctypes.
 *
 * Conventions
 *  - Every fallible call returns pp_status; no exception crosses the ABI.
 *    pp_last_error(ctx) returns a message for the last failure on ctx.
 *  - The caller owns every host buffer it passes in; the library owns its
 *    device buffers and the device-resident physics tables of a context.
 *  - A context is bound to one device; calls on one context are serialised
 *    by an internal mutex.  *_device entry points take device pointers and a
 *    cudaStream_t (as void*) and return without synchronising.
 *  - Units: metres, nanoseconds, nanometres.
 *
 * Citations are to the reference PhotonProp.jl (file:line).
 */
#ifndef PHOTONPROP_B200_H
#define PHOTONPROP_B200_H

#include <stdint.h>

#if defined(__GNUC__)
#define PP_API __attribute__((visibility("default")))
#else
#define PP_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define PP_ABI_VERSION 1

typedef enum {
  PP_OK = 0,
  PP_ERR_ARG = 1,      /* invalid argument; the reference throws ArgumentError */
  PP_ERR_OOM = 2,      /* device or host allocation failed */
  PP_ERR_OVERFLOW = 3, /* more hits than hit_capacity: the first hit_capacity
                          are returned, *n_hits holds the true count */
  PP_ERR_TIMEOUT = 4,  /* a bounded wait ran out (serving loop) */
  PP_ERR_CUDA = 5,     /* a CUDA runtime call failed */
  PP_ERR_STATE = 6,    /* call not valid in the object's current state */
  PP_ERR_BUSY = 7      /* admission refused: no slot or memory free now */
} pp_status;

enum { PP_MODE_COMPAT = 0, PP_MODE_PHYSICAL = 1 };
/* PP_EMITTER_CASCADE: a point source with the angular profile of an EM
 * cascade about `dir`, cherenkov_ang_dist(cos theta, n(lambda))
 * (src/emission.jl:32-44), sampled by inverse CDF; physical mode only (the
 * reference propagates isotropic photons and reweights them to this profile,
 * src/modelling.jl:46-49). */
enum { PP_EMITTER_ISOTROPIC = 0, PP_EMITTER_CHERENKOV_CONE = 1, PP_EMITTER_CASCADE = 2 };
enum { PP_SPECTRUM_CHERENKOV = 0, PP_SPECTRUM_MONOCHROMATIC = 1 };
enum {
  PP_OPT_PMT_WEIGHT = 1u, /* multiply hit weights by the PMT acceptance */
  PP_OPT_NORMALIZE = 2u,  /* divide each pair's histogram by its photon count */
  PP_OPT_NO_HITS = 4u,    /* accumulate statistics only; write no hit records */
  PP_OPT_COMPACT_HITS = 8u, /* write pp_hit32 records instead of pp_hit */
  PP_OPT_CASCADE = 16u      /* the pairs may include PP_EMITTER_CASCADE: launch the kernel variant that
                               samples the cascade profile.  The host-buffer entry points set it
                               themselves; on the *_device entry points the caller sets it, and a
                               cascade pair launched without it is emitted on the Cherenkov cone
                               and sets status bit 4 (value 4) in counters[2]. */
};

#define PP_MAX_KNOTS 64
#define PP_MAX_ABS 32
#define PP_MAX_PMT 256
#define PP_STATS 8 /* per pair: hits, sum w, sum w^2, sum w t, sum w t^2,
                      sum w ln t, photons, reserved */

/* WaterProperties, src/medium.jl:23-50 (permille, atm, degC, ppm, ppm,
 * g/cm^2) plus its absorption-length table, src/medium.jl:243-251
 * (n_abs == 0 selects the reference's 6-knot table). */
typedef struct {
  double salinity;
  double pressure;
  double temperature;
  double vol_conc_small_part;
  double vol_conc_large_part;
  double radiation_length;
  int32_t n_abs;
  int32_t pad;
  double abs_wl[PP_MAX_ABS];
  double abs_len[PP_MAX_ABS];
} pp_medium_desc;

/* CherenkovSpectrum(wl_range, interp_steps, medium), src/spectrum.jl:90-103,
 * or Monochromatic(wavelength), src/spectrum.jl:14-16 (wl_min). */
typedef struct {
  int32_t kind;
  int32_t n_knots;
  double wl_min;
  double wl_max;
} pp_spectrum_desc;

/* PMTWavelengthAcceptance table, src/detection.jl:18-33 (sorted by
 * wavelength; n == 0 means acceptance 1). */
typedef struct {
  int32_t n;
  int32_t pad;
  double wavelength[PP_MAX_PMT];
  double acceptance[PP_MAX_PMT];
} pp_pmt_desc;

/* One source-target pair: PhotonSource (src/emission.jl:102-109) plus
 * DetectionSphere (src/detection.jl:10-15).  80 bytes. */
typedef struct {
  float pos[3];      /* emitter position (track start for a cone emitter) */
  float t0;          /* emission time, ns */
  float dir[3];      /* track direction of a cone emitter (unit) */
  float track_len;   /* track length, m (cone emitter) */
  float target[3];   /* sphere centre */
  float radius;      /* sphere radius */
  int64_t n_photons; /* photons to propagate */
  uint64_t seed;     /* random stream: depends only on (seed, photon) */
  int32_t emitter;   /* PP_EMITTER_* */
  int32_t reserved[3];
} pp_pair;

/* Run options.  pp_default_opts fills the defaults of a mode. */
typedef struct {
  int32_t mode;       /* PP_MODE_COMPAT reproduces the reference arithmetic,
                         PP_MODE_PHYSICAL the physical model */
  int32_t max_steps;  /* compat: 10 (src/photon_prop_cuda.jl:319) */
  float g;            /* Henyey-Greenstein asymmetry (reference: 0.99, :229) */
  float t_max;        /* physical mode: photons end at this arrival time, ns */
  float hist_t0;      /* arrival-time histogram origin, ns */
  float hist_bin_width;
  int32_t hist_bins;  /* 0: no histogram */
  uint32_t flags;     /* PP_OPT_* */
  int32_t block_size; /* launch tuning; 0 = autotuned/default */
  int32_t blocks_per_sm;
  int32_t chunk_photons;
  int32_t reserved;
} pp_run_opts;

/* One detected photon.  64 bytes, written with four 16-byte stores. */
typedef struct {
  float pos[3];     /* hit position on the sphere */
  float time;       /* arrival time, ns */
  float dir0[3];    /* emission direction (reference output, :370) */
  float weight;     /* absorption weight x PMT acceptance (if enabled) */
  float dir[3];     /* arrival direction */
  float wavelength; /* nm */
  float dist;       /* path length, m */
  uint32_t pair;    /* index of the pair in the call */
  uint64_t photon;  /* photon index within the pair */
} pp_hit;

/* Compact hit record (PP_OPT_COMPACT_HITS), 32 bytes: what the serving loop
 * returns.  photon_lo holds the low 32 bits of the photon index. */
typedef struct {
  float pos[3];
  float time;
  float weight;
  float wavelength;
  uint32_t photon_lo;
  uint32_t pair;
} pp_hit32;

typedef struct pp_ctx pp_ctx;

/* ---- library ------------------------------------------------------------ */
PP_API int pp_abi_version(void);
PP_API const char* pp_version(void);
/* Kernels this process has launched through the library (all contexts). */
PP_API uint64_t pp_launch_count(void);
/* splitmix64 of (global_seed, index): the per-pair seed of a batch. */
PP_API uint64_t pp_pair_seed(uint64_t global_seed, uint64_t index);

/* ---- host physics (FP64; the reference's Medium/Spectral functions) ----- */
/* get_refractive_index, src/medium.jl:125-158,179-183 */
PP_API double pp_refractive_index(const pp_medium_desc* m, double wavelength_nm);
/* group index n - lambda dn/dlambda of the same model (no reference counterpart) */
PP_API double pp_group_index(const pp_medium_desc* m, double wavelength_nm);
/* get_scattering_length, src/medium.jl:201-235 */
PP_API double pp_scattering_length(const pp_medium_desc* m, double wavelength_nm);
/* get_absorption_length, src/medium.jl:243-251 */
PP_API double pp_absorption_length(const pp_medium_desc* m, double wavelength_nm);
/* p_one_pmt_acc, src/detection.jl:27-33 */
PP_API double pp_pmt_acceptance(const pp_pmt_desc* p, double wavelength_nm);
/* CherenkovSpectrum(...).knots, src/spectrum.jl:54-70,77-82,96-101 */
PP_API pp_status pp_cherenkov_knots(const pp_medium_desc* m, double wl_min, double wl_max,
                             int32_t n_knots, double* knots_out);
/* Fills the defaults of a mode: compat = 10 steps, g 0.99, no time window;
 * physical = g 0.95, t_max 500 ns, 500 x 1 ns bins. */
PP_API pp_status pp_default_opts(int32_t mode, pp_run_opts* out);

/* ---- context ------------------------------------------------------------ */
/* Builds the device-resident tables (spectrum knots, absorption and PMT
 * tables, medium coefficients) on `device`.  pmt may be NULL. */
PP_API pp_status pp_create(pp_ctx** out, int device, const pp_medium_desc* medium,
                    const pp_spectrum_desc* spectrum, const pp_pmt_desc* pmt);
PP_API void pp_destroy(pp_ctx* ctx);
PP_API const char* pp_last_error(const pp_ctx* ctx);
PP_API int pp_device(const pp_ctx* ctx);
/* The float spectrum knots resident on the device. */
PP_API pp_status pp_get_knots(const pp_ctx* ctx, float* out, int32_t cap, int32_t* n);

/* ---- hot path ------------------------------------------------------------ */
/* Batched persistent kernel over all pairs (device work queue of photon
 * chunks), host buffers, synchronous.  Replaces propagate_distance
 * (src/photon_prop_cuda.jl:588-644) for any number of source-target pairs.
 * hits: hit_capacity records (may be NULL with capacity 0); stats:
 * n_pairs x PP_STATS doubles; hist: n_pairs x hist_bins doubles (NULL if
 * hist_bins == 0).  *n_hits receives the total hit count. */
PP_API pp_status pp_propagate(pp_ctx* ctx, const pp_pair* pairs, int64_t n_pairs,
                       const pp_run_opts* opts, pp_hit* hits, int64_t hit_capacity,
                       int64_t* n_hits, double* stats, double* hist);

/* Same results, one kernel launch per pair with a host synchronisation and
 * copy-back after each, as propagate_distance does per distance
 * (src/modelling.jl:96-99). */
PP_API pp_status pp_propagate_plain(pp_ctx* ctx, const pp_pair* pairs, int64_t n_pairs,
                             const pp_run_opts* opts, pp_hit* hits, int64_t hit_capacity,
                             int64_t* n_hits, double* stats, double* hist);

/* Device-buffer, asynchronous form of pp_propagate on `stream` (a
 * cudaStream_t; NULL = legacy default stream).  counters: 4 uint64 on the
 * device, [0] = total hits, [1] = photon steps taken, [2] = status bits
 * (1 = hit overflow), [3] reserved; they are reset by the call.  The work
 * queue lives in context-owned device scratch memory.  Repeated calls with
 * the same shapes and buffers replay a captured CUDA graph. */
PP_API pp_status pp_propagate_device(pp_ctx* ctx, const pp_pair* d_pairs, int64_t n_pairs,
                              const pp_run_opts* opts, pp_hit* d_hits, int64_t hit_capacity,
                              uint64_t* d_counters, double* d_stats, double* d_hist,
                              void* stream);

/* Allocation-free form of pp_propagate_device.  It has no counterpart in the
 * reference.  It exists for callers that own all device memory through their
 * own pool and cannot let a library call cudaMalloc behind their back: Julia's
 * CUDA.jl allocator or PyTorch's caching allocator may hold the free memory,
 * so a library cudaMalloc can fail, and cudaMalloc/cudaFree can synchronise
 * the device in the middle of the caller's stream work.  The work-queue
 * scratch (chunk offsets and queue cursor) lives in one static device array
 * of (PP_NOALLOC_MAX_PAIRS + 33) x 8 bytes (about 512 KiB) that every GPU
 * which loads the library holds until the process exits.  The call allocates
 * nothing, launches directly (no graph) and otherwise behaves like
 * pp_propagate_device.  Limits and rules:
 *  - n_pairs above PP_NOALLOC_MAX_PAIRS is rejected with PP_ERR_ARG;
 *  - every call looks up the array's device address with the context's
 *    device current; the first call on a device is the set-up (it may load the
 *    library's device code there), so make that first call before any stream
 *    capture; later lookups allocate nothing, and after a device reset the
 *    call finds the new context's array;
 *  - all calls share the array and it keeps the last call's contents (each
 *    call resets what must start at zero), so calls that overlap on the GPU
 *    race: issue them on one stream or otherwise serialise them. */
#define PP_NOALLOC_MAX_PAIRS 65536
PP_API pp_status pp_propagate_device_noalloc(pp_ctx* ctx, const pp_pair* d_pairs, int64_t n_pairs,
                                             const pp_run_opts* opts, pp_hit* d_hits, int64_t hit_capacity,
                                             uint64_t* d_counters, double* d_stats, double* d_hist,
                                             void* stream);

/* Device-buffer form of the plain kernel for one pair (no graph). */
PP_API pp_status pp_propagate_plain_device(pp_ctx* ctx, const pp_pair* d_pair, const pp_pair* h_pair,
                                    int64_t pair_index, const pp_run_opts* opts, pp_hit* d_hits,
                                    int64_t hit_capacity, uint64_t* d_counters, double* d_stats,
                                    double* d_hist, void* stream);

/* Kernel-level drop-in for cuda_propagate_photons!
 * (src/photon_prop_cuda.jl:262-386) with the reference's output layout:
 * per-block hit stacks of stack_len entries in SoA device arrays
 * (positions/directions: 3 floats per entry), 1-based per-block stack
 * pointers (0 = empty block; the index of the block's last hit) and the
 * number of photons simulated.  Each of n_blocks x threads threads
 * simulates cld(n_photons, n_blocks*threads) photons and a block stops when
 * its stack is nearly full, as in the reference.  source_target gives the
 * source and sphere; opts the physics mode (compat reproduces the
 * reference). */
PP_API pp_status pp_cuda_propagate_photons(pp_ctx* ctx, float* d_out_positions,
                                    float* d_out_directions, float* d_out_wavelengths,
                                    float* d_out_dist_travelled,
                                    int32_t* d_out_stack_pointers,
                                    int64_t* d_out_n_ph_simulated, int32_t stack_len,
                                    int32_t n_blocks, int32_t threads,
                                    const pp_pair* source_target, const pp_run_opts* opts,
                                    void* stream);

/* ---- fit stage: Cherenkov reweighting and Gamma fits -------------------- */
/* The caller of the hot path in the reference (src/modelling.jl:46-111,
 * src/emission.jl:32-99): photons propagated from an isotropic source are
 * reweighted to the Cherenkov angular distribution of an EM cascade at each
 * observation angle a,
 *   w_dir = cherenkov_ang_dist(cos(theta0 - a), n) / (2 cherenkov_ang_dist_int(n)),
 * (theta0 the emission polar angle, n the phase index at the photon's
 * wavelength), multiplied by the hit weight, and a Gamma distribution is
 * fitted by maximum likelihood to the weighted arrival-time residuals
 * tres = t - (|target - source| - r) n(800 nm) / c.  The
 * detection fraction is the summed weight of all hits over the photons
 * generated.  The fit takes tres > 0 (the reference's mask is tres >= 0: a
 * residual of exactly 0, which FP32 rounding makes common for photons that
 * fly straight at the sphere, has no Gamma likelihood). */
#define PP_FIT_MOMENTS 4 /* per (pair, angle): sum w (all hits), then over tres > 0:
                            sum w, sum w tres, sum w ln(tres) */
#define PP_FIT_OUT 3     /* per (pair, angle): fit_alpha, fit_theta, det_fraction */
#define PP_MAX_FIT_ANGLES 4096
/* cherenkov_ang_dist with the e- parameters (4.27033, -6.02527, 0.29887,
 * -0.00103), src/emission.jl:19-44. */
PP_API double pp_cherenkov_ang_dist(double costheta, double ref_index);
/* _cherenkov_ang_dist_int over [lower, upper], the reference's closed form
 * with the upper incomplete gamma function, src/emission.jl:52-86. */
PP_API double pp_cherenkov_ang_dist_int_exact(double ref_index, double lower, double upper);
/* cherenkov_ang_dist_int: linear interpolation of the [-1, 1] integral on
 * ref_index = 1.1:0.01:1.5, src/emission.jl:88-99 (NaN outside). */
PP_API double pp_cherenkov_ang_dist_int(double ref_index);
/* cos(theta) of the cascade emitter for a uniform u in (0, 1) at refractive
 * index n, from the library's FP64 tables (the kernel samples the same
 * tables in FP32). */
PP_API double pp_cascade_cos_theta(double u, double ref_index);
/* get_dir_reweight(thetas, obs_angle, ref_ixs), src/modelling.jl:46-49:
 * out[i] = cherenkov_ang_dist(cos(thetas[i] - obs_angle), ref_ixs[i]) /
 *          (2 cherenkov_ang_dist_int(ref_ixs[i])). */
PP_API pp_status pp_dir_reweight(const double* thetas, double obs_angle, const double* ref_ixs, double* out,
                                 int64_t n);

/* Propagates the batch (as pp_propagate) and runs the fit stage on the
 * device for every pair and each of the n_angles observation angles
 * (radians, host array): fits = n_pairs x n_angles x PP_FIT_OUT doubles
 * (fit_alpha and fit_theta of the weighted Gamma maximum-likelihood fit, NaN
 * where no hit has tres > 0; det_fraction); moments (may be NULL) =
 * n_pairs x n_angles x PP_FIT_MOMENTS; stats / hist as pp_propagate (may be
 * NULL); *n_hits = all hits.  hit_capacity sizes the device hit buffer:
 * pairs run in waves whose hits fit it, planned from a pilot launch of the
 * first photons of every pair (a wave that overflows is repacked with the
 * exact per-pair hit counts it produced and run again), so it bounds
 * memory, not the number of hits; PP_ERR_OVERFLOW
 * only when one pair alone has more hits.  The whole of make_photon_fits
 * (src/modelling.jl:86-111) for all distances is one call. */
PP_API pp_status pp_propagate_fit(pp_ctx* ctx, const pp_pair* pairs, int64_t n_pairs,
                                  const pp_run_opts* opts, const double* obs_angles, int32_t n_angles,
                                  int64_t hit_capacity, int64_t* n_hits, double* fits, double* moments,
                                  double* stats, double* hist);

/* Device-buffer form of the fit stage over hits already on the device (full
 * pp_hit records from pp_propagate_device with the same pairs and mode):
 * hits counted by d_counters[0] (at most hit_capacity are read).  d_moments
 * and d_fits as above, device memory; obs_angles is a host array. */
PP_API pp_status pp_fit_hits_device(pp_ctx* ctx, const pp_pair* d_pairs, int64_t n_pairs, int32_t mode,
                                    const pp_hit* d_hits, int64_t hit_capacity, const uint64_t* d_counters,
                                    const double* obs_angles, int32_t n_angles, double* d_moments,
                                    double* d_fits, void* stream);

/* fit_photon_dist(obs_angles, obs_photon_df, n_ph_gen), src/modelling.jl:52-79,
 * over a hit table given as FP64 device columns (tres, initial_theta,
 * ref_ix, abs_weight, wavelength; n rows): the PMT acceptance of the
 * context is applied to each photon's wavelength as the reference does.
 * d_moments: n_angles x PP_FIT_MOMENTS, d_fits: n_angles x PP_FIT_OUT. */
PP_API pp_status pp_fit_photon_dist_device(pp_ctx* ctx, int64_t n, const double* d_tres,
                                           const double* d_initial_theta, const double* d_ref_ix,
                                           const double* d_abs_weight, const double* d_wavelength,
                                           const double* obs_angles, int32_t n_angles, int64_t n_ph_gen,
                                           double* d_moments, double* d_fits, void* stream);

/* ---- light yield: particles -> light sources (src/lightyield.jl) -------- */
enum { PP_PARTICLE_EMINUS = 11, PP_PARTICLE_EPLUS = -11, PP_PARTICLE_GAMMA = 22 };
/* Particle, src/lightyield.jl:201-207: position (m), time (ns), direction
 * (unit), energy (GeV), type (PP_PARTICLE_*).  48 bytes. */
typedef struct {
  float pos[3];
  float time;
  float dir[3];
  float energy;
  int32_t type;
  int32_t reserved[3];
} pp_particle;
/* Units of the longitudinal grid.  PP_LY_REFERENCE reproduces the
 * reference's arithmetic: grid values are centimetres in the shower profile
 * and are used unchanged as metres for the source positions and times
 * (src/lightyield.jl:253-256), and the water density is the reference's
 * expression A / B^((1 + (1 - T)/C)^D) with T in degC (src/medium.jl:78).
 * PP_LY_METRES takes the grid in metres (converted to centimetres for the
 * profile) and the DIPPR105 density A / B^(1 + (1 - T/C)^D), T in kelvin. */
enum { PP_LY_REFERENCE = 0, PP_LY_METRES = 1 };
/* density(medium) in kg/m^3 (src/medium.jl:69-92) */
PP_API double pp_medium_density(const pp_medium_desc* m, int32_t ly_mode);
/* longitudinal_profile(energy, z, medium, ptype), src/lightyield.jl:116-140:
 * energy in GeV, z in cm; per cm. */
PP_API double pp_longitudinal_profile(const pp_medium_desc* m, int32_t ly_mode, int32_t ptype, double energy_gev,
                                      double z_cm);
/* cherenkov_track_length(_dev), src/lightyield.jl:190-198 (cm); NaN for an unknown type. */
PP_API double pp_cherenkov_track_length(int32_t ptype, double energy_gev);
PP_API double pp_cherenkov_track_length_dev(int32_t ptype, double energy_gev);
/* frank_tamm_norm(wl_range, n(medium)), src/spectrum.jl:41-45: Cherenkov photons per cm of track. */
PP_API double pp_frank_tamm_norm(const pp_medium_desc* m, double wl_min, double wl_max);
/* fractional_contrib_long!(energy, z_grid, medium, ptype, out),
 * src/lightyield.jl:143-169: out[0] = 0, out[i] = the profile's share of
 * [z[i-1], z[i]] (50-point Gauss-Legendre over each interval and over the
 * whole grid); z in cm. */
PP_API pp_status pp_fractional_contrib_long(const pp_medium_desc* m, int32_t ly_mode, int32_t ptype,
                                            double energy_gev, const double* z_grid_cm, int64_t n, double* out);
/* particle_to_elongated_lightsource for n_particles particles on the device
 * (src/lightyield.jl:219-285): the grid len_min:precision:len_max (n_grid
 * points, Julia's range) gives n_grid - 1 sources per particle at the
 * interval midpoints, with round(frank_tamm_norm(wl_range) x
 * cherenkov_track_length(E) x fractional share) photons, written as pairs
 * (position, time, direction, photons, `emitter`; target and seed unset):
 * source k of particle p is d_sources[p * (n_grid - 1) + k].  An isotropic
 * or cascade-profile source sits at the midpoint; a Cherenkov-cone source is
 * a track over its interval along the particle.  n_grid comes back in
 * *n_grid. */
PP_API pp_status pp_particles_to_sources_device(pp_ctx* ctx, const pp_particle* d_particles, int64_t n_particles,
                                                double len_min, double len_max, double precision, int32_t ly_mode,
                                                double wl_min, double wl_max, int32_t emitter, pp_pair* d_sources,
                                                int64_t capacity, int64_t* n_grid, void* stream);
/* Every source with every target sphere (d_targets: x, y, z, radius floats):
 * d_pairs[s * n_targets + t], seed pp_pair_seed(seed, s * n_targets + t). */
PP_API pp_status pp_cross_pairs_device(pp_ctx* ctx, const pp_pair* d_sources, int64_t n_sources,
                                       const float* d_targets, int64_t n_targets, uint64_t seed, pp_pair* d_pairs,
                                       void* stream);

/* ---- event likelihood: Poisson x arrival-time mixture per module -------- */
/* The extended likelihood of example_full.jl:338-449 for n_hyp hypotheses
 * of one event at once, one block per (hypothesis, module).  Per source j
 * and module k, d_params[((h * n_modules + k) * n_sources + j) * PP_LLH_PARAMS]
 * (module-major: a module's sources are contiguous) holds
 * (A, w, alpha1, alpha2, theta, t_shift): the expected photons are
 * mu_jk = A x N_j (N_j = d_source_photons[h * n_sources + j], or 1 when that
 * pointer is NULL) and the arrival-time density is
 *   g_jk(x) = w Gamma(x - t_shift; alpha1, theta) + (1 - w) Gamma(x - t_shift; alpha2, theta).
 * With mu_k = sum_j mu_jk and the module's hit times x (CSR: d_hit_offsets
 * [n_modules + 1] into d_hit_times),
 *   llh_k = n_k ln mu_k - mu_k - ln n_k! + sum_x ln(sum_j q_jk g_jk(x)),
 * q_jk = mu_jk / mu_k (PP_LLH_SHIFTED), or q_jk = A_jk / sum_j A_jk
 * (PP_LLH_REFERENCE: shape_mixture_per_module weighs the sources by their
 * detection fraction alone, example_full.jl:362-377).  FP64 throughout;
 * d_llh[h * n_modules + k]. */
#define PP_LLH_PARAMS 6
enum { PP_LLH_REFERENCE = 0, PP_LLH_SHIFTED = 1 };
PP_API pp_status pp_event_llh_device(pp_ctx* ctx, int32_t mode, int64_t n_hyp, int64_t n_sources, int64_t n_modules,
                                     const double* d_params, const double* d_source_photons,
                                     const int64_t* d_hit_offsets, const double* d_hit_times, double* d_llh,
                                     void* stream);

/* ---- serving: continuous batching ----------------------------------------- */
/* A request is a list of pairs.  A scheduler thread admits waiting requests
 * while their hit buffers fit the HBM budget (bytes_per_hit per expected hit)
 * and an in-flight slot is free, packs every admitted request into one batched
 * launch on that slot's stream, and keeps up to max_inflight batches on the
 * device at once; requests that arrive while batches run join the next batch
 * as slots and memory free up.  The medium tables and the kernels' RNG (a
 * counter-based stream, no state) are resident in the context.  Results are
 * the same as a request alone: a pair's photons depend only on its seed. */
typedef struct {
  int32_t max_inflight;        /* batches on the device at once (streams); 0 = 2 */
  int32_t max_pairs_per_batch; /* 0 = 4096 */
  int64_t hbm_budget_bytes;    /* admission budget; 0 = 40 GiB */
  int32_t bytes_per_hit;       /* admission bytes per expected hit; 0 = 32 (pp_hit32) */
  float hit_safety;            /* hit slots per expected hit; 0 = 4 */
  int32_t max_queued;          /* waiting requests before submit says PP_ERR_BUSY; 0 = 100000 */
  int32_t reserved;
  pp_run_opts opts;            /* physics and histogram options of every request */
} pp_server_config;

typedef struct pp_server pp_server;

typedef struct {
  int64_t submitted, completed, batches, pairs, in_flight_batches, waiting;
  int64_t reserved_bytes;
  double photons;
} pp_server_counters;

/* Starts the scheduler thread on ctx's device; the context must outlive the server. */
PP_API pp_status pp_server_create(pp_ctx* ctx, const pp_server_config* cfg, pp_server** out);
/* Stops the scheduler after the batches on the device finish. */
PP_API void pp_server_destroy(pp_server* s);
/* Queues a request (the pairs are copied); never blocks.  PP_ERR_BUSY when
 * max_queued requests wait, PP_ERR_ARG when it could never fit the budget. */
PP_API pp_status pp_server_submit(pp_server* s, const pp_pair* pairs, int32_t n_pairs, uint64_t* request_id);
/* Waits up to timeout_s for a request (PP_ERR_TIMEOUT after that). */
PP_API pp_status pp_server_wait(pp_server* s, uint64_t request_id, double timeout_s);
/* Copies a finished request's results out and forgets it: compact hits (up
 * to hit_capacity; *n_hits = its hits in the buffer), stats [n_pairs x 8],
 * hist [n_pairs x bins], latency = completion - submission in seconds.
 * PP_ERR_STATE if the request is not finished; PP_ERR_OVERFLOW if some of its
 * hits did not fit the batch's hit buffer (stats and hist are complete). */
PP_API pp_status pp_server_result(pp_server* s, uint64_t request_id, pp_hit32* hits, int64_t hit_capacity,
                                  int64_t* n_hits, double* stats, double* hist, double* latency_s);
PP_API pp_status pp_server_get_counters(pp_server* s, pp_server_counters* out);

/* ---- learned surrogate ------------------------------------------------------ */
/* MLP 4 -> 128 -> 128 -> 128 -> 5 (GELU) replacing the reference's Flux
 * fits (src/modelling.jl:202-267).  Inputs per query (raw): log10 distance,
 * cos(emitter-target angle), log10 photons, emitter flag.  Outputs: ln(mu/N)
 * (mu = expected weighted hits), logit w, ln a1, ln a2, ln theta of a
 * two-component Gamma mixture w G(a1, theta) + (1-w) G(a2, theta) of the time
 * residual; `physical` returns (mu, w, a1, a2, theta) instead.  BF16 weights
 * and activations, FP32 accumulation; the 128 x 128 layers run on tcgen05
 * tensor cores.  Parameters: N_PARAMS FP32 values in the order W1[128][4],
 * b1, W2[128][128], b2, W3[128][128], b3, W4[5][128], b4. */
typedef struct pp_mlp pp_mlp;
PP_API pp_status pp_mlp_create(int device, uint64_t seed, pp_mlp** out);
PP_API void pp_mlp_destroy(pp_mlp* m);
PP_API const char* pp_mlp_last_error(const pp_mlp* m);
PP_API int32_t pp_mlp_num_params(void);
PP_API pp_status pp_mlp_get_params(pp_mlp* m, float* out);
PP_API pp_status pp_mlp_set_params(pp_mlp* m, const float* in);
/* Feature and target standardisation: x' = (x - mean) / std, y = y' std + mean. */
PP_API pp_status pp_mlp_set_normalization(pp_mlp* m, const float* x_mean, const float* x_std, const float* y_mean,
                                          const float* y_std);
PP_API pp_status pp_mlp_get_normalization(pp_mlp* m, float* out18);
/* Inference on device buffers: x [n][4], out [5][n]. */
PP_API pp_status pp_mlp_forward(pp_mlp* m, const float* d_x, float* d_out, int64_t n, int32_t physical,
                                void* stream);
/* One Adam step (lr > 0) on standardised device data xn [n][4], yt [n][5],
 * mask [n][5] with masked-MSE loss; *loss_out = mean loss; grad_out (host,
 * N_PARAMS) receives the gradients if not NULL (lr = 0: gradients only). */
PP_API pp_status pp_mlp_train_step(pp_mlp* m, const float* d_xn, const float* d_yt, const float* d_mask, int64_t n,
                                   float lr, float* loss_out, float* grad_out);
/* One 128 x 128 x 128 BF16 GEMM (c = a b^T, row-major) through the tcgen05
 * path: a check of the tensor-core descriptors. */
PP_API pp_status pp_mlp_gemm_selftest(int device, const uint16_t* a_bf16, const uint16_t* b_bf16, float* c);

/* Fits w G(a1, theta) + (1 - w) G(a2, theta) to each of n histograms
 * (device, FP64 [n][bins], bin b centred at t0 + (b + 1/2) bin_width) as a
 * function of t - tshift[i] by weighted EM (iters iterations); d_out [n][5] =
 * w, a1 <= a2, theta, mean log-likelihood (NaN for empty histograms). */
PP_API pp_status pp_gamma_mixture_fit(const double* d_hist, int64_t n, int32_t bins, float t0, float bin_width,
                                      const float* d_tshift, float* d_out, int32_t iters, void* stream);

/* ---- tuning and diagnostics ---------------------------------------------- */
/* Times the batched kernel over (block size, blocks per SM, chunk) on a
 * sample of `pairs` and stores the best in the context (and in the cache
 * file at cache_path if not NULL).  best_out may be NULL. */
PP_API pp_status pp_autotune(pp_ctx* ctx, const pp_pair* pairs, int64_t n_pairs,
                      const pp_run_opts* opts, const char* cache_path,
                      pp_run_opts* best_out, double* best_photons_per_s);

/* Evaluates a device helper on n inputs (unit tests of the device code, the
 * counterpart of the reference's apply_rot test kernel,
 * src/tests/test_photon_prob.jl:32-35).  op: 0 philox words (in: 6 per item
 * ctr0..3,key0..1 as doubles; out: 4), 1 uniform (in: word; out: 1),
 * 2 HG cos theta (in: g,u), 3 rotate_to_axis (in: old[3],new[3]; out: 3),
 * 4 update_position (in: pos[3],dir[3],step; out: 3), 5 equidistant
 * interpolation of the context's knots (in: u), 6 refractive index,
 * 7 group index, 8 scattering length, 9 absorption length, 10 PMT
 * acceptance (in: wavelength), 11 cascade-emitter cos theta (in: u, n),
 * 12 a step's Philox2x32-10 block and its three uniforms (in: counter
 * words 0, 1 and the key; out: w0, w1, u0, u1, u2). */
PP_API pp_status pp_device_eval(pp_ctx* ctx, int32_t op, const double* in, double* out, int64_t n);

/* Measures this device's FP32 FMA and MUFU (transcendental) issue peaks with
 * independent dependent-chain microbenchmarks over every SM (operations per
 * second) and its Philox4x32-10 block rate (blocks per second). */
PP_API pp_status pp_measure_peaks(int device, double* fp32_ops_per_s, double* mufu_ops_per_s,
                           double* philox_blocks_per_s);

/* Speed of light of the physical photon step on this device: photon steps
 * per second when every lane of every SM steps its own photon (one
 * Philox2x32-10 block, ray-sphere test, move, Henyey-Greenstein turn) with no
 * emission, refill, hit record or loop bookkeeping, at the batched kernel's
 * occupancy.  No reference counterpart: the ceiling the batched kernel's
 * step rate is reported against. */
PP_API pp_status pp_measure_step_rate(int device, double* steps_per_s);

#ifdef __cplusplus
}
#endif
#endif
