// Internal interfaces between the C-ABI layer (pp_capi.cu) and the kernels
// (pp_kernels.cu) / host physics (pp_host_physics.cpp).
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <mutex>

#include "photonprop_b200.h"

namespace pp {

// Named host-side range for profilers (NVTX, header only: without a
// profiler attached a push/pop pair is a check of one pointer).
struct Range {
  explicit Range(const char* name) { nvtxRangePushA(name); }
  ~Range() { nvtxRangePop(); }
  Range(const Range&) = delete;
  Range& operator=(const Range&) = delete;
};

// Everything one launch of the propagation kernels reads or writes.
struct LaunchArgs {
  const pp_pair* pairs;
  int64_t n_pairs;
  unsigned long long* chunk_offsets;  // [n_pairs + 1] scratch
  unsigned long long* queue;          // [1] scratch
  uint32_t chunk;
  pp_hit* hits;
  unsigned long long hit_cap;
  unsigned long long* counters;  // [4]
  double* stats;
  double* hist;
  const void* tables;  // device DevTables
  pp_run_opts opts;
  uint32_t pair_base;  // added to the pair index written into hits
};

void count_launches(uint64_t n);

size_t dev_tables_size();
// coeffs: a01, a2, a3, a4, sca0, sca1, sca2 (+ unused)
void fill_dev_tables(void* host_tables, const double coeffs[11], const float* knots, int n_knots,
                     const float* abs_wl, const float* abs_len, int n_abs, const float* pmt_wl,
                     const float* pmt_acc, int n_pmt);
// Points the tables at the cascade emitter's device tables (kCascNF + 1
// forward values, then kCascNI + 1 inverse values) with G's range.
void set_cascade_tables(void* host_tables, const float* d_casc, double gmin, double gmax);
void get_dev_knots(const void* host_tables, float* out, int* n);

cudaError_t launch_chunk_scan(const LaunchArgs& a, cudaStream_t s);
cudaError_t launch_reset_counters(unsigned long long* counters, cudaStream_t s);
cudaError_t launch_batched(const LaunchArgs& a, int grid, int block, cudaStream_t s);
cudaError_t launch_plain(const LaunchArgs& a, const pp_pair* d_pair, int pair_index, int grid, int block,
                         cudaStream_t s);
cudaError_t launch_stacks(const LaunchArgs& a, const pp_pair* d_pair, float* pos, float* dir, float* wl,
                          float* dist, int32_t* sp, int64_t* nsim, int stack_len, int grid, int block,
                          long long per_thread, cudaStream_t s);
cudaError_t launch_finalize(const pp_pair* pairs, int64_t n, double* stats, double* hist, int bins, int normalize,
                            int sm_count, cudaStream_t s);
cudaError_t launch_eval(int op, const double* in, double* out, int64_t n, const void* tables, cudaStream_t s);
int batched_max_blocks_per_sm(int mode, int block, bool cascade);
int plain_max_blocks_per_sm(int mode, int block);
cudaError_t run_peaks(int sm_count, double* fp32, double* mufu, double* iops);
cudaError_t run_step_rate(int sm_count, double* steps_per_s);

// batched launch with caller-owned scratch, direct launches (pp_capi.cu)
pp_status propagate_with_scratch(pp_ctx* c, const pp_pair* d_pairs, int64_t n_pairs, const pp_run_opts* opts,
                                 void* d_hits, int64_t cap, uint64_t* d_counters, double* d_stats,
                                 double* d_hist, unsigned long long* d_offsets, unsigned long long* d_queue,
                                 cudaStream_t stream);
int ctx_device(const pp_ctx* c);
int ctx_sm_count(const pp_ctx* c);
const pp_medium_desc* ctx_medium(const pp_ctx* c);
pp_status ctx_fail(pp_ctx* c, pp_status s, const char* msg);
pp_status ctx_cuda_fail(pp_ctx* c, cudaError_t e, const char* where);
std::mutex& ctx_mutex(pp_ctx* c);
cudaError_t ctx_llh_scratch(pp_ctx* c, size_t bytes, void** out);  // caller holds the context mutex

// Cherenkov angular distribution of EM cascades, e- parameters
// (src/emission.jl:19), and the reference's table of its [-1, 1] integral
// over the refractive index 1.1:0.01:1.5 (src/emission.jl:88-99).
constexpr double kAngA = 4.27033, kAngB = -6.02527, kAngC = 0.29887, kAngD = -0.00103;
constexpr int kAngIntN = 41;
constexpr double kAngIntN0 = 1.1, kAngIntDn = 0.01;
double upper_incomplete_gamma(double s, double z);
double cherenkov_ang_dist_int_closed(double ref_index, double lower, double upper);
void cherenkov_ang_dist_int_table(double* out);
double ang_int_interp(const double* table, double n);
// Inverse-CDF tables of the cascade emitter: G(v) = integral of
// a exp(b |v|^c) + d, v = cos(theta) - 1/n, on kCascNF + 1 uniform points of
// [kCascVMin, kCascVMax], and v at kCascNI + 1 uniform levels of G.
constexpr int kCascNF = 2048, kCascNI = 8192;
constexpr double kCascVMin = -1.85, kCascVMax = 0.35;  // 1/n in [0.65, 0.85]
double cascade_G(double v);
void cascade_tables(double* fwd, double* inv);
double cascade_sample(const double* fwd, const double* inv, double u, double ref_index);

// fit stage (pp_fit.cu)
struct FitConsts {
  float a, b_l2, c, d;         // cherenkov_ang_dist parameters, b in base 2
  float n800_phase, n800_group;  // refractive indices at 800 nm (tgeo)
  float inv_dn;
  float normf[kAngIntN];       // [-1, 1] integral on 1.1:0.01:1.5
};
struct FitRec {  // 32 bytes, one per hit
  float ct, st, c0, wn;  // cos / sin of the emission polar angle, 1/n, weight / (2 int(n))
  float tres, lnt;       // arrival-time residual and its log
  int32_t pair;
  int32_t pos;  // tres >= 0
};
static_assert(sizeof(FitRec) == 32, "FitRec is moved as two 16-byte words");
void fill_fit_consts(FitConsts* K, double n800_phase, double n800_group);
// Adds the moments of the stored hits (their pair fields index `pairs`) to
// moments [n_pairs x n_angles x 4]; the caller zeroes moments first.
cudaError_t launch_fit_moments_hits(const FitConsts& K, const void* tables, const pp_pair* pairs, int64_t n_pairs,
                                    int mode, const pp_hit* hits, unsigned long long cap,
                                    const unsigned long long* counters, unsigned long long* counts, FitRec* rec,
                                    const float2* cs, int n_angles, double* moments, int sm_count, cudaStream_t s);
// Gamma fits and detection fractions of every (pair, angle) from the moments.
cudaError_t launch_fit_gamma(const double* moments, int64_t n_pairs, int n_angles, const pp_pair* pairs,
                             int64_t n_gen, double* fits, cudaStream_t s);
cudaError_t launch_fit_columns(const FitConsts& K, const void* tables, int64_t n, const double* tres,
                               const double* theta, const double* ref_ix, const double* abs_w, const double* wl,
                               FitRec* rec, const float2* cs, int n_angles, int64_t n_gen, double* moments,
                               double* fits, int sm_count, cudaStream_t s);

// host physics (pp_host_physics.cpp)
void gl_nodes(int n, double* x, double* w);  // Gauss-Legendre nodes and weights on [-1, 1]
double frank_tamm_norm_cm(const pp_medium_desc* m, double wl_min, double wl_max);  // photons per cm
void medium_coeffs(const pp_medium_desc* m, double out[11]);
void default_abs_table(double* wl, double* len, int* n);

}  // namespace pp
