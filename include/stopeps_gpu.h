/* C ABI of libstopeps_gpu.so: the B200 engine for the StoPEPS sample-ensemble
 * hot path (row boundary-MPS contraction, full update, Born sampling,
 * energy/weight contraction).
 *
 * Every entry point returns 0 on success or a nonzero sps_status; the message
 * of the last failure is available through sps_last_error.  The library owns
 * all device tensors behind integer ids; callers pass and receive plain host
 * arrays, which are borrowed for the duration of the call only.  A handle
 * owns one CUDA stream and must not be shared between threads.
 *
 * Each declaration names the reference interface (StoPEPS.jl v0.2.0, path
 * relative to the project root) that it replaces.
 */
#ifndef STOPEPS_GPU_H
#define STOPEPS_GPU_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct sps_handle sps_handle;

enum sps_status {
  SPS_OK = 0,
  SPS_ERR_ARGUMENT = 1,    /* ArgumentError / DimensionMismatch */
  SPS_ERR_CUDA = 2,        /* CUDA runtime failure */
  SPS_ERR_NUMERIC = 3,     /* "nonfinite boundary norm" (src/contraction/boundary_mps.jl:131) and
                              the other error(...) paths on nonfinite / nonpositive values */
  SPS_ERR_BORN = 4,        /* "invalid Born conditional ... increase chi_sampling",
                              "zero total mass" (src/sampling/born.jl:140-142) */
  SPS_ERR_CONVERGENCE = 5, /* device iteration cap reached (Jacobi SVD / eigh) */
  SPS_ERR_REPAIR = 6,      /* "PSD repair did not remove the FU residual failure"
                              (src/evolution/full_update.jl:500) */
  SPS_ERR_STATE = 7        /* unknown handle / state / cache id */
};

/* Model and solver controls: the RunConfig fields this path reads
 * (src/driver/config.jl:28-62), TFIM (src/models/tfim.jl:9-19) and
 * FullUpdate (src/evolution/full_update.jl:11-17). */
typedef struct sps_config {
  int32_t Lx, Ly;
  double J, h;
  int32_t trotter_order;
  int32_t fu_max_iterations;
  double fu_error_tolerance;
  double fu_diagonal_shift;
  int32_t fu_linear_max_iterations;
  double fu_linear_tolerance;
  int32_t record_boundary_entropy;
  int32_t device;
} sps_config;

/* BoundaryMPS(chi, sector_space) (src/contraction/boundary_mps.jl:11-18);
 * space0/space1 < 0 means sector_space = nothing.  absorption 0 is the
 * reference's row absorption (exact LQ sweep + truncated SVD sweep,
 * compress_boundary!, boundary_mps.jl:94-134); 1 is this library's zip-up
 * absorption (one sweep of truncated SVDs without a canonical form), which
 * has no counterpart in the reference; 2 is BoundaryMPSDiagonal
 * (src/contraction/diagonal_mps.jl: anti-diagonal layers, site blocks,
 * truncation of the bonds a block opens), taken by sps_lognorm,
 * sps_measure_energy, the sampling caches and, for its bond environments,
 * the full update (src/evolution/diagonal_update.jl); 3 is
 * BoundaryMPSRowVariational (src/contraction/row_variational.jl: every row
 * absorbed by a two-site variational fit; its sweep options are the
 * handle's, sps_set_variational); 4 is BoundaryMPSDiagonalVariational
 * (src/contraction/diagonal_variational.jl: every diagonal layer absorbed by
 * a two-site variational fit, the same options). */
typedef struct sps_boundary {
  int32_t chi;
  int32_t space0, space1;
  int32_t absorption;
} sps_boundary;

/* Report of evolution_step! (src/evolution/full_update.jl:580-596). */
typedef struct sps_step_report {
  double beta;
  double max_state_truncation;
  double max_environment_truncation;
  double max_boundary_entropy;
  double max_solver_residual;
  double max_iteration_limit_error;
  int32_t bond_updates;
  int32_t iteration_limit_hits;
  int32_t stop_error_tolerance, stop_iteration_limit, stop_residual_fallback, stop_disabled;
  int32_t linear_unconverged_updates;
  int32_t repairs;
  int32_t fallbacks;
  double log_normalization_sum;
} sps_step_report;

/* lognorm (src/contraction/boundary_mps.jl:180-186). */
typedef struct sps_lognorm_result {
  double log_norm, tensor_log_norm, max_environment_truncation;
} sps_lognorm_result;

/* measure_energy (src/measurement/energy.jl:31-78); x_sum is the on-site
 * ratio sum the reference forms at energy.jl:43-46, exposed as <sum X_i>. */
typedef struct sps_energy {
  double energy_total, energy_per_site;
  double log_norm, tensor_log_norm;
  double max_environment_truncation;
  double x_sum, zz_sum;
} sps_energy;

/* sample_configuration result (src/sampling/born.jl:86-163). */
typedef struct sps_sample_report {
  double log_probability;
  double max_environment_truncation;
  int32_t near_boundary; /* draws whose uniform lay within 1e-12 of a cumulative probability */
  /* kind = physical (the resampling proposal): the `repairs` records of the
   * draw (born.jl:119-131) as counts, 0 for the auxiliary kind */
  int32_t metric_repairs;          /* site metrics whose negative eigenvalues were clipped */
  int32_t zero_proposals;          /* sites whose allowed outcomes all had zero weight */
  double min_relative_eigenvalue;  /* smallest site-metric eigenvalue / its spectral scale (<= 0) */
} sps_sample_report;

/* --- lifetime ------------------------------------------------------------ */
int sps_create(const sps_config* cfg, sps_handle** out);
void sps_destroy(sps_handle* h);
int sps_last_error(const sps_handle* h, char* buf, size_t n);
int sps_counters(sps_handle* h, long long* kernel_launches, double* flops);
/* Measurement support (no reference counterpart): per-kernel CUDA-event
 * timing on the handle's stream, reported as JSON
 * {"kernel": {"ms":..,"count":..,"flops":..,"bytes":..}, ...}; and a
 * device-side stopwatch (events on the handle's stream; stop synchronizes). */
int sps_set_profile(sps_handle* h, int32_t enable);
int sps_kernel_stats_json(sps_handle* h, char* buf, size_t n);
int sps_timer_start(sps_handle* h);
int sps_timer_stop(sps_handle* h, double* milliseconds);

/* Self-test / timing entry points of the dense factorization kernels (no
 * reference counterpart; they stand in for LAPACK gesdd / geqrf+orgqr).
 * Column-major host matrices.  sps_la_svd: a (m x n) = u (m x k) diag(s) vt
 * (k x n), k = min(m,n), s descending; sweeps = Jacobi sweeps taken.
 * sps_la_qr: a (m x n) = q (m x k) r (k x n).  ms = device time. */
int sps_la_svd(sps_handle* h, int32_t m, int32_t n, const double* a, double* u, double* s, double* vt,
               int32_t* sweeps, double* ms);
int sps_la_qr(sps_handle* h, int32_t m, int32_t n, const double* a, double* q, double* r, double* ms);
/* Left singular vectors and values only (the U-only Jacobi of the truncated
 * boundary SVD), m >= n: a = u diag(s) v^T, u (m x n), s (n). */
int sps_la_svd_left(sps_handle* h, int32_t m, int32_t n, const double* a, double* u, double* s, int32_t* sweeps,
                    double* ms);
/* Dense FP64 GEMM of the factorizations: c = alpha op(a) b + beta c, all
 * column-major; op(a) = a (m x k, ld m) or a^T (a is k x m, ld k); b k x n
 * (ld k); c m x n (ld m). */
int sps_la_gemm(sps_handle* h, int32_t transpose_a, int32_t m, int32_t n, int32_t k, double alpha, const double* a,
                const double* b, double beta, double* c, double* ms);
/* No counterpart in the reference.  The low-precision contraction GEMM on
 * the tcgen05 tensor cores (the kernel behind sps_set_precision), on dense
 * row-major host matrices: c (m x n) = a (m x k) b (k x n) with operands
 * rounded to TF32 (mode 1) or split into two TF32 (2) or two BF16 (3) parts,
 * FP32 accumulation, FP64 result; ms = device time of pack + GEMM. */
int sps_la_gemm_mixed(sps_handle* h, int32_t mode, int32_t m, int32_t n, int32_t k, const double* a,
                      const double* b, double* c, double* ms);
/* No counterpart in the reference.  Caps the cooperative launches of the
 * handle's own (serial) path at `ctas` CTAs each, 0 = the whole GPU: for a
 * handle that shares its GPU with other work.  sps_set_concurrency sets the
 * caps of the concurrent samples' engines. */
int sps_set_sm_share(sps_handle* h, int32_t ctas);
/* Leading k singular triplets by block subspace iteration with Rayleigh-Ritz
 * extraction (the truncated boundary SVD when no entropy is recorded):
 * u (m x k), s (k, descending), v (n x k), column-major; iterations = the
 * count used.  gram != 0 iterates on a a^T (the zip-up splits' mode; the
 * extraction and the residual test still use a); when the spectrum decays
 * too fast for a a^T to keep the wanted directions above its rounding level,
 * the call iterates on a instead.  rtol: the residual bound relative to s[0]
 * (0 selects 5e-14).  SPS_ERR_CONVERGENCE when the residuals did not reach it
 * within the iteration cap, or when a has fewer than k singular values above
 * its rounding level. */
int sps_la_svd_topk(sps_handle* h, int32_t m, int32_t n, int32_t k, const double* a, int32_t gram, double rtol,
                    double* u, double* s, double* v, int32_t* iterations, double* ms);

/* No counterpart in the reference.  The one-sided Jacobi SVD of one small
 * matrix for callers that cannot allocate device memory (no cudaMalloc /
 * cudaFree / allocating library call is made): a (m x n), u (m x k),
 * s (k) and vt (k x n) are column-major DEVICE buffers of the caller,
 * k = min(m,n), a = u diag(s) vt with s descending; u and vt stay
 * orthonormal where singular values are zero (completed to an orthonormal
 * set).  NaN or Inf input returns SPS_ERR_NUMERIC.  All scratch is one
 * fixed file-scope device array (max(m,n) <= 256, min(m,n) <= 128; larger
 * sizes return SPS_ERR_ARGUMENT) shared by every call on the device: calls
 * whose kernels overlap on the GPU race, so serialise them.  The first call
 * on a device looks up the array's device address; make it before any
 * stream capture.  Runs on `stream` (a cudaStream_t, NULL = default) and
 * synchronizes it before returning; SPS_ERR_CONVERGENCE if Jacobi did not
 * converge. */
int sps_la_svd_noalloc(int32_t device, void* stream, int32_t m, int32_t n, const double* a, double* u,
                       double* s, double* vt);

/* --- states: FiniteState (src/states/finite.jl:27-49) ---------------------
 * Site tensors have legs (W,N,Pout,Paux,E,S); each leg is described by its
 * even and odd multiplicities (n0,n1), even states first.  leg_dims holds
 * Lx*Ly*6*2 int32 in site order x + y*Lx; data holds every site's dense
 * row-major block back to back in the same order. */
int sps_identity_pepo(sps_handle* h, int32_t* state_id);           /* identity_pepo, finite.jl:80-86 */
int sps_state_upload(sps_handle* h, int32_t is_pepo, double beta, double log_amplitude,
                     const int32_t* leg_dims, const double* data, int32_t* state_id);
int sps_state_layout(sps_handle* h, int32_t state_id, int32_t* leg_dims, int64_t* total);
int sps_state_download(sps_handle* h, int32_t state_id, double* data, int64_t capacity);
int sps_state_info(sps_handle* h, int32_t state_id, double* beta, double* log_amplitude, int32_t* is_pepo);
int sps_state_set_beta(sps_handle* h, int32_t state_id, double beta);
int sps_state_copy(sps_handle* h, int32_t state_id, int32_t* new_id);           /* Base.copy, finite.jl:41 */
int sps_state_free(sps_handle* h, int32_t state_id);
int sps_normalize_state(sps_handle* h, int32_t state_id, double* log_normalizations); /* finite.jl:89-100 */

/* --- hot path -------------------------------------------------------------- */
/* evolution_step!(state, model, delta, D, FullUpdate, BoundaryMPS; order,
 * sector_space) (src/evolution/full_update.jl:559-597).  space: bond sector
 * budget (n0,n1) or NULL. */
int sps_evolution_step(sps_handle* h, int32_t state_id, double delta, int32_t D, const int32_t* space,
                       const sps_boundary* environment, sps_step_report* report);
/* lognorm(state, BoundaryMPS) (src/contraction/boundary_mps.jl:180-186) */
int sps_lognorm(sps_handle* h, int32_t state_id, const sps_boundary* method, sps_lognorm_result* out);
/* measure_energy(state, model, BoundaryMPS; record_entropy)
 * (src/measurement/energy.jl:31-78; the diagonal method
 * src/measurement/diagonal_energy.jl:12-45).  site_x (Lx*Ly), se_north /
 * se_south (the Se profile: (Ly-1)*(Lx-1) for the row methods; for the
 * diagonal one the northwest / southeast per-site profiles, Lx*Ly each,
 * index x + y*Lx) may be NULL. */
int sps_measure_energy(sps_handle* h, int32_t state_id, const sps_boundary* method, sps_energy* out,
                       double* site_x, double* se_north, double* se_south);
/* SamplingCache(state, BoundaryMPS; kind=:auxiliary) (src/sampling/born.jl:56-73) */
int sps_sampling_cache(sps_handle* h, int32_t pepo_id, const sps_boundary* method, int32_t* cache_id);
/* SamplingCache(state, BoundaryMPS; kind) (src/sampling/born.jl:56-73):
 * kind 0 = :auxiliary (state a PEPO; the same as sps_sampling_cache), 1 =
 * :physical (state a PEPS, e.g. a projected and evolved sample: the Born
 * proposal of annealed resampling over physical labels 1 (even) / 2 (odd),
 * conditionals from the PSD-projected site holes, born.jl:117-134, and
 * configurations restricted to the PEPS's total parity). */
int sps_sampling_cache_kind(sps_handle* h, int32_t state_id, const sps_boundary* method, int32_t kind,
                            int32_t* cache_id);
int sps_sampling_cache_free(sps_handle* h, int32_t cache_id);
/* sample_configuration(cache; rng) with the Lx*Ly uniforms in place of
 * rand(rng) (src/sampling/born.jl:86-163, src/sampling/diagonal_born.jl:24-97):
 * uniforms[i] is consumed by the i-th site drawn, row-major for the row
 * methods, by anti-diagonals for the diagonal one (x + y = 0, 1, ...; even
 * diagonals by increasing x, odd ones by decreasing x).  configuration
 * receives SymmetryBasis labels 1 (even) / 2 (odd), index x + y*Lx. */
int sps_sample(sps_handle* h, int32_t cache_id, const double* uniforms, int32_t* configuration,
               sps_sample_report* report);
/* sample_configuration with the `conditionals` of its result (born.jl:95,
 * :146): the Lx*Ly conditional probabilities of the chosen labels in site
 * order x + y*Lx (0 past a zero-probability stop).  Draws from `uniforms`, or
 * evaluates `given` (labels) when it is not NULL. */
int sps_sample_conditionals(sps_handle* h, int32_t cache_id, const double* uniforms, const int32_t* given,
                            int32_t* configuration, double* conditionals, sps_sample_report* report);
/* sample_configuration(cache; configuration) : probability of a given draw */
int sps_sample_probability(sps_handle* h, int32_t cache_id, const int32_t* configuration,
                           sps_sample_report* report);
/* sample_configuration(cache; configuration) for n configurations (n x
 * Lx*Ly labels): the scores of a resampling event (_score_configurations!,
 * src/resample/scores.jl:38-71) in one call, spread over the concurrent
 * samples like sps_sample_batch; reports may be NULL. */
int sps_sample_probability_batch(sps_handle* h, int32_t cache_id, int32_t n, const int32_t* configurations,
                                 double* log_probabilities, sps_sample_report* reports);
/* No counterpart in the reference (its ensemble is spread over MPI ranks):
 * the number of samples sps_sample_batch draws at the same time, each on its
 * own CUDA stream and device workspace, sharing the read-only SamplingCache
 * (1..16, default 1).  Each concurrent sample's cooperative launches use at
 * most 1/samples of the SMs. */
int sps_set_concurrency(sps_handle* h, int32_t samples);
/* No counterpart in the reference (it computes in Float64 throughout,
 * src/states/finite.jl:80): the arithmetic of the large contraction GEMMs --
 * row absorptions, row and slab steps, reduced metrics
 * (boundary_mps.jl:136-151, :216-246; full_update.jl:151-172).
 * mode 0 = FP64 (default); 1 = TF32, 2 = 3xTF32 (split operands, three
 * products), 3 = 3xBF16 (split operands, three products), all three on the
 * tcgen05 tensor cores with FP32 accumulation.  QR/SVD truncations, gauge
 * and normalisation scales, log-weights and Born probability
 * normalisations stay FP64 in every mode. */
int sps_set_precision(sps_handle* h, int32_t mode);
/* No counterpart in the reference.  enable != 0: launch shapes (the split-K
 * slice count of the table-driven contraction, the tile width of the tcgen05
 * GEMM) are picked by timing the candidates on the first call with a new
 * shape; the choice is kept for the process and shared by every handle on the
 * device.  Off by default (a choice changes the order of floating-point sums,
 * so a tuned run can differ from an untuned one at rounding level).
 * sps_autotune_report writes the table as JSON (key -> choice and the
 * candidates' milliseconds). */
int sps_set_autotune(sps_handle* h, int32_t enable);
int sps_autotune_report(sps_handle* h, char* buf, size_t n);
/* No counterpart in the reference (MatrixAlgebraKit computes every truncated
 * SVD from the full spectrum).  method 0 (default): truncated SVDs that keep
 * a few vectors of a large block take the subspace iteration when no entropy
 * is recorded; method 1: every truncated SVD from the full spectrum (the
 * one-sided Jacobi path), slower, for comparisons with a full-spectrum SVD. */
int sps_set_truncated_svd(sps_handle* h, int32_t method);
/* Per-site transverse fields h_i (index x + y*Lx), an extension of the
 * reference's uniform TFIM (src/models/tfim.jl:9-19: one h).  With fields
 * set, the Trotter bond gates split each site's h_i over its bonds as the
 * uniform gate splits h (src/models/tfim.jl:44-48), the 1x1 gate uses
 * h_0, and sps_measure_energy's total is -J sum ZZ - sum_i h_i <X_i>.
 * n = Lx*Ly sets them; n = 0 clears them (cfg.h everywhere again). */
int sps_set_site_fields(sps_handle* h, int32_t n, const double* fields);
/* The sweep options of BoundaryMPSRowVariational (row_variational.jl:10-25)
 * for the handle's later calls with absorption 3: max_sweep >= 1 round trips,
 * threshold_sweep >= 0 on the relative change of the squared norm (0 runs
 * every sweep).  Defaults 4 and 1e-8. */
int sps_set_variational(sps_handle* h, int32_t max_sweep, double threshold_sweep);
/* No counterpart in the reference (it has no derivatives).  lognorm with the
 * row method's exact compression (src/contraction/boundary_mps.jl:180-186)
 * and its derivative with respect to every site tensor by reverse mode
 * (QR-free: the canonical sweep by full SVDs, a gauge choice; the SVD reverse
 * rule per parity block with Lorentzian broadening).  checkpoint_rows != 0
 * keeps only each row's incoming boundary and recomputes the row's
 * factorizations in the reverse pass (memory of one row's tape instead of
 * all rows').  grads receives the derivatives in the layout of
 * sps_state_download (sites x + y*Lx, each row-major); capacity is its
 * length in doubles. */
int sps_lognorm_gradient(sps_handle* h, int32_t state_id, const sps_boundary* method, int32_t checkpoint_rows,
                         double* log_norm, double* grads, int64_t capacity);
/* No counterpart in the reference.  The per-site field derivatives from one
 * reverse pass of sps_lognorm_gradient: site_x[i] = <X_i> = half the
 * derivative of lnZ along A_i -> A_i + e X A_i (X = diag(1, -1) on the
 * physical leg), and d_fields[i] = d lnZ / dh_i = beta <X_i> for the thermal
 * state exp(-beta H) the PEPO represents at its beta (the reference's direct
 * route to the same numbers is one ratio per site, measure_energy's
 * energy.jl:43-46).  site_x and d_fields hold Lx*Ly values (x + y*Lx). */
int sps_lognorm_field_gradient(sps_handle* h, int32_t state_id, const sps_boundary* method, int32_t checkpoint_rows,
                               double* log_norm, double* site_x, double* d_fields);
/* lognorm with the fit summary of a variational method
 * (row_variational.jl:331-339, _variational_summary): counts = {layers,
 * max_sweeps, sweep_limit_hits, fallback_count}; max_relative_change. */
int sps_lognorm_variational(sps_handle* h, int32_t state_id, const sps_boundary* method, sps_lognorm_result* out,
                            int32_t* counts, double* max_relative_change);
/* No counterpart in the reference: host-side failure injection for tests
 * (nothing faults on the device; the library takes its ordinary error
 * paths).  force_repair != 0 treats every full-update bond fit as triggered,
 * so update_bond! takes its PSD-repair branch (src/evolution/full_update.jl:
 * 490-501) on well-conditioned input; svd_sweep_cap > 0 caps the sweeps of
 * the single-CTA Jacobi SVD and eigh kernels, which then report
 * SPS_ERR_CONVERGENCE (the non-convergence status of _retry_svd,
 * src/states/svd.jl:2-33); 0 restores the default cap of 80.
 * multi_cta_eigh_min > 0: parity blocks of the PSD repair's eigendecomposition
 * with at least that many rows take the multi-CTA route (one-sided Jacobi of
 * the shifted hole); 0 restores the default of 1024. */
int sps_set_injection(sps_handle* h, int32_t force_repair, int32_t svd_sweep_cap, int32_t multi_cta_eigh_min);
/* n draws in one call (the MPI sample loop of src/driver/run.jl:45-49 on one device);
 * reports (n) may be NULL. */
int sps_sample_batch(sps_handle* h, int32_t cache_id, int32_t n, const double* uniforms,
                     int32_t* configurations, double* log_probabilities, sps_sample_report* reports);
/* project_configuration(checkpoint, configuration) (src/sampling/born.jl:27-36) */
int sps_project(sps_handle* h, int32_t pepo_id, const int32_t* configuration, int32_t* state_id,
                double* log_normalizations);

/* --- batched variants -------------------------------------------------------
 * One call over n samples, in place of the reference's per-particle loops
 * (src/driver/run.jl:52-57 projection + observation of the unique
 * configurations, :104-108 _advance_particle! per node).  Up to the
 * sps_set_concurrency count run at the same time, each on its own CUDA
 * stream and workspace; results are those of the single-sample calls.  Each
 * state id may appear once per call.  On error the first failing sample's
 * status is returned (the others have completed). */
/* n x project_configuration: configurations (n x Lx*Ly labels), state_ids (n)
 * receive new PEPS states, log_normalizations (n x Lx*Ly) may be NULL. */
int sps_project_batch(sps_handle* h, int32_t pepo_id, int32_t n, const int32_t* configurations,
                      int32_t* state_ids, double* log_normalizations);
/* n x evolution_step! (full_update.jl:559-597) with per-state delta; reports (n) may be NULL. */
int sps_evolution_step_batch(sps_handle* h, int32_t n, const int32_t* state_ids, const double* deltas, int32_t D,
                             const int32_t* space, const sps_boundary* environment, sps_step_report* reports);
/* n x measure_energy (energy.jl:31-78): out (n), site_x (n x Lx*Ly, may be NULL). */
int sps_measure_energy_batch(sps_handle* h, int32_t n, const int32_t* state_ids, const sps_boundary* method,
                             sps_energy* out, double* site_x);
/* n x lognorm (boundary_mps.jl:180-186), the observation at nodes without an energy measurement
 * (src/driver/particles.jl:35-40). */
int sps_lognorm_batch(sps_handle* h, int32_t n, const int32_t* state_ids, const sps_boundary* method,
                      sps_lognorm_result* out);

#ifdef __cplusplus
}
#endif
#endif
