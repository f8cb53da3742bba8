// The sample-ensemble hot path on the Z2 engine: row boundary-MPS
// contraction, full update, Born sampling and energy measurement.  Each
// function restates the reference function named beside it.
#pragma once
#include "engine.h"
#include <array>
#include <functional>
#include <cmath>

namespace sps {

struct Model {
  double J = 1.0, h = 0.7;
  // per-site transverse fields (x + y*Lx), an extension for per-site
  // gradients (the reference's TFIM has one h); empty: h everywhere
  std::vector<double> fields;
  double field(int x, int y, int Lx) const { return fields.empty() ? h : fields[x + y * Lx]; }
};

struct FUOptions {   // FullUpdate (src/evolution/full_update.jl:11-17)
  int max_iterations = 4;
  double error_tolerance = 1e-8;
  double diagonal_shift = 1e-10;
  int linear_max_iterations = 24;
  double linear_tolerance = 1e-9;
};

struct BMPS {        // BoundaryMPS (src/contraction/boundary_mps.jl:11-18)
  int chi = 32;
  int space[2] = {-1, -1};
  bool zipup = false;   // zip-up row absorption (this engine's variant) instead of the exact compression
  // BoundaryMPSDiagonal (src/contraction/diagonal_mps.jl:3-9): anti-diagonal
  // layers instead of rows, same chi and sector budget
  bool diagonal = false;
  // BoundaryMPSRowVariational (src/contraction/row_variational.jl:10-25): rows
  // absorbed by a two-site variational fit
  bool variational = false;
  int max_sweep = 4;
  double threshold_sweep = 1e-8;
};

// one absorption of the row variational method (the records that
// _variational_summary collects, diagonal_variational.jl:40-46)
struct VariationalRecord {
  enum { DIRECT = 0, ZERO_TARGET = 1, SWEEP_LIMIT = 2, THRESHOLD_SWEEP = 3, NUMERICAL_FALLBACK = 4 };
  int layer = 0;
  bool reverse = false;
  int sweeps = 0;
  double relative_change = 0;
  int stop_reason = DIRECT;
  double max_local_discarded_weight = 0;
  bool fallback = false;
  std::string fallback_reason;
  double initial_residual = 0, residual = 0;   // diagonal method: |C - T|^2 before and after the fit
  bool used_svd = false;                      // diagonal method: the fallback took the SVD absorption
};

struct State {       // FiniteState (src/states/finite.jl:27-49)
  int Lx = 0, Ly = 0;
  std::vector<Tensor> sites;   // x + y*Lx, legs (W,N,Pout,Paux,E,S)
  double beta = 0, log_amplitude = 0;
  bool pepo = true;
  Tensor& at(int x, int y) { return sites[x + y * Lx]; }
  const Tensor& at(int x, int y) const { return sites[x + y * Lx]; }
};

struct Env {         // BoundaryEnvironment (boundary_mps.jl:79-83)
  std::vector<Tensor> t;
  double log_scale = 0, max_trunc = 0;
  // the row variational method's canonical centre and fit records
  // (RowVariationalBoundary, row_variational.jl:37-43)
  int center = 0;
  std::vector<VariationalRecord> variational;
};

struct Entropy {     // BoundaryEntropy (boundary_mps.jl:44-57)
  double maximum = 0;
  bool profile = false;
  int Lx = 0, Ly = 0;
  std::vector<double> north, south;   // (Ly-1) x (Lx-1), row-major [row][bond]
  // diagonal method (diagonal_mps.jl:143-157): per site x + y*Lx, the entropy
  // of the bond its block split opened, for each sweep direction
  std::vector<double> northwest, southeast;
  void record(bool south_side, int row, int bond, double v) {
    maximum = std::max(maximum, v);
    if (profile && row >= 1 && row <= Ly - 1) (south_side ? south : north)[(row - 1) * (Lx - 1) + bond - 1] = v;
  }
};

struct DiagEnv {     // DiagonalBoundary (diagonal_mps.jl:106-118)
  std::vector<Tensor> t;      // (l, edge, r) per frontier edge, in frontier order
  std::vector<int> edges;     // the frontier's edge labels
  double log_scale = 0, max_trunc = 0;
  double scalar = 1;          // the closed network after the last layer
  int center = 0;             // the canonical centre
  std::vector<VariationalRecord> variational;   // fit records of the diagonal variational method
};

struct Layer {       // a row entry: plain double layer or SlabColumn (boundary_mps.jl:212-215)
  Tensor a, b;
  bool slab = false;
  // when set, `a` is double_layer(ket, ket) of the single-layer `ket` (legs
  // W,N,P,Aux,E,S) and the row steps contract ket and bra one after the other
  Tensor ket;
  bool layered = false;
};

// contraction
Tensor unit_tensor(Engine& E, const std::vector<Par>& legs);
Tensor double_layer(Engine& E, const Tensor& ket, const Tensor& bra, const Tensor* physical = nullptr);
std::vector<Tensor> row_layers(Engine& E, const State& s);
Env trivial_boundary(Engine& E, const std::vector<Tensor>& row, bool north);
struct CompressReport { double max_trunc, log_scale; };
CompressReport compress_boundary(Engine& E, std::vector<Tensor>& B, const BMPS& m, bool reverse,
                                 Entropy* ent, bool south_side, int row_cut);
// kets: optional single layers of the row (row[x] = double_layer(kets[x], kets[x])),
// used by the zip-up absorption to contract ket and bra one after the other
Env absorb(Engine& E, const Env& env, const std::vector<Tensor>& row, const BMPS& m, bool north,
           Entropy* ent = nullptr, int row_cut = 0, const std::vector<Tensor>* kets = nullptr);
double close_boundary(Engine& E, const std::vector<Tensor>& B);
struct LogNorm {
  double log_norm, tensor_log_norm, max_env_trunc;
  std::vector<VariationalRecord> variational;
};
// _absorb for BoundaryMPSRowVariational (variational.cu; row_variational.jl:306-329)
Env absorb_variational(Engine& E, const Env& env, const std::vector<Tensor>& row, const BMPS& m, bool north,
                       Entropy* ent, int row_cut);
LogNorm lognorm(Engine& E, const State& s, const BMPS& m);
struct Envs { std::vector<Env> north, south; double max_trunc = 0; };
Envs boundary_environments(Engine& E, const std::vector<Tensor>& layers, int Lx, int Ly, const BMPS& m,
                           int side /*0 both,1 north,2 south*/, Entropy* ent);
// X (w, b, n, c) times double_layer(ket, ket) over (w, n) -> (b, c, e, s), ket then bra
Tensor layer_apply_wn(Engine& E, const Tensor& X, const Tensor& ket);
// the two steps of layer_apply_wn in one kernel (layered.cu): X5 (x, y, b, u, v, c)
// and ket (x, u, p, a, e, f) to Z (b, c, e, g, f, h); false when its tiles do not
// fit in shared memory (Z untouched)
bool layer_wn_fused(Engine& E, const Tensor& X5, const Tensor& ket, Tensor& Z);
Tensor left_step(Engine& E, const Tensor& L, const Tensor& T, const Layer& row, const Tensor& B);
Tensor right_step(Engine& E, const Tensor& T, const Layer& row, const Tensor& B, const Tensor& R);
Tensor row_edge(Engine& E, const std::vector<Tensor>& top, const std::vector<Layer>& row,
                const std::vector<Tensor>& bottom, bool left);
struct RowEnvs { std::vector<Tensor> left, right; };
RowEnvs row_environments(Engine& E, const std::vector<Tensor>& top, const std::vector<Layer>& row,
                         const std::vector<Tensor>& bottom, int side /*0 both,1 left,2 right*/);
// full contraction of a row position; result accumulated into device slot
void row_scalar_to(Engine& E, const Tensor& L, const Tensor& T, const Layer& row, const Tensor& B,
                   const Tensor& R, int slot);

// full update
struct BondReport {
  double initial_cost = 0, final_cost = 0, residual = 0;
  int iterations = 0;
  bool iteration_limit_reached = false;
  int stop_reason = 0;   // 0 error_tolerance, 1 iteration_limit, 2 residual_fallback, 3 disabled
  int repairs = 0;
  int fallbacks = 0;
  double max_env_trunc = 0;
};
struct StepReport {
  double beta = 0;
  std::vector<double> log_normalizations;
  int bond_updates = 0, iteration_limit_hits = 0;
  double max_state_truncation = 0, max_environment_truncation = 0, max_boundary_entropy = NAN;
  double max_solver_residual = 0, max_iteration_limit_error = 0;
  int stop_reasons[4] = {0, 0, 0, 0};
  int repairs = 0, fallbacks = 0, linear_unconverged = 0;
};
Tensor trotter_gate(Engine& E, const Model& m, int Lx, int Ly, int ax, int ay, int bx, int by, double delta);
// a bond environment as update_bond! uses it: the reduced metric N[rb, sb, rk, sk]
// of the reduced pair's Q factors, and the bond hole (six exterior legs, each
// split (ket, bra)) for the PSD repair
struct PairEnv {
  std::function<Tensor(const Tensor& Qa, const Tensor& Qb)> metric;
  std::function<Tensor()> hole;
  bool horizontal = true;
};
// update_bond! (src/evolution/full_update.jl:484-508)
BondReport update_bond_env(Engine& E, State& s, int ix, int iy, int jx, int jy, const Tensor& gate, int D,
                           const FUOptions& o, const PairEnv& env, const int space[2], bool force_repair);
void record_bond(StepReport& rep, const BondReport& br, const FUOptions& o);
// _sweep! on diagonal boundaries (src/evolution/diagonal_update.jl:61-102)
void sweep_diagonal(Engine& E, State& s, const Model& m, double delta, int D, const FUOptions& o,
                    const BMPS& method, bool horizontal, bool reverse, const int space[2], Entropy* ent,
                    StepReport& rep, double& env_err, bool force_repair);
StepReport evolution_step(Engine& E, State& s, const Model& m, double delta, int D, const FUOptions& o,
                          const BMPS& env_method, int order, const int space[2], bool record_entropy,
                          bool force_repair = false);
std::vector<double> normalize_state(Engine& E, State& s);

// sampling
enum SamplingKind : int { KIND_AUXILIARY = 0, KIND_PHYSICAL = 1 };
struct SamplingCache {
  int Lx, Ly;
  int kind = KIND_AUXILIARY;   // the leg the draw labels: auxiliary (PEPO) or physical (PEPS proposal)
  int target = -1;             // physical kind: the PEPS's total parity, which a configuration must fuse to
  std::vector<Tensor> layers;
  std::vector<std::array<Tensor, 2>> candidates;
  std::vector<std::array<Tensor, 2>> candidate_kets;   // the projected single layers of the candidates
  std::vector<Env> south;
  std::vector<DiagEnv> southeast;   // diagonal method: se[t] holds the layers from t on
  BMPS method;
  const State* state_ref = nullptr;
};
SamplingCache make_sampling_cache(Engine& E, const State& s, const BMPS& m, int kind = KIND_AUXILIARY);
struct SampleResult {
  std::vector<int> config;   // labels 1/2, index x + y*Lx
  double log_probability = 0;
  double max_env_trunc = 0;
  std::vector<double> conditionals;
  int near_boundary = 0;     // draws within 1e-12 of a cumulative boundary
  // physical kind: the PSD projections of the site metrics (born.jl:119-121)
  int metric_repairs = 0;              // site metrics with negative eigenvalues clipped
  double min_relative_eigenvalue = 0;  // the smallest eigenvalue / spectral scale over the sites
  int zero_proposals = 0;              // sites whose allowed outcomes all had zero weight
};
SampleResult sample_configuration(Engine& E, const SamplingCache& c, const double* uniforms,
                                  const int* configuration);
State project_configuration(Engine& E, const State& pepo, const int* configuration,
                            std::vector<double>* log_norms);

// measurement
struct EnergyResult {
  double energy_total, energy_per_site, log_norm, tensor_log_norm, max_env_trunc;
  double x_sum, zz_sum;
  std::vector<double> site_x;
  Entropy entropy;
};
EnergyResult measure_energy(Engine& E, const State& s, const Model& m, const BMPS& method,
                            bool record_entropy);

State identity_pepo(Engine& E, int Lx, int Ly);

// helpers shared by the row and diagonal methods (boundary.cu)
double positive_real(double z, const char* name);
Tensor project_aux(Engine& E, const Tensor& A, int k);
Tensor project_physical(Engine& E, const Tensor& A, int k);
int categorical(const std::vector<double>& lm, double u, int* near);
// _positive_metric(H; square_root=true) of a site hole H with legs
// (wk, wb, nk, nb, ek, eb, sk, sb): the eigenvectors on the ket legs scaled by
// the square roots of the clipped eigenvalues, legs (w, n, e, s, z)
Tensor metric_root(Engine& E, const Tensor& H, SampleResult& res);
void operator_factors(Engine& E, Tensor& F, Tensor& G);
void operator_pair(Engine& E, const Tensor& A, const Tensor& B, const Tensor& F, const Tensor& G, bool horizontal,
                   Tensor& C, Tensor& D);
double real_ratio(double a, double b);

// reverse-mode derivative of the row lognorm with respect to the site
// tensors (adjoint.cu; exact compression only)
struct LognormGradient {
  double log_norm = 0;
  std::vector<Tensor> grads;   // per site x + y*Lx, legs of the site tensor
};
LognormGradient lognorm_gradient(Engine& E, const State& s, const BMPS& m, bool checkpoint_rows = false);
// per-site <X_i> from one reverse pass (the derivative along X insertions)
// and d lnZ/dh_i = beta <X_i> of the thermal state the PEPO represents
struct FieldGradient {
  double log_norm = 0;
  std::vector<double> site_x, d_fields;
};
FieldGradient lognorm_field_gradient(Engine& E, const State& s, const BMPS& m, bool checkpoint_rows = false);

// diagonal boundary MPS (diagonal.cu; src/contraction/diagonal_mps.jl,
// src/sampling/diagonal_born.jl, src/measurement/diagonal_energy.jl)
LogNorm lognorm_diagonal(Engine& E, const State& s, const BMPS& m);
void diagonal_southeast(Engine& E, const State& s, const BMPS& m, std::vector<DiagEnv>& se);
SampleResult sample_diagonal(Engine& E, const SamplingCache& c, const double* uniforms, const int* configuration);
EnergyResult measure_energy_diagonal(Engine& E, const State& s, const Model& m, const BMPS& method,
                                     bool record_entropy);
// the order in which a diagonal draw visits the sites (x + y*Lx), _diagonal_order
std::vector<int> diagonal_draw_order(int Lx, int Ly);

}  // namespace sps
