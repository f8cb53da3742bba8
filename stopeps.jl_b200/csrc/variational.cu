// Row variational boundary MPS on the Z2 engine (BoundaryMPSRowVariational):
// restates src/contraction/row_variational.jl with the helpers it takes from
// src/contraction/diagonal_variational.jl (_VariationalNumericalError,
// _variational_message, _variational_identity, _variational_space_map).
//
// A row is absorbed by a two-site variational fit of the truncated candidate
// MPS C to the target T = (input boundary) x (row): C starts from the input
// boundary with its physical legs mapped onto the row's output legs; each
// two-site update is the normalised projection of T onto C's environment,
// split by a truncated SVD; sweeps (left to right, then back) stop at
// max_sweep or when the squared norm changes by at most threshold_sweep.
// C's amplitude stays in a log scale and the best admissible candidate is
// kept.  Row sites are fused double layers (w, n, e, s), the tensors the
// reference's FactorizedRowSite stands for, so only the absorption differs
// from the row method.
#include "pipeline.h"
#include <algorithm>
#include <cfloat>

namespace sps {
namespace {

struct VarFail : Error {   // _VariationalNumericalError
  std::string reason;
  explicit VarFail(const std::string& r) : Error(SPS_ERR_NUMERIC, "variational boundary: " + r), reason(r) {}
};

struct Msg {   // _VariationalMessage: a normalised tensor and its log scale
  Tensor t;
  double log_scale = 0;
};

Msg message(Engine& E, Tensor t, double log_scale = 0.0) {
  t = contiguous(E, t);
  const double s = norm(E, t);
  if (!std::isfinite(s)) throw VarFail("nonfinite_overlap");
  if (s == 0) return {t, -INFINITY};
  scale_inplace(E, t, 1.0 / s);
  return {t, log_scale + std::log(s)};
}

// _variational_identity: the normalised identity of a single-layer leg of d
// states as a vector on its fused (ket, bra) leg
Tensor identity_vector(Engine& E, const Par& p) {
  const int dd = (int)p->size(), d = (int)std::lround(std::sqrt((double)dd));
  std::vector<double> v(dd, 0.0);
  for (int k = 0; k < d; ++k) v[k * d + k] = 1.0 / std::sqrt((double)d);
  return E.upload({p}, v.data());
}

// _variational_space_map (diagonal_variational.jl:232-237): Q <- P, the
// identity on the first min(P_c, Q_c) states of each parity c
Tensor space_map(Engine& E, const Par& Q, const Par& P) {
  const int nq = (int)Q->size(), np = (int)P->size();
  std::vector<double> m((size_t)nq * np, 0.0);
  for (int c = 0; c < 2; ++c) {
    std::vector<int> qi, pi;
    for (int i = 0; i < nq; ++i)
      if ((*Q)[i] == c) qi.push_back(i);
    for (int i = 0; i < np; ++i)
      if ((*P)[i] == c) pi.push_back(i);
    for (size_t k = 0; k < std::min(qi.size(), pi.size()); ++k) m[(size_t)qi[k] * np + pi[k]] = 1.0;
  }
  return E.upload({Q, P}, m.data());
}

// _RowLayerTarget (row_variational.jl:53-77)
struct Target {
  Engine& E;
  const Env& input;
  std::vector<Tensor> row;   // double layers divided by |ket| |bra|
  bool north;
  double log_scale;
  double reference = NAN;
  bool zero;
  int out;                   // the output leg of a double layer (s north, n south)

  Target(Engine& e, const Env& env, const std::vector<Tensor>& r, bool n)
      : E(e), input(env), north(n), log_scale(env.log_scale), zero(env.log_scale == -INFINITY), out(n ? 3 : 1) {
    if (env.t.size() != r.size()) throw Error(SPS_ERR_ARGUMENT, "row boundary length");
    for (const Tensor& L : r) {
      // |ket| |bra| of a ket = bra layer: its trace over every (ket, bra) pair
      Tensor x = ein(E, "a,abcd->bcd", identity_vector(E, L.legs[0]), L);
      x = ein(E, "b,bcd->cd", identity_vector(E, L.legs[1]), x);
      x = ein(E, "c,cd->d", identity_vector(E, L.legs[2]), x);
      double ab = dot(E, identity_vector(E, L.legs[3]), x);
      // each identity vector carries 1/sqrt(d): undo that
      for (int k = 0; k < 4; ++k) ab *= std::sqrt(std::sqrt((double)L.legs[k]->size()));
      if (!std::isfinite(ab)) throw VarFail("nonfinite_target");
      if (ab <= 0) {
        zero = true;
        row.push_back(L);
      } else {
        Tensor c = clone(E, L);
        scale_inplace(E, c, 1.0 / ab);
        row.push_back(c);
        log_scale += std::log(ab);
      }
    }
  }

  // _row_half_projection: (cand, out, input bond, horizontal) after the input
  // tensor and row site i, entering from the left (msg (c, a, w)) or the right
  // (msg (c, b, e))
  Msg half(const Msg& m, int i, bool left) const {
    const Tensor& B = input.t[i];
    Tensor X = left ? ein(E, "caw,apb->cwpb", m.t, B) : ein(E, "cbe,apb->ceap", m.t, B);
    Tensor Y;
    if (left) Y = ein(E, north ? "cwpb,wpeo->cobe" : "cwpb,woep->cobe", X, row[i]);
    else Y = ein(E, north ? "ceap,wpeo->coaw" : "ceap,woep->coaw", X, row[i]);
    return message(E, Y, m.log_scale);
  }
  // _row_mixed_step: the half projection closed with the candidate
  Msg mixed_step(const Msg& m, int i, const Tensor& A, bool left) const {
    Msg h = half(m, i, left);
    return message(E, left ? ein(E, "cobe,coC->Cbe", h.t, A) : ein(E, "coaw,Coc->Caw", h.t, A), h.log_scale);
  }
  Msg edge(const std::vector<Tensor>& C, bool left) const {   // _row_mixed_edge
    const int i = left ? 0 : (int)row.size() - 1, a = left ? 0 : 2;
    return message(E, unit_tensor(E, {C[i].legs[a], input.t[i].legs[a], row[i].legs[left ? 0 : 2]}));
  }
  std::vector<Msg> messages(const std::vector<Tensor>& C, bool left) const {
    const int n = (int)C.size();
    std::vector<Msg> out(n + 1);
    if (left) {
      out[0] = edge(C, true);
      for (int i = 0; i < n; ++i) out[i + 1] = mixed_step(out[i], i, C[i], true);
    } else {
      out[n] = edge(C, false);
      for (int i = n - 1; i >= 0; --i) out[i] = mixed_step(out[i + 1], i, C[i], false);
    }
    return out;
  }
  // _row_project_pair: the normalised two-site projection (c, o, O, C)
  Msg project_pair(int i, const Msg& L, const Msg& R) const {
    Msg l = half(L, i, true), r = half(R, i + 1, false);
    Tensor theta = contiguous(E, ein(E, "cobe,CObe->coOC", l.t, r.t));
    const double s = norm(E, theta);
    if (!std::isfinite(s)) throw VarFail("nonfinite_projection");
    if (s == 0) throw VarFail("zero_local_projection");
    const double ln = l.log_scale + r.log_scale + std::log(s);
    if (!std::isfinite(ln)) throw VarFail("zero_local_projection");
    scale_inplace(E, theta, 1.0 / s);
    return {theta, ln};
  }
};

struct Candidate {
  std::vector<Tensor> t;
  int center = 0;
  double log_scale = 0, max_trunc = 0;
};

void move_center(Engine& E, Candidate& C, int target) {   // _diagonal_center!
  while (C.center < target) {
    const int i = C.center;
    QRres f = qr(E, C.t[i], {0, 1}, {2});
    C.t[i] = f.Q;
    C.t[i + 1] = ein(E, "lk,kpr->lpr", f.R, C.t[i + 1]);
    C.center++;
  }
  while (C.center > target) {
    const int i = C.center;
    LQres f = lq(E, C.t[i], {0}, {1, 2});
    C.t[i] = f.Q;
    C.t[i - 1] = ein(E, "lpk,kr->lpr", C.t[i - 1], f.L);
    C.center--;
  }
}

Candidate product(Engine& E, const Target& t) {   // _row_product
  Candidate C;
  Par triv = make_par(1, 0);
  for (const Tensor& L : t.row) {
    Tensor v = identity_vector(E, L.legs[t.out]);
    Tensor u = v;
    u.legs = {triv, v.legs[0], triv};
    u.dims = {1, v.dims[0], 1};
    u.strides = {v.dims[0], 1, 1};
    C.t.push_back(u);
  }
  return C;
}

Candidate warm_start(Engine& E, const Target& t) {   // _row_warm_start (row_variational.jl:100-117)
  Candidate C;
  C.t = t.input.t;
  C.center = t.input.center;
  for (int i = 0; i < (int)C.t.size(); ++i) {
    const Par& P = C.t[i].legs[1];
    const Par& Q = t.row[i].legs[t.out];
    if (*P == *Q) continue;
    bool projects = false;
    for (int c = 0; c < 2; ++c) projects |= par_count(P, c) > par_count(Q, c);
    if (projects) move_center(E, C, i);
    C.t[i] = ein(E, "qp,lpr->lqr", space_map(E, Q, P), C.t[i]);
  }
  move_center(E, C, 0);
  C.t[0] = contiguous(E, C.t[0]);
  const double s = norm(E, C.t[0]);
  if (!std::isfinite(s)) throw VarFail("nonfinite_initialization");
  if (s == 0) return product(E, t);
  C.t[0] = clone(E, C.t[0]);
  scale_inplace(E, C.t[0], 1.0 / s);
  return C;
}

bool allowed(const Candidate& C, const BMPS& m) {   // _row_candidate_allowed
  for (size_t i = 0; i + 1 < C.t.size(); ++i) {
    const Par& p = C.t[i].legs[2];
    if ((int)p->size() > m.chi) return false;
    if (m.space[0] >= 0 && (par_count(p, 0) > m.space[0] || par_count(p, 1) > m.space[1])) return false;
  }
  return true;
}

bool initialize_amplitude(Engine& E, Target& t, Candidate& C, const std::vector<Msg>& fixed) {
  const Msg& terminal = fixed[0];
  Msg edge = t.edge(C.t, true);
  const double z = dot(E, terminal.t, edge.t);
  if (!std::isfinite(z)) throw VarFail("nonfinite_overlap");
  if (z == 0 || terminal.log_scale == -INFINITY) {
    C.log_scale = -INFINITY;
    return false;
  }
  t.reference = std::log(std::fabs(z)) + terminal.log_scale + edge.log_scale;
  if (z < 0) {
    C.t[0] = clone(E, C.t[0]);
    scale_inplace(E, C.t[0], -1.0);
  }
  C.log_scale = 0;
  return true;
}

// _row_half_sweep! (row_variational.jl:197-233)
std::vector<Msg> half_sweep(Engine& E, Candidate& C, Target& t, const BMPS& m, bool right, Entropy* ent,
                            std::vector<double>& profile, const std::vector<Msg>& fixed) {
  const int n = (int)C.t.size();
  Msg rolling = t.edge(C.t, right);
  const bool bounded = allowed(C, m);
  std::vector<Msg> next(n + 1);
  next[right ? 0 : n] = rolling;
  Trunc tr;
  tr.chi = m.chi;
  tr.space[0] = m.space[0];
  tr.space[1] = m.space[1];
  for (int q = 0; q + 1 < n; ++q) {
    const int i = right ? q : n - 2 - q;
    const Msg& L = right ? rolling : fixed[i];
    const Msg& R = right ? fixed[i + 2] : rolling;
    Msg theta = t.project_pair(i, L, R);
    if (std::isnan(t.reference)) t.reference = theta.log_scale;
    SVDres f = svd(E, theta.t, {0, 1}, {2, 3}, tr, ent != nullptr);
    if (ent) ent->maximum = std::max(ent->maximum, f.entropy);
    double s2 = 0;
    for (int c = 0; c < 2; ++c)
      for (double v : f.S[c]) s2 += v * v;
    const double s = std::sqrt(s2);
    if (!(std::isfinite(s) && s > 0)) throw VarFail("zero_local_projection");
    const double newscale = theta.log_scale - t.reference + std::log(s);
    if (bounded && !(newscale >= C.log_scale - 512 * DBL_EPSILON * std::max(1.0, std::fabs(C.log_scale))))
      throw VarFail("objective_increase");
    std::vector<double> kept(f.S[0]);
    kept.insert(kept.end(), f.S[1].begin(), f.S[1].end());
    for (double& v : kept) v /= s;
    if (right) {
      C.t[i] = f.U;
      C.t[i + 1] = scale_leg(E, f.V, 0, kept);
    } else {
      C.t[i] = scale_leg(E, f.U, 2, kept);
      C.t[i + 1] = f.V;
    }
    C.center = right ? i + 1 : i;
    C.log_scale = newscale;
    profile[i] = ent ? f.entropy : NAN;
    C.max_trunc = std::max(C.max_trunc, f.err * f.err);
    const int k = right ? i : i + 1;
    rolling = t.mixed_step(rolling, k, C.t[k], right);
    next[right ? k + 1 : k] = rolling;
  }
  return next;
}

double relative_change(double a, double b) {   // _row_relative_change
  const double largest = std::max(a, b);
  return -std::expm1(-std::fabs(a - b)) * std::exp(largest - std::max(largest, std::log(DBL_MIN)));
}

}  // namespace

// _absorb for BoundaryMPSRowVariational (row_variational.jl:306-329)
Env absorb_variational(Engine& E, const Env& env, const std::vector<Tensor>& row, const BMPS& m, bool north,
                       Entropy* ent, int row_cut) {
  if (m.chi < 1) throw Error(SPS_ERR_ARGUMENT, "chi must be positive");
  if (m.max_sweep < 1) throw Error(SPS_ERR_ARGUMENT, "max_sweep must be positive");
  Target t(E, env, row, north);
  const int n = (int)row.size();
  std::vector<double> profile(std::max(0, n - 1), NAN);
  VariationalRecord rec;
  rec.layer = north ? row_cut : row_cut + 1;
  rec.reverse = !north;
  Candidate C;
  if (t.zero) {
    C = product(E, t);
    C.t[0] = clone(E, C.t[0]);
    scale_inplace(E, C.t[0], 0.0);
    C.log_scale = -INFINITY;
    t.reference = 0;
    rec.stop_reason = VariationalRecord::ZERO_TARGET;
  } else if (n == 1) {   // _row_direct (row_variational.jl:288-304)
    C = product(E, t);
    Msg h = t.half(t.edge(C.t, true), 0, true);   // (c, o, b, e), b and e trivial
    Tensor A = h.t;
    A.legs = {h.t.legs[0], h.t.legs[1], make_par(1, 0)};
    A.dims = {h.t.dims[0], h.t.dims[1], 1};
    A.strides = {h.t.strides[0], h.t.strides[1], 1};
    A = contiguous(E, A);
    const double s = norm(E, A);
    if (!std::isfinite(s)) throw VarFail("nonfinite_projection");
    if (s != 0) {
      A = clone(E, A);
      scale_inplace(E, A, 1.0 / s);
    }
    C.t[0] = A;
    C.log_scale = s == 0 ? -INFINITY : h.log_scale + std::log(s);
    t.reference = 0;
    rec.stop_reason = s == 0 ? VariationalRecord::ZERO_TARGET : VariationalRecord::DIRECT;
  } else {   // _row_variational_fit (row_variational.jl:240-286)
    C = warm_start(E, t);
    std::vector<Msg> fixed = t.messages(C.t, false);
    const bool valid = initialize_amplitude(E, t, C, fixed);
    bool have_best = valid && allowed(C, m);
    Candidate best = C;
    std::vector<double> bestprofile = profile;
    double previous = NAN, change = INFINITY, maxdiscard = 0;
    int reason = VariationalRecord::SWEEP_LIMIT, sweeps = 0;
    for (int sweep = 1; sweep <= m.max_sweep; ++sweep) {
      sweeps = sweep;
      std::string failure;
      try {
        for (bool right : {true, false}) {
          fixed = half_sweep(E, C, t, m, right, ent, profile, fixed);
          if (allowed(C, m) && (!have_best || C.log_scale >= best.log_scale)) {
            best = C;
            bestprofile = profile;
            have_best = true;
          }
        }
      } catch (const VarFail& ex) {
        failure = ex.reason;
      } catch (const Error& ex) {
        if (ex.code != SPS_ERR_CONVERGENCE) throw;
        failure = "factorization_failure";
      }
      if (!failure.empty()) {
        // recover from the last valid centre
        if (std::isfinite(C.log_scale) && allowed(C, m) && (!have_best || C.log_scale > best.log_scale)) {
          best = C;
          bestprofile = profile;
          have_best = true;
        }
        if (!have_best) throw Error(SPS_ERR_NUMERIC, "variational boundary: " + failure);
        rec.fallback = true;
        rec.fallback_reason = failure;
        reason = VariationalRecord::NUMERICAL_FALLBACK;
        maxdiscard = std::max(maxdiscard, C.max_trunc);
        break;
      }
      maxdiscard = std::max(maxdiscard, C.max_trunc);
      const double w = 2 * C.log_scale;
      change = sweep == 1 ? INFINITY : relative_change(w, previous);
      previous = w;
      if (sweep > 1 && m.threshold_sweep > 0 && change <= m.threshold_sweep) {
        reason = VariationalRecord::THRESHOLD_SWEEP;
        break;
      }
    }
    if (!have_best) throw Error(SPS_ERR_NUMERIC, "variational boundary: no_valid_candidate");
    C = best;
    profile = bestprofile;
    rec.sweeps = sweeps;
    rec.relative_change = change;
    rec.stop_reason = reason;
    rec.max_local_discarded_weight = maxdiscard;
  }
  Env out;
  out.t = C.t;
  out.center = C.center;
  out.log_scale = C.log_scale + t.log_scale + t.reference;
  out.max_trunc = std::max(env.max_trunc, rec.max_local_discarded_weight);
  out.variational = env.variational;
  out.variational.push_back(rec);
  if (ent && ent->profile && row_cut >= 1 && row_cut <= ent->Ly - 1)
    for (int b = 0; b < n - 1; ++b) (north ? ent->north : ent->south)[(row_cut - 1) * (ent->Lx - 1) + b] = profile[b];
  E.check_flag("variational absorption");
  return out;
}

}  // namespace sps
