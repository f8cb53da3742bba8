// Row boundary-MPS contraction, Born sampling and energy measurement on the
// Z2 engine.  Restates src/contraction/boundary_mps.jl (whole file),
// src/sampling/born.jl:27-163 (auxiliary kind, SymmetryBasis) and
// src/measurement/energy.jl.
#include "pipeline.h"
#include <algorithm>
#include <cfloat>

namespace sps {

static const double EPS = DBL_EPSILON;

Tensor unit_tensor(Engine& E, const std::vector<Par>& legs) {
  for (auto& p : legs)
    if (p->size() != 1 || (*p)[0] != 0) throw Error(SPS_ERR_ARGUMENT, "nontrivial OBC leg");
  double one = 1.0;
  return E.upload(legs, &one);
}

// double_layer (boundary_mps.jl:65-73): legs (w,n,e,s), each fused (ket,bra)
Tensor double_layer(Engine& E, const Tensor& ket, const Tensor& bra, const Tensor* physical) {
  Tensor A = physical ? ein(E, "pu,wnuaes->wnpaes", *physical, ket) : ket;
  Tensor raw = ein(E, "wnpaes,WNpaES->wWnNeEsS", A, bra);
  for (int axis : {6, 4, 2, 0}) raw = fuse(E, raw, axis, 2);
  return raw;
}

std::vector<Tensor> row_layers(Engine& E, const State& s) {
  std::vector<Tensor> out;
  out.reserve(s.sites.size());
  for (auto& A : s.sites) out.push_back(double_layer(E, A, A));
  return out;
}

static std::vector<Tensor> column(const std::vector<Tensor>& layers, int Lx, int y) {
  return std::vector<Tensor>(layers.begin() + y * Lx, layers.begin() + (y + 1) * Lx);
}

Env trivial_boundary(Engine& E, const std::vector<Tensor>& row, bool north) {
  Env env;
  Par triv = make_par(1, 0);
  int axis = north ? 1 : 3;
  for (auto& A : row) env.t.push_back(unit_tensor(E, {triv, A.legs[axis], triv}));
  return env;
}

// compress_boundary! (boundary_mps.jl:94-134)
CompressReport compress_boundary(Engine& E, std::vector<Tensor>& B, const BMPS& m, bool reverse,
                                 Entropy* ent, bool south_side, int row_cut) {
  if (m.chi < 1) throw Error(SPS_ERR_ARGUMENT, "chi must be positive");
  const int N = (int)B.size();
  double max_error = 0;
  Trunc tr;
  tr.chi = m.chi;
  tr.space[0] = m.space[0];
  tr.space[1] = m.space[1];
  if (!reverse) {
    for (int x = N - 1; x >= 1; --x) {
      LQres f = lq(E, B[x], {0}, {1, 2});
      B[x] = f.Q;
      B[x - 1] = ein(E, "lpk,kr->lpr", B[x - 1], f.L);
    }
    for (int x = 0; x < N - 1; ++x) {
      Tensor U, R;
      double err, nrm, entv;
      if (svd_prefers_kept(B[x], {0, 1}, {2}, tr, ent != nullptr)) {
        KeptSVD f = svd_kept(E, B[x], {0, 1}, {2}, tr, ent != nullptr, true);
        U = f.F;
        R = f.W;   // S V^T = U^T M
        err = f.err;
        nrm = f.norm;
        entv = f.entropy;
      } else {
        SVDres f = svd(E, B[x], {0, 1}, {2}, tr, ent != nullptr);
        std::vector<double> s(f.S[0]);
        s.insert(s.end(), f.S[1].begin(), f.S[1].end());
        U = f.U;
        R = scale_leg(E, f.V, 0, s);
        err = f.err;
        nrm = f.norm;
        entv = f.entropy;
      }
      if (ent) ent->record(south_side, row_cut, x + 1, entv);
      max_error = std::max(max_error, nrm == 0 ? 0.0 : (err / nrm) * (err / nrm));
      B[x] = U;
      B[x + 1] = ein(E, "lk,kpr->lpr", R, B[x + 1]);
    }
  } else {
    for (int x = 0; x < N - 1; ++x) {
      QRres f = qr(E, B[x], {0, 1}, {2});
      B[x] = f.Q;
      B[x + 1] = ein(E, "lk,kpr->lpr", f.R, B[x + 1]);
    }
    for (int x = N - 1; x >= 1; --x) {
      Tensor V, L;
      double err, nrm, entv;
      if (svd_prefers_kept(B[x], {0}, {1, 2}, tr, ent != nullptr)) {
        KeptSVD f = svd_kept(E, B[x], {0}, {1, 2}, tr, ent != nullptr, false);
        V = f.F;
        L = f.W;   // U S = M V
        err = f.err;
        nrm = f.norm;
        entv = f.entropy;
      } else {
        SVDres f = svd(E, B[x], {0}, {1, 2}, tr, ent != nullptr);
        std::vector<double> s(f.S[0]);
        s.insert(s.end(), f.S[1].begin(), f.S[1].end());
        V = f.V;
        L = scale_leg(E, f.U, 1, s);
        err = f.err;
        nrm = f.norm;
        entv = f.entropy;
      }
      if (ent) ent->record(south_side, row_cut, x, entv);
      max_error = std::max(max_error, nrm == 0 ? 0.0 : (err / nrm) * (err / nrm));
      B[x] = V;
      B[x - 1] = ein(E, "lpk,kr->lpr", B[x - 1], L);
    }
  }
  int center = reverse ? 0 : N - 1;
  double scale = norm(E, B[center]);
  if (!std::isfinite(scale)) throw Error(SPS_ERR_NUMERIC, "nonfinite boundary norm");
  if (scale != 0) scale_inplace(E, B[center], 1.0 / scale);
  return {max_error, scale == 0 ? -INFINITY : std::log(scale)};
}

// Truncated split of T (rows | cols) for the zip-up: `left` keeps the left
// vectors as F (rows..., k) and returns W = S V^T (k, cols...); otherwise F =
// V^T (k, cols...) and W = U S (rows..., k).
static void zipup_split(Engine& E, const Tensor& T, const Trunc& tr, bool left, Tensor& F, Tensor& W,
                        double& max_err) {
  const std::vector<int> rows{0, 1}, cols{2, 3};
  double err, nrm;
  if (svd_prefers_kept(T, rows, cols, tr, false)) {
    KeptSVD f = svd_kept(E, T, rows, cols, tr, false, left);
    F = f.F;
    W = f.W;
    err = f.err;
    nrm = f.norm;
  } else {
    SVDres f = svd(E, T, rows, cols, tr, false);
    std::vector<double> sv(f.S[0]);
    sv.insert(sv.end(), f.S[1].begin(), f.S[1].end());
    if (left) {
      F = f.U;
      W = scale_leg(E, f.V, 0, sv);
    } else {
      F = f.V;
      W = scale_leg(E, f.U, 2, sv);
    }
    err = f.err;
    nrm = f.norm;
  }
  max_err = std::max(max_err, nrm == 0 ? 0.0 : (err / nrm) * (err / nrm));
}

// Zip-up row absorption, this engine's variant (no counterpart in the
// reference): the boundary is brought into the canonical form opposite to the
// sweep (LQ sweep north, QR sweep south, on the small chi-bond tensors), then
// one sweep in which the carried factor times the boundary tensor times the
// row tensor is split by a truncated SVD with the truncation of
// _boundary_svd (boundary_mps.jl:33-42); the isometry becomes the new boundary
// tensor, the rest is carried on.  No canonical form is built, so no LQ/QR of
// the (chi d) x (d chi d) absorbed tensors is needed.  The centre is
// normalised as in compress_boundary! (boundary_mps.jl:129-133).
static Env absorb_zipup(Engine& E, const Env& env, const std::vector<Tensor>& row, const BMPS& m, bool north,
                        const std::vector<Tensor>* kets) {
  const int N = (int)row.size();
  Trunc tr;
  tr.chi = m.chi;
  tr.space[0] = m.space[0];
  tr.space[1] = m.space[1];
  // the zip-up's own truncation error is far above rounding: its splits
  // accept singular triplets at a relative residual of 1e-10
  tr.rtol = 1e-10;
  tr.gram = true;
  std::vector<Tensor> out(N);
  double max_err = 0;
  Par triv = make_par(1, 0);
  int center;
  std::vector<Tensor> B = env.t;
  if (north) {
    // right-canonical boundary (LQ sweep on the chi-bond tensors), so that
    // everything right of the zip front except the row is an isometry
    for (int x = N - 1; x >= 1; --x) {
      LQres f = lq(E, B[x], {0}, {1, 2});
      B[x] = f.Q;
      B[x - 1] = ein(E, "lnk,kr->lnr", B[x - 1], f.L);
    }
    Tensor C = unit_tensor(E, {triv, B[0].legs[0], row[0].legs[0]});   // (a, l, w)
    for (int x = 0; x < N; ++x) {
      Tensor T1 = ein(E, "alw,lnr->awnr", C, B[x]);
      Tensor T;
      if (kets) {   // (a, r, e, s) by ket then bra, viewed as (a, s, r, e)
        T = perm_view(layer_apply_wn(E, perm_view(T1, {1, 0, 2, 3}), (*kets)[x]), {0, 3, 1, 2});
      } else {
        T = ein(E, "awnr,wnes->asre", T1, row[x]);
      }
      if (x == N - 1) {
        out[x] = fuse(E, T, 2, 2);
        break;
      }
      zipup_split(E, T, tr, true, out[x], C, max_err);
    }
    center = N - 1;
  } else {
    // left-canonical boundary (QR sweep)
    for (int x = 0; x < N - 1; ++x) {
      QRres f = qr(E, B[x], {0, 1}, {2});
      B[x] = f.Q;
      B[x + 1] = ein(E, "lk,knr->lnr", f.R, B[x + 1]);
    }
    Tensor C = unit_tensor(E, {B[N - 1].legs[2], row[N - 1].legs[2], triv});   // (r, e, a)
    for (int x = N - 1; x >= 0; --x) {
      Tensor T1 = ein(E, "lsr,rea->lsea", B[x], C);
      Tensor T = ein(E, "lsea,wnes->lwna", T1, row[x]);
      if (x == 0) {
        out[x] = fuse(E, T, 0, 2);
        break;
      }
      zipup_split(E, T, tr, false, out[x], C, max_err);
    }
    center = 0;
  }
  double scale = norm(E, out[center]);
  if (!std::isfinite(scale)) throw Error(SPS_ERR_NUMERIC, "nonfinite boundary norm");
  if (scale != 0) scale_inplace(E, out[center], 1.0 / scale);
  Env res;
  res.t = std::move(out);
  res.log_scale = env.log_scale + (scale == 0 ? -INFINITY : std::log(scale));
  res.max_trunc = std::max(env.max_trunc, max_err);
  return res;
}

// _absorb for the row method (boundary_mps.jl:136-151)
Env absorb(Engine& E, const Env& env, const std::vector<Tensor>& row, const BMPS& m, bool north,
           Entropy* ent, int row_cut, const std::vector<Tensor>* kets) {
  if (m.variational) return absorb_variational(E, env, row, m, north, ent, row_cut);
  if (m.zipup) return absorb_zipup(E, env, row, m, north, north ? kets : nullptr);
  std::vector<Tensor> B;
  B.reserve(row.size());
  for (size_t x = 0; x < row.size(); ++x) {
    Tensor C = north ? ein(E, "lnr,wnep->lwpre", env.t[x], row[x]) : ein(E, "lsr,wpes->lwpre", env.t[x], row[x]);
    B.push_back(fuse(E, fuse(E, C, 3, 2), 0, 2));
  }
  CompressReport rep = compress_boundary(E, B, m, !north, ent, !north, row_cut);
  Env out;
  out.t = std::move(B);
  out.log_scale = env.log_scale + rep.log_scale;
  out.max_trunc = std::max(env.max_trunc, rep.max_trunc);
  return out;
}

// _close_boundary (boundary_mps.jl:153-163)
double close_boundary(Engine& E, const std::vector<Tensor>& B) {
  Tensor V = unit_tensor(E, {B[0].legs[0]});
  for (auto& A : B) {
    if (A.dims[1] != 1) throw Error(SPS_ERR_ARGUMENT, "close_boundary: open physical leg");
    Tensor P = unit_tensor(E, {A.legs[1]});
    Tensor W = ein(E, "l,lpr->pr", V, A);
    V = ein(E, "p,pr->r", P, W);
  }
  return sum_all(E, V);
}

double positive_real(double z, const char* name) {
  if (!(std::isfinite(z) && z > 0))
    throw Error(SPS_ERR_NUMERIC, std::string(name) + " requires a finite positive real value; received " +
                                     std::to_string(z));
  return z;
}

// lognorm / contract_layers (boundary_mps.jl:165-186)
LogNorm lognorm(Engine& E, const State& s, const BMPS& m) {
  if (m.diagonal) return lognorm_diagonal(E, s, m);
  auto layers = row_layers(E, s);
  Env env = trivial_boundary(E, column(layers, s.Lx, 0), true);
  for (int y = 0; y < s.Ly; ++y) env = absorb(E, env, column(layers, s.Lx, y), m, true, nullptr, y + 1);
  double v = positive_real(close_boundary(E, env.t), "norm");
  return {std::log(v) + env.log_scale + 2 * s.log_amplitude, std::log(v) + env.log_scale, env.max_trunc,
          env.variational};
}

// boundary_environments (boundary_mps.jl:193-209)
Envs boundary_environments(Engine& E, const std::vector<Tensor>& layers, int Lx, int Ly, const BMPS& m,
                           int side, Entropy* ent) {
  Envs r;
  r.north.resize(Ly + 1);
  r.south.resize(Ly + 1);
  r.north[0] = trivial_boundary(E, column(layers, Lx, 0), true);
  r.south[Ly] = trivial_boundary(E, column(layers, Lx, Ly - 1), false);
  if (side != 2)
    for (int y = 0; y < Ly; ++y) r.north[y + 1] = absorb(E, r.north[y], column(layers, Lx, y), m, true, ent, y + 1);
  if (side != 1)
    for (int y = Ly - 1; y >= 0; --y) r.south[y] = absorb(E, r.south[y + 1], column(layers, Lx, y), m, false, ent, y);
  r.max_trunc = std::max(side == 2 ? 0.0 : r.north[Ly].max_trunc, side == 1 ? 0.0 : r.south[0].max_trunc);
  return r;
}

// _left_step / _right_step, plain and slab (boundary_mps.jl:216-246)
// X (w, b, n, c) contracted over (w, n) with double_layer(ket, ket): the
// (b, c, e, s) of ein("wbnc,wnes->bces", X, E) in two single-layer steps,
// ket then bra (2 chi^2 D^6 P A flops each instead of 2 chi^2 D^8): one fused
// kernel when its shared-memory tiles fit, else two table-driven contractions.
Tensor layer_apply_wn(Engine& E, const Tensor& X, const Tensor& ket) {
  Tensor X5 = split(E, split(E, X, 2, {ket.legs[1], ket.legs[1]}), 0, {ket.legs[0], ket.legs[0]});   // w1 w2 b n1 n2 c
  Tensor Z;
  // the fused kernel is FP64; a low-precision mode takes the two contractions
  if (E.precision > 0 || !layer_wn_fused(E, X5, ket, Z)) {
    Tensor Y = ein(E, "xybuvc,xupaef->ybvcpaef", X5, ket);
    Z = ein(E, "ybvcpaef,yvpagh->bcegfh", Y, ket);
  }
  return fuse(E, fuse(E, Z, 4, 2), 2, 2);
}

// X (a, n, e, d) contracted over (n, e) with double_layer(ket, ket): the
// (a, d, w, s) of ein("aned,wnes->adws", X, E), ket then bra.
static Tensor layer_apply_ne(Engine& E, const Tensor& X, const Tensor& ket) {
  Tensor X6 = split(E, split(E, X, 2, {ket.legs[4], ket.legs[4]}), 1, {ket.legs[1], ket.legs[1]});   // a n1 n2 e1 e2 d
  Tensor Y = ein(E, "auvxyd,wupqxs->avydwpqs", X6, ket);
  Tensor Z = ein(E, "avydwpqs,zvpqyt->adwzst", Y, ket);
  return fuse(E, fuse(E, Z, 4, 2), 2, 2);
}

Tensor left_step(Engine& E, const Tensor& L, const Tensor& T, const Layer& row, const Tensor& B) {
  if (row.slab) {
    Tensor X = ein(E, "awvb,anc->wvbnc", L, T);
    Tensor Y = ein(E, "wvbnc,wnek->vbcek", X, row.a);
    Tensor Z = ein(E, "vbcek,vkfs->bcefs", Y, row.b);
    return ein(E, "bcefs,bsd->cefd", Z, B);
  }
  Tensor X = ein(E, "awb,anc->wbnc", L, T);
  Tensor Y = row.layered ? layer_apply_wn(E, X, row.ket) : ein(E, "wbnc,wnes->bces", X, row.a);
  return ein(E, "bces,bsd->ced", Y, B);
}

Tensor right_step(Engine& E, const Tensor& T, const Layer& row, const Tensor& B, const Tensor& R) {
  if (row.slab) {
    Tensor X = ein(E, "anc,cefd->anefd", T, R);
    Tensor Y = ein(E, "anefd,wnek->awkfd", X, row.a);
    Tensor Z = ein(E, "awkfd,vkfs->awvsd", Y, row.b);
    return ein(E, "awvsd,bsd->awvb", Z, B);
  }
  Tensor X = ein(E, "anc,ced->aned", T, R);
  if (row.layered) return ein(E, "adws,bsd->awb", layer_apply_ne(E, X, row.ket), B);
  Tensor Y = ein(E, "aned,wnes->awsd", X, row.a);
  return ein(E, "awsd,bsd->awb", Y, B);
}

Tensor row_edge(Engine& E, const std::vector<Tensor>& top, const std::vector<Layer>& row,
                const std::vector<Tensor>& bottom, bool left) {
  int i = left ? 0 : (int)row.size() - 1;
  int a = left ? 0 : 2;
  if (row[i].slab)
    return unit_tensor(E, {top[i].legs[a], row[i].a.legs[a], row[i].b.legs[a], bottom[i].legs[a]});
  return unit_tensor(E, {top[i].legs[a], row[i].a.legs[a], bottom[i].legs[a]});
}

// row_environments (boundary_mps.jl:261-273)
RowEnvs row_environments(Engine& E, const std::vector<Tensor>& top, const std::vector<Layer>& row,
                         const std::vector<Tensor>& bottom, int side) {
  int N = (int)row.size();
  RowEnvs r;
  r.left.resize(N + 1);
  r.right.resize(N + 1);
  r.left[0] = row_edge(E, top, row, bottom, true);
  r.right[N] = row_edge(E, top, row, bottom, false);
  if (side != 2)
    for (int x = 0; x < N; ++x) {
      r.left[x + 1] = left_step(E, r.left[x], top[x], row[x], bottom[x]);
      safe_scale_inplace(E, r.left[x + 1]);
    }
  if (side != 1)
    for (int x = N - 1; x >= 0; --x) {
      r.right[x] = right_step(E, top[x], row[x], bottom[x], r.right[x + 1]);
      safe_scale_inplace(E, r.right[x]);
    }
  return r;
}

void row_scalar_to(Engine& E, const Tensor& L, const Tensor& T, const Layer& row, const Tensor& B,
                   const Tensor& R, int slot) {
  Tensor X = left_step(E, L, T, row, B);
  dot_to(E, X, R, slot);
}

// ---------------------------------------------------------------------------
// states
// ---------------------------------------------------------------------------
State identity_pepo(Engine& E, int Lx, int Ly) {
  State s;
  s.Lx = Lx;
  s.Ly = Ly;
  Par t = make_par(1, 0), p2 = make_par(1, 1);
  double a[4] = {1, 0, 0, 1};   // A[0,0,p,a,0,0] = delta_pa
  for (int i = 0; i < Lx * Ly; ++i) s.sites.push_back(E.upload({t, t, p2, p2, t, t}, a));
  s.beta = 0;
  s.log_amplitude = 0;
  s.pepo = true;
  return s;
}

// normalize_state! (src/states/finite.jl:89-100), row-major site order
std::vector<double> normalize_state(Engine& E, State& s) {
  int n = s.Lx * s.Ly;
  if (n > Engine::NSCAL) throw Error(SPS_ERR_ARGUMENT, "lattice too large");
  for (int i = 0; i < n; ++i) norm2_to(E, s.sites[i], i);
  SPS_CUDA(cudaMemcpyAsync(E.hscal, E.dscal, sizeof(double) * n, cudaMemcpyDeviceToHost, E.stream));
  E.sync();
  std::vector<double> inc(n);
  for (int y = 0; y < s.Ly; ++y)
    for (int x = 0; x < s.Lx; ++x) {
      int i = x + y * s.Lx;
      double v = std::sqrt(E.hscal[i]);
      if (!(std::isfinite(v) && v > 0))
        throw Error(SPS_ERR_NUMERIC, "zero or nonfinite tensor at (" + std::to_string(x + 1) + "," +
                                         std::to_string(y + 1) + ")");
      scale_inplace(E, s.sites[i], 1.0 / v);
      inc[i] = std::log(v);
      s.log_amplitude += inc[i];
    }
  return inc;
}

// ---------------------------------------------------------------------------
// Born sampling (src/sampling/born.jl:56-163), kind = :auxiliary and :physical
// ---------------------------------------------------------------------------
Tensor project_aux(Engine& E, const Tensor& A, int k) {
  return slice_leg(E, A, 3, k, k == 0 ? make_par(1, 0) : make_par(0, 1));
}

// _project(A, B, k, :physical) for SymmetryBasis (basis.jl:87): the physical
// leg restricted to its basis state k, a one-dimensional leg of that state's parity
Tensor project_physical(Engine& E, const Tensor& A, int k) {
  const int c = (*A.legs[2])[k];
  return slice_leg(E, A, 2, k, c == 0 ? make_par(1, 0) : make_par(0, 1));
}

SamplingCache make_sampling_cache(Engine& E, const State& s, const BMPS& m, int kind) {
  if (kind != KIND_AUXILIARY && kind != KIND_PHYSICAL) throw Error(SPS_ERR_ARGUMENT, "unknown sampling kind");
  SamplingCache c;
  c.Lx = s.Lx;
  c.Ly = s.Ly;
  c.kind = kind;
  c.method = m;
  c.state_ref = &s;
  if (kind == KIND_PHYSICAL) {
    // a PEPS (one-dimensional auxiliary legs); its total charge is the fusion
    // of the auxiliary charges (_state_charge, basis.jl:89-92), which every
    // physical configuration of nonzero amplitude fuses to
    c.target = 0;
    for (auto& A : s.sites) {
      if (A.dims[3] != 1) throw Error(SPS_ERR_ARGUMENT, "proposal requires PEPS");
      if (A.dims[2] != 2) throw Error(SPS_ERR_ARGUMENT, "proposal sampling needs a two-state physical leg");
      c.target ^= (*A.legs[3])[0];
    }
  }
  if (m.diagonal) {
    // the diagonal draw keeps the projected kets and the southeast
    // boundaries of every layer (diagonal_born.jl:11-21)
    for (auto& A : s.sites) {
      std::array<Tensor, 2> kets;
      for (int k = 0; k < 2; ++k) kets[k] = kind == KIND_PHYSICAL ? project_physical(E, A, k) : project_aux(E, A, k);
      c.candidate_kets.push_back(kets);
    }
    diagonal_southeast(E, s, m, c.southeast);
    return c;
  }
  c.layers = row_layers(E, s);
  for (auto& A : s.sites) {
    std::array<Tensor, 2> cand, kets;
    for (int k = 0; k < 2; ++k) {
      kets[k] = kind == KIND_PHYSICAL ? project_physical(E, A, k) : project_aux(E, A, k);
      cand[k] = double_layer(E, kets[k], kets[k]);
    }
    c.candidates.push_back(cand);
    c.candidate_kets.push_back(kets);
  }
  c.south.resize(s.Ly + 1);
  c.south[s.Ly] = trivial_boundary(E, column(c.layers, s.Lx, s.Ly - 1), false);
  for (int y = s.Ly - 1; y >= 0; --y)
    c.south[y] = absorb(E, c.south[y + 1], column(c.layers, s.Lx, y), m, false, nullptr, y);
  return c;
}

// _rs_logsumexp and _categorical (src/resample/selection.jl:1-7, 68-80)
static double logsumexp(const std::vector<double>& x) {
  if (x.empty()) return -INFINITY;
  double pivot = *std::max_element(x.begin(), x.end());
  if (pivot == -INFINITY) return -INFINITY;
  if (!std::isfinite(pivot)) throw Error(SPS_ERR_NUMERIC, "nonfinite positive log mass");
  double s = 0;
  for (double v : x) s += std::exp(v - pivot);
  return pivot + std::log(s);
}

int categorical(const std::vector<double>& lm, double u, int* near) {
  double z = logsumexp(lm);
  if (!std::isfinite(z)) throw Error(SPS_ERR_NUMERIC, "proposal requires positive total probability");
  double cum = 0;
  int last = -1;
  for (int j = 0; j < (int)lm.size(); ++j) {
    if (lm[j] == -INFINITY) continue;
    last = j;
    cum += std::exp(lm[j] - z);
    if (std::fabs(u - cum) < 1e-12 && near) ++*near;
    if (u < cum) return j;
  }
  return last;
}

// One Born conditional on the device (born.jl:130-151 with _categorical,
// selection.jl:68-80): raw[0..1] are the two candidates' scalars.  Validity
// checks, normalisation, the categorical choice with the site's uniform, the
// log-probability and the conditional are computed by one thread; the choice
// goes to cfg[site] (label 1/2) and *sel (0/1).  err[0] records the first
// failure (1 invalid conditional, 2 zero total mass) and err[1] its site;
// once set, later sites only copy their choice so that the draw stays
// well-defined until the host reads the flag at the end of the row.
__global__ void born_step_kernel(const double* raw, const double* u, int site, int* cfg, int* sel, double* logp,
                                 double* cond, int* err, int* near) {
  if (threadIdx.x != 0) return;
  const double r0 = raw[0], r1 = raw[1];
  const double scale = fmax(fabs(r0), fabs(r1));
  int k = 0;
  if (err[0] == 0) {
    const bool bad = !(isfinite(r0) && r0 >= -64 * DBL_EPSILON * scale) ||
                     !(isfinite(r1) && r1 >= -64 * DBL_EPSILON * scale);
    const double v0 = fmax(r0, 0.0), v1 = fmax(r1, 0.0), total = v0 + v1;
    if (bad || !(total > 0)) {
      err[0] = bad ? 1 : 2;
      err[1] = site;
    } else {
      const double p[2] = {v0 / total, v1 / total};
      const double lm[2] = {p[0] > 0 ? log(p[0]) : -INFINITY, p[1] > 0 ? log(p[1]) : -INFINITY};
      const double pivot = fmax(lm[0], lm[1]);
      double ssum = 0;
      for (int j = 0; j < 2; ++j) ssum += exp(lm[j] - pivot);
      const double z = pivot + log(ssum);
      double cum = 0;
      int last = -1;
      k = -1;
      for (int j = 0; j < 2; ++j) {
        if (lm[j] == -INFINITY) continue;
        last = j;
        cum += exp(lm[j] - z);
        if (fabs(u[site] - cum) < 1e-12) ++*near;
        if (u[site] < cum) {
          k = j;
          break;
        }
      }
      if (k < 0) k = last;
      cond[site] = p[k];
      *logp += log(p[k]);
    }
  }
  cfg[site] = k + 1;
  *sel = k;
}

// out = sel ? b : a, elementwise (a and b share one layout)
__global__ void select2_kernel(const double* __restrict__ a, const double* __restrict__ b, const int* sel,
                               double* __restrict__ out, int64_t n) {
  const double* src = *sel ? b : a;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = src[i];
}

// A draw from uniforms with the conditionals decided on the device: the
// contractions of a row are queued without a host round trip per site (the
// chosen candidate's step becomes the next left environment by a device-side
// select), and the host synchronises once per row to learn the row's
// choices, which fix the tensors of the row's absorption.  Same arithmetic
// and order as the host path below.
static SampleResult sample_device(Engine& E, const SamplingCache& c, const double* uniforms) {
  const int Lx = c.Lx, Ly = c.Ly, L = Lx * Ly;
  SampleResult res;
  res.config.assign(L, 0);
  Buf ib = E.alloc(sizeof(int) * (L + 8));
  Buf db = E.alloc(sizeof(double) * (2 * (size_t)L + 8));
  int* dcfg = (int*)ib->ptr;
  int* derr = dcfg + L;      // 2 ints
  int* dnear = derr + 2;
  int* dsel = derr + 3;
  double* dlogp = (double*)db->ptr;
  double* dcond = dlogp + 1;
  double* du = dcond + L;
  SPS_CUDA(cudaMemsetAsync(ib->ptr, 0, sizeof(int) * (L + 8), E.stream));
  SPS_CUDA(cudaMemsetAsync(db->ptr, 0, sizeof(double) * (L + 1), E.stream));
  E.stage(uniforms, sizeof(double) * L, du);
  Env north = trivial_boundary(E, column(c.layers, Lx, 0), true);
  double maxtr = 0;
  for (auto& e : c.south) maxtr = std::max(maxtr, e.max_trunc);
  // row choices + err[2] + near, clear of the log-probability and conditionals at the front
  int* hrow = reinterpret_cast<int*>(E.hscal + Engine::NSCAL - 64);
  for (int y = 0; y < Ly; ++y) {
    std::vector<Layer> row(Lx);
    std::vector<Tensor> rowt = column(c.layers, Lx, y);
    for (int x = 0; x < Lx; ++x) {
      row[x].a = rowt[x];
      row[x].ket = c.state_ref->sites[x + y * Lx];
      row[x].layered = true;
    }
    const auto& top = north.t;
    const auto& bottom = c.south[y + 1].t;
    RowEnvs e = row_environments(E, top, row, bottom, 2);
    Tensor left = e.left[0];
    for (int x = 0; x < Lx; ++x) {
      const int site = x + y * Lx;
      Tensor LT = ein(E, "awb,anc->wbnc", left, top[x]);
      Tensor step[2];
      for (int k = 0; k < 2; ++k) {
        Tensor Y = layer_apply_wn(E, LT, c.candidate_kets[site][k]);
        step[k] = ein(E, "bces,bsd->ced", Y, bottom[x]);
        dot_to(E, step[k], e.right[x + 1], 10 + k);
      }
      born_step_kernel<<<1, 32, 0, E.stream>>>(E.dscal + 10, du, site, dcfg, dsel, dlogp, dcond, derr, dnear);
      SPS_CUDA(cudaGetLastError());
      E.launches++;
      if (x < Lx - 1) {
        if (!step[0].contiguous() || !step[1].contiguous() || step[0].dims != step[1].dims)
          throw Error(SPS_ERR_ARGUMENT, "sample_configuration: candidate steps differ in layout");
        Tensor nl = E.empty(step[0].legs);
        const int64_t n = nl.size();
        select2_kernel<<<(int)std::min<int64_t>((n + 255) / 256, 1024), 256, 0, E.stream>>>(
            step[0].ptr(), step[1].ptr(), dsel, nl.ptr(), n);
        SPS_CUDA(cudaGetLastError());
        E.launches++;
        left = nl;
        safe_scale_inplace(E, left);
      }
    }
    // the row's choices (and the first failure) to the host: one synchronisation per row
    SPS_CUDA(cudaMemcpyAsync(hrow, dcfg + y * Lx, sizeof(int) * Lx, cudaMemcpyDeviceToHost, E.stream));
    SPS_CUDA(cudaMemcpyAsync(hrow + Lx, derr, sizeof(int) * 3, cudaMemcpyDeviceToHost, E.stream));
    E.sync();
    if (hrow[Lx] != 0) {
      SPS_CUDA(cudaMemsetAsync(E.dflag, 0, sizeof(int), E.stream));   // flags raised by the draw after the failure
      const int s = hrow[Lx + 1];
      const std::string where = "(" + std::to_string(s % Lx + 1) + "," + std::to_string(s / Lx + 1) + ")";
      if (hrow[Lx] == 1)
        throw Error(SPS_ERR_BORN, "invalid Born conditional at " + where + "; increase chi_sampling");
      throw Error(SPS_ERR_BORN, "Born conditional has zero total mass at " + where);
    }
    E.check_flag("sample_configuration");
    std::vector<Tensor> rt(Lx), rk(Lx);
    for (int x = 0; x < Lx; ++x) {
      const int k = hrow[x] - 1;
      if (k < 0 || k > 1) throw Error(SPS_ERR_NUMERIC, "sample_configuration: no candidate chosen");
      res.config[x + y * Lx] = k + 1;
      rt[x] = c.candidates[x + y * Lx][k];
      rk[x] = c.candidate_kets[x + y * Lx][k];
    }
    if (y == Ly - 1) {   // log-probability, conditionals and near-boundary count with the last row
      SPS_CUDA(cudaMemcpyAsync(E.hscal, dlogp, sizeof(double) * (L + 1), cudaMemcpyDeviceToHost, E.stream));
      E.sync();
      res.log_probability = E.hscal[0];
      res.conditionals.assign(E.hscal + 1, E.hscal + 1 + L);
      res.near_boundary = hrow[Lx + 2];
    }
    north = absorb(E, north, rt, c.method, true, nullptr, y + 1, &rk);
    maxtr = std::max(maxtr, north.max_trunc);
  }
  res.max_env_trunc = maxtr;
  return res;
}

// The site hole of a row (born.jl:75-84): left, top, bottom and right
// environments joined around site x, each fused double-layer leg split into
// (ket, bra), as a symmetric matrix on the ket virtual legs: scaled by its
// Frobenius norm and symmetrised, then projected on its nonnegative spectrum
// (_positive_metric with square_root, tensors.jl:65-94).  Returns the
// eigenvectors scaled by the square roots of the clipped eigenvalues (legs
// w, n, e, s, z), so that a candidate's weight is |v . root|^2.
static Tensor site_metric_root(Engine& E, const Tensor& left, const Tensor& top, const Tensor& bottom,
                               const Tensor& right, const Tensor& A, SampleResult& res) {
  Tensor X = ein(E, "awb,anc->wbnc", left, top);
  Tensor Y = ein(E, "bsd,ced->bsce", bottom, right);
  Tensor H = contiguous(E, ein(E, "wbnc,bsce->wnes", X, Y));
  const int vl[4] = {0, 1, 4, 5};   // the site's virtual legs w, n, e, s
  for (int k = 3; k >= 0; --k) H = split(E, H, k, {A.legs[vl[k]], A.legs[vl[k]]});   // (wk wb nk nb ek eb sk sb)
  return metric_root(E, H, res);
}

Tensor metric_root(Engine& E, const Tensor& H, SampleResult& res) {
  if (!all_finite(E, H)) throw Error(SPS_ERR_NUMERIC, "nonfinite norm metric");
  const double scale = norm(E, H);
  Tensor Hm = contiguous(E, perm_view(H, {1, 3, 5, 7, 0, 2, 4, 6}));   // (bras, kets)
  Tensor HmT = perm_view(Hm, {4, 5, 6, 7, 0, 1, 2, 3});
  const double f = scale != 0 ? 0.5 / scale : 0.5;
  Tensor Hs = axpby(E, f, Hm, f, HmT);
  int64_t half = 1;
  for (int k = 0; k < 4; ++k) half *= Hs.dims[k];
  EIGres eg = (half / 2 >= E.eigh_multi_min) ? eigh_unit_shifted(E, Hs, {0, 1, 2, 3}, {4, 5, 6, 7})
                                             : eigh(E, Hs, {0, 1, 2, 3}, {4, 5, 6, 7});
  std::vector<double> root;
  double lo = 0.0, hi = 0.0;
  int negative = 0;
  for (int c = 0; c < 2; ++c)
    for (double v : eg.w[c]) {
      lo = std::min(lo, v);
      hi = std::max(hi, std::fabs(v));
      negative += v < 0;
      root.push_back(v > 0 ? std::sqrt(v) : 0.0);
    }
  res.metric_repairs += negative > 0;
  res.min_relative_eigenvalue = std::min(res.min_relative_eigenvalue, lo / std::max(hi, DBL_MIN));
  return scale_leg(E, eg.V, 4, root);
}

// sample_configuration for kind = :physical (born.jl:86-163): the Born
// proposal of a PEPS over its physical labels.  Each conditional weighs the
// site's two physically projected kets with the PSD-projected site hole;
// outcomes that cannot reach the PEPS's total parity get no weight (the
// charge rule of born.jl:114-116, which binds at the last site), all-zero
// weights fall back to the uniform choice among the allowed outcomes
// (born.jl:127-131), and the last row is not absorbed.
static SampleResult sample_physical(Engine& E, const SamplingCache& c, const double* uniforms,
                                    const int* configuration) {
  const int Lx = c.Lx, Ly = c.Ly, L = Lx * Ly;
  SampleResult res;
  res.config.assign(L, 0);
  double maxtr = 0;
  for (auto& e : c.south) maxtr = std::max(maxtr, e.max_trunc);
  res.max_env_trunc = maxtr;
  if (configuration) {
    int charge = 0;
    for (int i = 0; i < L; ++i) {
      if (configuration[i] != 1 && configuration[i] != 2)
        throw Error(SPS_ERR_ARGUMENT, "configuration contains an unknown basis label");
      charge ^= configuration[i] - 1;
    }
    if (charge != c.target) {
      for (int i = 0; i < L; ++i) res.config[i] = configuration[i];
      res.log_probability = -INFINITY;
      return res;
    }
  }
  Env north = trivial_boundary(E, column(c.layers, Lx, 0), true);
  int prefix = 0;
  double logp = 0;
  for (int y = 0; y < Ly; ++y) {
    std::vector<Layer> row(Lx);
    std::vector<Tensor> rowt = column(c.layers, Lx, y);
    for (int x = 0; x < Lx; ++x) {
      row[x].a = rowt[x];
      row[x].ket = c.state_ref->sites[x + y * Lx];
      row[x].layered = true;
    }
    const auto& top = north.t;
    const auto& bottom = c.south[y + 1].t;
    RowEnvs e = row_environments(E, top, row, bottom, 2);
    Tensor left = e.left[0];
    std::vector<Tensor> rt(Lx), rk(Lx);
    for (int x = 0; x < Lx; ++x) {
      const int site = x + y * Lx;
      const Tensor& A = c.state_ref->sites[site];
      Tensor root = site_metric_root(E, left, top[x], bottom[x], e.right[x + 1], A, res);
      bool allowed[2];
      double values[2];
      for (int k = 0; k < 2; ++k) {
        // every later site offers both parities, so only the last site is bound
        allowed[k] = site < L - 1 || (prefix ^ (*A.legs[2])[k]) == c.target;
        values[k] = 0.0;
        if (!allowed[k]) continue;
        Tensor u = ein(E, "wnpaes,wnesz->paz", c.candidate_kets[site][k], root);
        values[k] = dot(E, u, u);
      }
      if (!allowed[0] && !allowed[1]) throw Error(SPS_ERR_BORN, "sampling prefix violates the total symmetry sector");
      const double total = values[0] + values[1];
      if (!std::isfinite(total)) throw Error(SPS_ERR_NUMERIC, "nonfinite proposal weight");
      double p[2];
      if (total == 0) {
        const int n = (int)allowed[0] + (int)allowed[1];
        for (int k = 0; k < 2; ++k) p[k] = allowed[k] ? 1.0 / n : 0.0;
        res.zero_proposals++;
      } else {
        for (int k = 0; k < 2; ++k) p[k] = values[k] / total;
      }
      int k;
      if (configuration) {
        k = configuration[site] - 1;
      } else {
        std::vector<double> lm{p[0] > 0 ? std::log(p[0]) : -INFINITY, p[1] > 0 ? std::log(p[1]) : -INFINITY};
        k = categorical(lm, uniforms[site], &res.near_boundary);
      }
      res.config[site] = k + 1;
      res.conditionals.push_back(p[k]);
      if (p[k] == 0.0) {
        res.log_probability = -INFINITY;
        res.max_env_trunc = maxtr;
        return res;
      }
      logp += std::log(p[k]);
      prefix ^= (*A.legs[2])[k];
      rt[x] = c.candidates[site][k];
      rk[x] = c.candidate_kets[site][k];
      if (x < Lx - 1) {
        Tensor LT = ein(E, "awb,anc->wbnc", left, top[x]);
        Tensor Yk = layer_apply_wn(E, LT, rk[x]);
        left = ein(E, "bces,bsd->ced", Yk, bottom[x]);
        safe_scale_inplace(E, left);
      }
    }
    if (y < Ly - 1) {
      north = absorb(E, north, rt, c.method, true, nullptr, y + 1, &rk);
      maxtr = std::max(maxtr, north.max_trunc);
    }
  }
  res.log_probability = logp;
  res.max_env_trunc = maxtr;
  return res;
}

SampleResult sample_configuration(Engine& E, const SamplingCache& c, const double* uniforms,
                                  const int* configuration) {
  if (c.method.diagonal) return sample_diagonal(E, c, uniforms, configuration);
  if (c.kind == KIND_PHYSICAL) return sample_physical(E, c, uniforms, configuration);
  if (uniforms && !configuration && c.Lx * c.Ly + 1 <= Engine::NSCAL - 64 && c.Lx + 3 <= 128)
    return sample_device(E, c, uniforms);
  const int Lx = c.Lx, Ly = c.Ly;
  SampleResult res;
  res.config.assign(Lx * Ly, 0);
  Env north = trivial_boundary(E, column(c.layers, Lx, 0), true);
  double maxtr = 0;
  for (auto& e : c.south) maxtr = std::max(maxtr, e.max_trunc);
  double logp = 0;
  for (int y = 0; y < Ly; ++y) {
    std::vector<Layer> row(Lx);
    std::vector<Tensor> rowt = column(c.layers, Lx, y);
    for (int x = 0; x < Lx; ++x) {
      row[x].a = rowt[x];
      row[x].ket = c.state_ref->sites[x + y * Lx];
      row[x].layered = true;
    }
    const auto& top = north.t;
    const auto& bottom = c.south[y + 1].t;
    RowEnvs e = row_environments(E, top, row, bottom, 2);
    Tensor left = e.left[0];
    for (int x = 0; x < Lx; ++x) {
      const auto& cand = c.candidates[x + y * Lx];
      // the two candidate scalars share left x top; each candidate's left
      // step is kept, so the chosen one becomes the next left environment
      // (the same contractions as left_step, so identical values)
      Tensor LT = ein(E, "awb,anc->wbnc", left, top[x]);
      Tensor step[2];
      for (int k = 0; k < 2; ++k) {
        Tensor Y = layer_apply_wn(E, LT, c.candidate_kets[x + y * Lx][k]);
        step[k] = ein(E, "bces,bsd->ced", Y, bottom[x]);
        dot_to(E, step[k], e.right[x + 1], 10 + k);
      }
      SPS_CUDA(cudaMemcpyAsync(E.hscal + 10, E.dscal + 10, 2 * sizeof(double), cudaMemcpyDeviceToHost, E.stream));
      E.sync();
      E.check_flag("sample_configuration");
      double raw[2] = {E.hscal[10], E.hscal[11]};
      double scale = std::max(std::fabs(raw[0]), std::fabs(raw[1]));
      for (double z : raw)
        if (!(std::isfinite(z) && z >= -64 * EPS * scale))
          throw Error(SPS_ERR_BORN, "invalid Born conditional at (" + std::to_string(x + 1) + "," +
                                        std::to_string(y + 1) + "); increase chi_sampling");
      double v0 = std::max(raw[0], 0.0), v1 = std::max(raw[1], 0.0);
      double total = v0 + v1;
      if (!(total > 0))
        throw Error(SPS_ERR_BORN, "Born conditional has zero total mass at (" + std::to_string(x + 1) + "," +
                                      std::to_string(y + 1) + ")");
      double p[2] = {v0 / total, v1 / total};
      int k;
      if (configuration) {
        k = configuration[x + y * Lx] - 1;
        if (k < 0 || k > 1) throw Error(SPS_ERR_ARGUMENT, "configuration contains an unknown basis label");
      } else {
        std::vector<double> lm{p[0] > 0 ? std::log(p[0]) : -INFINITY, p[1] > 0 ? std::log(p[1]) : -INFINITY};
        k = categorical(lm, uniforms[x + y * Lx], &res.near_boundary);
      }
      res.config[x + y * Lx] = k + 1;
      res.conditionals.push_back(p[k]);
      if (p[k] == 0.0) {
        res.log_probability = -INFINITY;
        res.max_env_trunc = maxtr;
        return res;
      }
      logp += std::log(p[k]);
      row[x].a = cand[k];
      if (x < Lx - 1) {
        left = step[k];
        safe_scale_inplace(E, left);
      }
    }
    std::vector<Tensor> rt(Lx), rk(Lx);
    for (int x = 0; x < Lx; ++x) {
      rt[x] = row[x].a;
      rk[x] = c.candidate_kets[x + y * Lx][res.config[x + y * Lx] - 1];
    }
    north = absorb(E, north, rt, c.method, true, nullptr, y + 1, &rk);
    maxtr = std::max(maxtr, north.max_trunc);
  }
  res.log_probability = logp;
  res.max_env_trunc = maxtr;
  return res;
}

// project_configuration (born.jl:27-36)
State project_configuration(Engine& E, const State& pepo, const int* configuration,
                            std::vector<double>* log_norms) {
  State s;
  s.Lx = pepo.Lx;
  s.Ly = pepo.Ly;
  s.beta = pepo.beta;
  s.log_amplitude = pepo.log_amplitude;
  s.pepo = false;
  for (int i = 0; i < pepo.Lx * pepo.Ly; ++i) {
    int k = configuration[i] - 1;
    if (k < 0 || k > 1) throw Error(SPS_ERR_ARGUMENT, "configuration contains an unknown basis label");
    s.sites.push_back(project_aux(E, pepo.sites[i], k));
  }
  auto inc = normalize_state(E, s);
  if (log_norms) *log_norms = inc;
  return s;
}

// ---------------------------------------------------------------------------
// energy (src/measurement/energy.jl)
// ---------------------------------------------------------------------------
// _operator_factors(ZZ) for the Z2 TFIM: M[(p,u),(q,v)] = z[p,u] z[q,v] is
// rank one in the odd block with singular value 2, so F = sqrt(2) z and
// G = z / sqrt(2) on a one-state odd leg r (energy.jl:8-12).
void operator_factors(Engine& E, Tensor& F, Tensor& G) {
  Par p2 = make_par(1, 1), r = make_par(0, 1);
  double s2 = std::sqrt(2.0);
  double f[4] = {0, s2, s2, 0};          // F[p,u,r]: (0,1)->s2, (1,0)->s2
  double g[4] = {0, 1 / s2, 1 / s2, 0};  // G[r,q,v]
  F = E.upload({p2, p2, r}, f);
  G = E.upload({r, p2, p2}, g);
}

void operator_pair(Engine& E, const Tensor& A, const Tensor& B, const Tensor& F, const Tensor& G, bool horizontal,
                   Tensor& C, Tensor& D) {
  if (horizontal) {
    C = fuse(E, ein(E, "wnuaes,pur->wnpaers", A, F), 4, 2);
    D = fuse(E, ein(E, "wnvaes,rqv->wrnqaes", B, G), 0, 2);
  } else {
    C = fuse(E, ein(E, "wnuaes,pur->wnpaesr", A, F), 5, 2);
    D = fuse(E, ein(E, "wnvaes,rqv->wnrqaes", B, G), 1, 2);
  }
}

double real_ratio(double a, double b) {
  if (b == 0) throw Error(SPS_ERR_NUMERIC, "zero local norm environment");
  double z = a / b;
  if (!std::isfinite(z)) throw Error(SPS_ERR_NUMERIC, "nonreal observable");
  return z;
}

EnergyResult measure_energy(Engine& E, const State& s, const Model& m, const BMPS& method,
                            bool record_entropy) {
  if (method.diagonal) return measure_energy_diagonal(E, s, m, method, record_entropy);
  const int Lx = s.Lx, Ly = s.Ly;
  EnergyResult out;
  out.entropy.profile = record_entropy;
  out.entropy.Lx = Lx;
  out.entropy.Ly = Ly;
  if (record_entropy) {
    out.entropy.north.assign(std::max(0, (Ly - 1) * (Lx - 1)), NAN);
    out.entropy.south.assign(std::max(0, (Ly - 1) * (Lx - 1)), NAN);
  }
  auto layers = row_layers(E, s);
  Envs env = boundary_environments(E, layers, Lx, Ly, method, 0, record_entropy ? &out.entropy : nullptr);
  Par p2 = make_par(1, 1);
  double xo[4] = {1, 0, 0, -1};
  Tensor X = E.upload({p2, p2}, xo);
  Tensor F, G;
  operator_factors(E, F, G);
  // slot layout: [100 + 2*k] numerator, [101 + 2*k] denominator
  int nterm = Lx * Ly + Ly * (Lx - 1) + (Ly - 1) * Lx;
  if (100 + 2 * nterm > Engine::NSCAL) throw Error(SPS_ERR_ARGUMENT, "lattice too large for measurement");
  int term = 0;
  for (int y = 0; y < Ly; ++y) {
    std::vector<Layer> row(Lx);
    for (int x = 0; x < Lx; ++x) row[x].a = layers[x + y * Lx];
    const auto& top = env.north[y].t;
    const auto& bottom = env.south[y + 1].t;
    RowEnvs e = row_environments(E, top, row, bottom, 0);
    for (int x = 0; x < Lx; ++x) {
      Layer xl;
      xl.a = double_layer(E, s.at(x, y), s.at(x, y), &X);
      row_scalar_to(E, e.left[x], top[x], xl, bottom[x], e.right[x + 1], 100 + 2 * term);
      row_scalar_to(E, e.left[x], top[x], row[x], bottom[x], e.right[x + 1], 101 + 2 * term);
      ++term;
    }
    for (int x = 0; x < Lx - 1; ++x) {
      const Tensor& A = s.at(x, y);
      const Tensor& B = s.at(x + 1, y);
      Tensor C, D;
      operator_pair(E, A, B, F, G, true, C, D);
      Layer lc, ld;
      lc.a = double_layer(E, C, A);
      ld.a = double_layer(E, D, B);
      Tensor left = left_step(E, e.left[x], top[x], lc, bottom[x]);
      row_scalar_to(E, left, top[x + 1], ld, bottom[x + 1], e.right[x + 2], 100 + 2 * term);
      left = left_step(E, e.left[x], top[x], row[x], bottom[x]);
      row_scalar_to(E, left, top[x + 1], row[x + 1], bottom[x + 1], e.right[x + 2], 101 + 2 * term);
      ++term;
    }
  }
  int first_vertical = term;
  for (int y = 0; y < Ly - 1; ++y) {
    std::vector<Layer> row(Lx);
    for (int x = 0; x < Lx; ++x) {
      row[x].a = layers[x + y * Lx];
      row[x].b = layers[x + (y + 1) * Lx];
      row[x].slab = true;
    }
    const auto& top = env.north[y].t;
    const auto& bottom = env.south[y + 2].t;
    RowEnvs e = row_environments(E, top, row, bottom, 0);
    for (int x = 0; x < Lx; ++x) {
      const Tensor& A = s.at(x, y);
      const Tensor& B = s.at(x, y + 1);
      Tensor C, D;
      operator_pair(E, A, B, F, G, false, C, D);
      Layer imp;
      imp.a = double_layer(E, C, A);
      imp.b = double_layer(E, D, B);
      imp.slab = true;
      row_scalar_to(E, e.left[x], top[x], row[x], bottom[x], e.right[x + 1], 101 + 2 * term);
      row_scalar_to(E, e.left[x], top[x], imp, bottom[x], e.right[x + 1], 100 + 2 * term);
      ++term;
    }
  }
  SPS_CUDA(cudaMemcpyAsync(E.hscal + 100, E.dscal + 100, sizeof(double) * 2 * nterm, cudaMemcpyDeviceToHost,
                           E.stream));
  E.sync();
  E.check_flag("measure_energy");
  std::vector<double> vals(E.hscal + 100, E.hscal + 100 + 2 * nterm);
  double xsum = 0, zzsum = 0;
  out.site_x.assign(Lx * Ly, 0);
  term = 0;
  for (int y = 0; y < Ly; ++y) {
    for (int x = 0; x < Lx; ++x) {
      double r = real_ratio(vals[2 * term], vals[2 * term + 1]);
      out.site_x[x + y * Lx] = r;
      xsum += r;
      ++term;
    }
    for (int x = 0; x < Lx - 1; ++x) {
      zzsum += real_ratio(vals[2 * term], vals[2 * term + 1]);
      ++term;
    }
  }
  for (term = first_vertical; term < nterm; ++term) zzsum += real_ratio(vals[2 * term], vals[2 * term + 1]);
  const Env& fin = env.north[Ly];
  double ln = std::log(positive_real(close_boundary(E, fin.t), "norm")) + fin.log_scale;
  double hx = m.h * xsum;
  if (!m.fields.empty()) {   // sum_i h_i <X_i>
    hx = 0;
    for (int i = 0; i < Lx * Ly; ++i) hx += m.fields[i] * out.site_x[i];
  }
  out.energy_total = -m.J * zzsum - hx;
  out.energy_per_site = out.energy_total / (Lx * Ly);
  out.log_norm = ln + 2 * s.log_amplitude;
  out.tensor_log_norm = ln;
  out.max_env_trunc = env.max_trunc;
  out.x_sum = xsum;
  out.zz_sum = zzsum;
  return out;
}

}  // namespace sps
