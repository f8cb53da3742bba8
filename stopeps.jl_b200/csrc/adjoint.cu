// Reverse-mode derivative of the row boundary-MPS lognorm with respect to the
// site tensors.  The reference has no derivatives; this is the adjoint of its
// lognorm (src/contraction/boundary_mps.jl:180-186) through double_layer
// (:65-73), _absorb (:136-151), compress_boundary! (:94-134) and
// _close_boundary (:153-163), the first piece of per-site-field gradients.
//
// The truncated state of compress_boundary! depends only on the boundary's
// state, not on the gauge in which it is brought into canonical form, so the
// forward pass here canonicalizes with a full SVD (L = U S, Q = V^T) where the
// reference takes an LQ; every factorization then shares one reverse rule:
// the thin SVD's, per parity block, with the couplings 1 / (s_j^2 - s_i^2)
// split into 1 / (s_j - s_i) and 1 / (s_j + s_i) terms; those and 1 / s are
// Lorentzian-broadened.  (The LQ reverse rule solves with L and loses
// accuracy on numerically rank-deficient boundary blocks; the broadened SVD
// rule does not.)  The truncated SVDs keep the leading columns of the full
// ones, so discarded columns get zero cotangents.
//
// The tape of a row (its factorizations) is the memory of the reverse pass;
// with checkpoint_rows only each row's incoming boundary is kept and the
// row's factorizations are recomputed from it when the reverse pass reaches
// it (the same operations on the same boundary give the same tape).
#include "pipeline.h"
#include <algorithm>
#include <cfloat>

namespace sps {
namespace {

const double BROADENING = 1e-24;

__global__ void hadamard_kernel(const double* __restrict__ a, const double* __restrict__ b, double* __restrict__ c,
                                int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    c[i] = a[i] * b[i];
}

// elementwise product of two tensors with the same legs
Tensor hadamard(Engine& E, const Tensor& A0, const Tensor& B0) {
  Tensor A = contiguous(E, A0), B = contiguous(E, B0);
  if (A.size() != B.size()) throw Error(SPS_ERR_ARGUMENT, "hadamard: size mismatch");
  Tensor C = E.empty(A.legs);
  const int64_t n = C.size();
  if (n) {
    const int blocks = (int)std::min<int64_t>((n + 255) / 256, 148 * 8);
    hadamard_kernel<<<blocks, 256, 0, E.stream>>>(A.ptr(), B.ptr(), C.ptr(), n);
    SPS_CUDA(cudaGetLastError());
    E.launches++;
  }
  return C;
}

struct FullSVD {   // thin SVD of (rows | cols) with every value: U (rows..., K), Vt (K, cols...)
  Tensor U, Vt;
  std::vector<double> s;   // in the order of the K leg (block 0 first)
  Par leg;
};

FullSVD full_svd(Engine& E, const Tensor& A, const std::vector<int>& rows, const std::vector<int>& cols) {
  Trunc all;   // no truncation: every value, zeros with orthonormal completions
  SVDres f = svd(E, A, rows, cols, all, false);
  FullSVD out;
  out.U = f.U;
  out.Vt = f.V;
  out.s = f.S[0];
  out.s.insert(out.s.end(), f.S[1].begin(), f.S[1].end());
  out.leg = f.U.legs.back();
  return out;
}

// a (leg a, leg b) matrix from host values, entries between different
// parities zero
Tensor leg_matrix(Engine& E, const Par& a, const Par& b, std::vector<double> m) {
  const int na = (int)a->size(), nb = (int)b->size();
  for (int i = 0; i < na; ++i)
    for (int j = 0; j < nb; ++j)
      if ((*a)[i] != (*b)[j]) m[(size_t)i * nb + j] = 0.0;
  return E.upload({a, b}, m.data());
}

// reverse rule of the thin SVD A = U diag(s) Vt (every value kept); nrow = 1
// for (l | p r), 2 for (l p | r)
Tensor svd_backward(Engine& E, const FullSVD& f, const Tensor& Ub, const std::vector<double>& sb, const Tensor& Vtb,
                    int nrow) {
  const std::string ru = nrow == 2 ? "lp" : "l", cv = nrow == 2 ? "r" : "pr";
  const int K = (int)f.s.size();
  // the couplings (A_ij s_j + s_i B_ij) / (s_j^2 - s_i^2), A = U^T Ub - Ub^T U,
  // B = V^T Vb - Vb^T V, split as (A + B)_ij / 2 (s_j - s_i) + (A - B)_ij / 2
  // (s_j + s_i): for a gauge-invariant function A + B vanishes with s_j - s_i,
  // so the broadening of 1 / (s_j - s_i) only removes rounding noise
  std::vector<double> Fmv((size_t)K * K, 0.0), Fpv((size_t)K * K, 0.0), D((size_t)K * K, 0.0), sinv(K);
  for (int i = 0; i < K; ++i) {
    D[(size_t)i * K + i] = sb[i];
    sinv[i] = f.s[i] / (f.s[i] * f.s[i] + BROADENING);
    for (int j = 0; j < K; ++j)
      if (i != j) {
        const double dm = f.s[j] - f.s[i], dp = f.s[j] + f.s[i];
        Fmv[(size_t)i * K + j] = 0.5 * dm / (dm * dm + BROADENING);
        Fpv[(size_t)i * K + j] = 0.5 * dp / (dp * dp + BROADENING);
      }
  }
  Tensor Fm = leg_matrix(E, f.leg, f.leg, Fmv), Fp = leg_matrix(E, f.leg, f.leg, Fpv);
  Tensor Dm = leg_matrix(E, f.leg, f.leg, D);
  Tensor X = ein(E, ru + "K," + ru + "L->KL", f.U, Ub);                 // U^T Ub
  Tensor A = axpby(E, 1.0, X, -1.0, perm_view(X, {1, 0}));
  Tensor Y = ein(E, "K" + cv + ",L" + cv + "->KL", f.Vt, Vtb);           // V^T Vb
  Tensor B = axpby(E, 1.0, Y, -1.0, perm_view(Y, {1, 0}));
  Tensor core = axpby(E, 1.0, hadamard(E, Fm, axpby(E, 1.0, A, 1.0, B)), 1.0,
                      hadamard(E, Fp, axpby(E, 1.0, A, -1.0, B)));
  core = axpby(E, 1.0, core, 1.0, Dm);
  const std::string out = ru + cv;
  Tensor Ab = ein(E, ru + "L,L" + cv + "->" + out, ein(E, ru + "K,KL->" + ru + "L", f.U, core), f.Vt);
  // (1 - U U^T) Ub S^-1 Vt: zero where U is square
  Tensor Z = scale_leg(E, Ub, nrow, sinv);
  Tensor UtZ = ein(E, ru + "K," + ru + "L->KL", f.U, Z);
  Tensor Zp = axpby(E, 1.0, Z, -1.0, ein(E, ru + "K,KL->" + ru + "L", f.U, UtZ));
  Ab = axpby(E, 1.0, Ab, 1.0, ein(E, ru + "L,L" + cv + "->" + out, Zp, f.Vt));
  // U S^-1 Vtb (1 - V V^T): zero where V is square
  Tensor W = scale_leg(E, Vtb, 0, sinv);
  Tensor WV = ein(E, "K" + cv + ",L" + cv + "->KL", W, f.Vt);
  Tensor Wp = axpby(E, 1.0, W, -1.0, ein(E, "KL,L" + cv + "->K" + cv, WV, f.Vt));
  Ab = axpby(E, 1.0, Ab, 1.0, ein(E, ru + "K,K" + cv + "->" + out, f.U, Wp));
  return Ab;
}

struct CanonStep {   // B[x] = L Q with L = U S, Q = Vt, then B[x-1] <- B[x-1] L
  FullSVD f;
  Tensor prev, L;
};
struct SweepStep {   // B[x] = U_k, R = S_k Vt_k, B[x+1] <- R B[x+1]
  FullSVD f;
  Tensor P;                   // (K, k): the kept columns
  std::vector<double> sk;
  Tensor Vk, R, next;
};
struct RowTape {
  std::vector<Tensor> env, row;
  std::vector<CanonStep> canon;
  std::vector<SweepStep> sweep;
  Tensor center;
  double scale = 1;
};

}  // namespace

LognormGradient lognorm_gradient(Engine& E, const State& s, const BMPS& m, bool checkpoint_rows) {
  if (m.zipup || m.diagonal || m.variational)
    throw Error(SPS_ERR_ARGUMENT, "the lognorm derivative takes the row method's exact compression");
  const int Lx = s.Lx, Ly = s.Ly;
  Trunc tr;
  tr.chi = m.chi;
  tr.space[0] = m.space[0];
  tr.space[1] = m.space[1];
  std::vector<Tensor> layers(Lx * Ly);
  for (int i = 0; i < Lx * Ly; ++i) layers[i] = double_layer(E, s.sites[i], s.sites[i]);
  // one row's absorption and compression, recorded in rt; returns the new
  // boundary (centre normalised) and leaves the centre's norm in rt.scale
  auto forward_row = [&](RowTape& rt) {
    std::vector<Tensor> B(Lx);
    for (int x = 0; x < Lx; ++x)
      B[x] = fuse(E, fuse(E, ein(E, "lnr,wnep->lwpre", rt.env[x], rt.row[x]), 3, 2), 0, 2);
    rt.canon.assign(Lx, CanonStep());
    for (int x = Lx - 1; x >= 1; --x) {
      CanonStep& c = rt.canon[x];
      c.f = full_svd(E, B[x], {0}, {1, 2});
      c.L = scale_leg(E, c.f.U, 1, c.f.s);
      c.prev = B[x - 1];
      B[x] = c.f.Vt;
      B[x - 1] = ein(E, "lpk,kr->lpr", B[x - 1], c.L);
    }
    rt.sweep.assign(Lx, SweepStep());
    for (int x = 0; x + 1 < Lx; ++x) {
      SweepStep& w = rt.sweep[x];
      w.f = full_svd(E, B[x], {0, 1}, {2});
      // the kept set of the truncation: a prefix of each parity block
      std::vector<double> sv[2];
      std::vector<int> pos[2];
      for (int i = 0; i < (int)w.f.s.size(); ++i) {
        sv[(*w.f.leg)[i]].push_back(w.f.s[i]);
        pos[(*w.f.leg)[i]].push_back(i);
      }
      std::vector<char> kp[2];
      truncation_keep(sv, tr, kp);
      int kk[2] = {0, 0};
      for (int c = 0; c < 2; ++c)
        for (size_t i = 0; i < kp[c].size(); ++i)
          if (kp[c][i]) {
            if ((int)i != kk[c]) throw Error(SPS_ERR_NUMERIC, "lognorm derivative: non-prefix truncation");
            kk[c]++;
          }
      Par kleg = make_par(kk[0], kk[1]);
      const int K = (int)w.f.s.size(), k = kk[0] + kk[1];
      std::vector<double> P((size_t)K * k, 0.0);
      for (int c = 0, col = 0; c < 2; ++c)
        for (int i = 0; i < kk[c]; ++i, ++col) {
          P[(size_t)pos[c][i] * k + col] = 1.0;
          w.sk.push_back(sv[c][i]);
        }
      w.P = E.upload({w.f.leg, kleg}, P.data());
      Tensor Uk = ein(E, "lpK,Kk->lpk", w.f.U, w.P);
      w.Vk = ein(E, "Kk,Kr->kr", w.P, w.f.Vt);
      w.R = scale_leg(E, w.Vk, 0, w.sk);
      w.next = B[x + 1];
      B[x] = Uk;
      B[x + 1] = ein(E, "lk,kpr->lpr", w.R, B[x + 1]);
    }
    rt.center = B[Lx - 1];
    rt.scale = norm(E, B[Lx - 1]);
    if (!(std::isfinite(rt.scale) && rt.scale > 0)) throw Error(SPS_ERR_NUMERIC, "nonfinite boundary norm");
    B[Lx - 1] = clone(E, B[Lx - 1]);
    scale_inplace(E, B[Lx - 1], 1.0 / rt.scale);
    return B;
  };
  std::vector<Tensor> firstrow(layers.begin(), layers.begin() + Lx);
  std::vector<Tensor> env = trivial_boundary(E, firstrow, true).t;
  double log_scale = 0;
  std::vector<RowTape> tape(Ly);
  for (int y = 0; y < Ly; ++y) {
    RowTape& rt = tape[y];
    rt.env = env;
    rt.row.assign(layers.begin() + y * Lx, layers.begin() + (y + 1) * Lx);
    env = forward_row(rt);
    log_scale += std::log(rt.scale);
    if (checkpoint_rows) {   // keep the row's incoming boundary only
      rt.canon.clear();
      rt.sweep.clear();
      rt.center = Tensor();
    }
  }
  // close (_close_boundary) on the host: the last boundary has one-state
  // physical legs, V_{x+1} = V_x A_x[:, 0, :], value = sum V_Lx
  std::vector<std::vector<double>> host(Lx), vecs(Lx + 1);
  vecs[0].assign(env[0].dims[0], 1.0);
  for (int x = 0; x < Lx; ++x) {
    if (env[x].dims[1] != 1) throw Error(SPS_ERR_ARGUMENT, "open boundary physical leg at the lattice edge");
    host[x] = E.download(env[x]);
    const int64_t a = env[x].dims[0], b = env[x].dims[2];
    vecs[x + 1].assign(b, 0.0);
    for (int64_t i = 0; i < a; ++i)
      for (int64_t j = 0; j < b; ++j) vecs[x + 1][j] += vecs[x][i] * host[x][i * b + j];
  }
  double closed = 0;
  for (double v : vecs[Lx]) closed += v;
  LognormGradient out;
  out.log_norm = std::log(positive_real(closed, "norm")) + log_scale + 2 * s.log_amplitude;
  std::vector<Tensor> envbar(Lx);
  std::vector<double> vb(vecs[Lx].size(), 1.0 / closed);
  for (int x = Lx - 1; x >= 0; --x) {
    const int64_t a = env[x].dims[0], b = env[x].dims[2];
    std::vector<double> g((size_t)a * b);
    std::vector<double> nvb(a, 0.0);
    for (int64_t i = 0; i < a; ++i)
      for (int64_t j = 0; j < b; ++j) {
        g[i * b + j] = vecs[x][i] * vb[j];
        nvb[i] += host[x][i * b + j] * vb[j];
      }
    envbar[x] = E.upload(env[x].legs, g.data());
    vb = nvb;
  }
  std::vector<Tensor> layerbar(Lx * Ly);
  for (int y = Ly - 1; y >= 0; --y) {
    RowTape& rt = tape[y];
    if (checkpoint_rows) forward_row(rt);   // the same operations on the same boundary
    std::vector<Tensor> Bb = envbar;
    // centre normalisation: out = B / s, and log s enters the value with weight 1
    {
      Tensor o = clone(E, rt.center);
      scale_inplace(E, o, 1.0 / rt.scale);
      const double go = dot(E, Bb[Lx - 1], o);
      Tensor t = axpby(E, 1.0, Bb[Lx - 1], 1.0 - go, o);
      scale_inplace(E, t, 1.0 / rt.scale);
      Bb[Lx - 1] = t;
    }
    for (int x = Lx - 2; x >= 0; --x) {
      SweepStep& w = rt.sweep[x];
      const Tensor G = Bb[x + 1];
      Tensor Rb = ein(E, "lpr,kpr->lk", G, w.next);
      Bb[x + 1] = ein(E, "lk,lpr->kpr", w.R, G);
      // R = S_k Vt_k: sbar_i = sum_j Rb_ij Vk_ij, Vkbar = S_k Rb
      Tensor RV = ein(E, "kr,Kr->kK", Rb, w.Vk);
      std::vector<double> rv = E.download(contiguous(E, RV));
      const int k = (int)w.sk.size(), K = (int)w.f.s.size();
      std::vector<double> sbk(k);
      for (int i = 0; i < k; ++i) sbk[i] = rv[(size_t)i * k + i];
      Tensor Vkb = scale_leg(E, Rb, 0, w.sk);
      // pad to the full SVD: discarded columns carry no cotangent
      Tensor Ubf = ein(E, "lpk,Kk->lpK", Bb[x], w.P);
      Tensor Vtbf = ein(E, "Kk,kr->Kr", w.P, Vkb);
      std::vector<double> P = E.download(contiguous(E, w.P)), sbf(K, 0.0);
      for (int i = 0; i < K; ++i)
        for (int j = 0; j < k; ++j)
          if (P[(size_t)i * k + j] != 0) sbf[i] = sbk[j];
      Bb[x] = svd_backward(E, w.f, Ubf, sbf, Vtbf, 2);
    }
    for (int x = 1; x < Lx; ++x) {
      CanonStep& c = rt.canon[x];
      const Tensor G = Bb[x - 1];
      Tensor Lb = ein(E, "lpr,lpk->kr", G, c.prev);
      Bb[x - 1] = ein(E, "lpr,kr->lpk", G, c.L);
      // L = U S: Ubar = Lbar S, sbar_i = (U^T Lbar)_ii; Q = Vt: Vtbar = Qbar
      Tensor Ub = scale_leg(E, Lb, 1, c.f.s);
      Tensor UL = ein(E, "lK,lL->KL", c.f.U, Lb);
      std::vector<double> ul = E.download(contiguous(E, UL));
      const int K = (int)c.f.s.size();
      std::vector<double> sb(K);
      for (int i = 0; i < K; ++i) sb[i] = ul[(size_t)i * K + i];
      Bb[x] = svd_backward(E, c.f, Ub, sb, Bb[x], 1);
    }
    if (checkpoint_rows) {
      rt.canon.clear();
      rt.sweep.clear();
    }
    for (int x = 0; x < Lx; ++x) {
      Tensor C = ein(E, "lnr,wnep->lwpre", rt.env[x], rt.row[x]);
      // the fused legs are the row-major reshape of C's: split them back
      if (Bb[x].size() != C.size()) throw Error(SPS_ERR_ARGUMENT, "lognorm derivative: boundary size");
      Tensor Cb = split(E, contiguous(E, Bb[x]), 2, {C.legs[3], C.legs[4]});
      Cb = split(E, Cb, 0, {C.legs[0], C.legs[1]});
      envbar[x] = ein(E, "lwpre,wnep->lnr", Cb, rt.row[x]);
      layerbar[x + y * Lx] = ein(E, "lwpre,lnr->wnep", Cb, rt.env[x]);
    }
  }
  for (int i = 0; i < Lx * Ly; ++i) {
    const Tensor& A = s.sites[i];
    Tensor Db = contiguous(E, layerbar[i]);
    const int ax[4] = {0, 1, 4, 5};
    for (int k = 3; k >= 0; --k) {
      if (*Db.legs[k] != *fused_par({A.legs[ax[k]], A.legs[ax[k]]}))
        throw Error(SPS_ERR_ARGUMENT, "lognorm derivative: layer legs do not match the site");
      Db = split(E, Db, k, {A.legs[ax[k]], A.legs[ax[k]]});
    }
    Tensor g1 = ein(E, "wWnNeEsS,WNpaES->wnpaes", Db, A);
    Tensor g2 = ein(E, "wWnNeEsS,wnpaes->WNpaES", Db, A);
    out.grads.push_back(axpby(E, 1.0, g1, 1.0, g2));
  }
  E.check_flag("lognorm derivative");
  return out;
}

FieldGradient lognorm_field_gradient(Engine& E, const State& s, const BMPS& m, bool checkpoint_rows) {
  LognormGradient g = lognorm_gradient(E, s, m, checkpoint_rows);
  FieldGradient out;
  out.log_norm = g.log_norm;
  const std::vector<double> X = {1.0, -1.0};   // X on the physical leg in the Z2 basis
  for (size_t i = 0; i < s.sites.size(); ++i) {
    const Tensor& A = s.sites[i];
    if (A.dims[2] != 2) throw Error(SPS_ERR_ARGUMENT, "field derivative: the physical leg is not a spin");
    // lnZ along A_i -> A_i + e X A_i grows by 2 e <X_i>
    const double x = 0.5 * dot(E, g.grads[i], scale_leg(E, A, 2, X));
    out.site_x.push_back(x);
    out.d_fields.push_back(s.beta * x);
  }
  return out;
}

}  // namespace sps
