// Full update on the Z2 engine: environment-gauged two-site ALS with
// Jacobi-preconditioned CG solves, QR/LQ centre motion, bond balancing and the
// full-hole PSD repair.  Restates src/evolution/full_update.jl (whole file)
// for the row boundary-MPS contraction.
#include "pipeline.h"
#include <algorithm>
#include <cfloat>

namespace sps {

static const double EPS = DBL_EPSILON;
static const double FLOATMIN = DBL_MIN;
static const double RESIDUAL_ROUNDOFF_TOLERANCE = 1e-8;

// ---------------------------------------------------------------------------
// host 4x4 symmetric exponential for the Trotter gate (src/models/tfim.jl:44-48)
// ---------------------------------------------------------------------------
static void jacobi_sym(int n, double* a, double* v, double* w) {
  for (int i = 0; i < n * n; ++i) v[i] = (i % (n + 1) == 0) ? 1.0 : 0.0;
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0;
    for (int p = 0; p < n; ++p)
      for (int q = p + 1; q < n; ++q) off += a[p * n + q] * a[p * n + q];
    if (off == 0) break;
    for (int p = 0; p < n; ++p)
      for (int q = p + 1; q < n; ++q) {
        double apq = a[p * n + q];
        if (apq == 0) continue;
        double zeta = (a[q * n + q] - a[p * n + p]) / (2 * apq);
        double t = std::copysign(1.0, zeta) / (std::fabs(zeta) + std::hypot(1.0, zeta));
        double c = 1 / std::sqrt(1 + t * t), s = c * t;
        for (int k = 0; k < n; ++k) {  // A <- A J
          double x = a[k * n + p], y = a[k * n + q];
          a[k * n + p] = c * x - s * y;
          a[k * n + q] = s * x + c * y;
        }
        for (int k = 0; k < n; ++k) {  // A <- J^T A
          double x = a[p * n + k], y = a[q * n + k];
          a[p * n + k] = c * x - s * y;
          a[q * n + k] = s * x + c * y;
        }
        for (int k = 0; k < n; ++k) {
          double x = v[k * n + p], y = v[k * n + q];
          v[k * n + p] = c * x - s * y;
          v[k * n + q] = s * x + c * y;
        }
      }
  }
  for (int i = 0; i < n; ++i) w[i] = a[i * n + i];
}

static int degree(int Lx, int Ly, int x, int y) {
  return (x > 0) + (x < Lx - 1) + (y > 0) + (y < Ly - 1);
}

Tensor trotter_gate(Engine& E, const Model& m, int Lx, int Ly, int ax, int ay, int bx, int by, double delta) {
  // H[p,q,u,v] = -J z z - h/deg_a X(x)I - h/deg_b I(x)X, Z2 basis: X = diag(1,-1), z flips parity
  double X[2] = {1, -1};
  double H[16] = {0};
  double da = degree(Lx, Ly, ax, ay), db = degree(Lx, Ly, bx, by);
  const double ha = m.field(ax, ay, Lx), hb = m.field(bx, by, Lx);   // each site's own field
  for (int p = 0; p < 2; ++p)
    for (int q = 0; q < 2; ++q)
      for (int u = 0; u < 2; ++u)
        for (int v = 0; v < 2; ++v) {
          double zz = (p != u && q != v) ? 1.0 : 0.0;
          double xa = (p == u && q == v) ? X[p] : 0.0;
          double xb = (p == u && q == v) ? X[q] : 0.0;
          H[(p * 2 + q) * 4 + (u * 2 + v)] = -m.J * zz - ha / da * xa - hb / db * xb;
        }
  double V[16], w[4], A[16];
  std::copy(H, H + 16, A);
  jacobi_sym(4, A, V, w);
  double G[16];
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) {
      double s = 0;
      for (int k = 0; k < 4; ++k) s += V[i * 4 + k] * std::exp(-delta * w[k]) * V[j * 4 + k];
      G[i * 4 + j] = s;
    }
  Par p2 = make_par(1, 1);
  return E.upload({p2, p2, p2, p2}, G);
}

// ---------------------------------------------------------------------------
// device CG (_solve_core, full_update.jl:371-400): one CTA, operator n x n
// acting on n x P right-hand sides; no host round trip per iteration.
// ---------------------------------------------------------------------------
static constexpr int CG_T = 256;

__device__ double cg_block_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0;
    for (int w = 0; w < CG_T / 32; ++w) s += red[w];
    red[32] = s;
  }
  __syncthreads();
  return red[32];
}

__global__ void __launch_bounds__(CG_T) cg_kernel(const double* __restrict__ M, const double* __restrict__ b,
                                                  const double* __restrict__ x0, double* __restrict__ x,
                                                  double* work, int n, int P, double diag_shift, int maxit,
                                                  double tol, double* out_residual) {
  __shared__ double red[33];
  const int nv = n * P;
  double* den = work;
  double* r = den + n;
  double* z = r + nv;
  double* p = z + nv;
  double* Ap = p + nv;
  double lm = 0;
  for (int i = threadIdx.x; i < n; i += CG_T) {
    double d = fmax(M[(size_t)i * n + i], 0.0);
    den[i] = d;
    lm = fmax(lm, d);
  }
  // block max
  for (int o = 16; o > 0; o >>= 1) lm = fmax(lm, __shfl_xor_sync(0xffffffffu, lm, o));
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = lm;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0;
    for (int w = 0; w < CG_T / 32; ++w) s = fmax(s, red[w]);
    red[32] = s;
  }
  __syncthreads();
  const double scale = red[32];
  const double shift = diag_shift * fmax(scale, DBL_MIN);
  const double floor_ = fmax(fmax(shift, DBL_EPSILON * scale), DBL_MIN);
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += CG_T) den[i] = fmax(den[i] + shift, floor_);
  for (int e = threadIdx.x; e < nv; e += CG_T) x[e] = x0[e];
  __syncthreads();
  // r = b - (M x + shift x)
  double bb = 0, rr = 0;
  for (int e = threadIdx.x; e < nv; e += CG_T) {
    int i = e / P, c = e % P;
    double s = 0;
    for (int j = 0; j < n; ++j) s += M[(size_t)i * n + j] * x[j * P + c];
    double re = b[e] - (s + shift * x[e]);
    r[e] = re;
    rr += re * re;
    bb += b[e] * b[e];
  }
  const double rhsnorm = fmax(sqrt(cg_block_sum(bb, red)), DBL_MIN);
  double residual = sqrt(cg_block_sum(rr, red)) / rhsnorm;
  if (!(residual <= tol)) {
    double rz = 0;
    for (int e = threadIdx.x; e < nv; e += CG_T) {
      double ze = r[e] / den[e / P];
      z[e] = ze;
      p[e] = ze;
      rz += r[e] * ze;
    }
    rz = cg_block_sum(rz, red);
    for (int it = 0; it < maxit; ++it) {
      double pap = 0, pp = 0, aa = 0;
      for (int e = threadIdx.x; e < nv; e += CG_T) {
        int i = e / P, c = e % P;
        double s = 0;
        for (int j = 0; j < n; ++j) s += M[(size_t)i * n + j] * p[j * P + c];
        s += shift * p[e];
        Ap[e] = s;
        pap += p[e] * s;
        pp += p[e] * p[e];
        aa += s * s;
      }
      double curvature = cg_block_sum(pap, red);
      double pn = sqrt(cg_block_sum(pp, red));
      double an = sqrt(cg_block_sum(aa, red));
      if (!(curvature > DBL_EPSILON * fmax(pn * an, DBL_MIN))) break;
      double alpha = rz / curvature;
      double r2 = 0;
      for (int e = threadIdx.x; e < nv; e += CG_T) {
        x[e] += alpha * p[e];
        double re = r[e] - alpha * Ap[e];
        r[e] = re;
        r2 += re * re;
      }
      residual = sqrt(cg_block_sum(r2, red)) / rhsnorm;
      if (residual <= tol) break;
      double nx = 0;
      for (int e = threadIdx.x; e < nv; e += CG_T) {
        double ze = r[e] / den[e / P];
        z[e] = ze;
        nx += r[e] * ze;
      }
      nx = cg_block_sum(nx, red);
      if (!(nx >= 0)) break;
      double beta = nx / fmax(rz, DBL_MIN);
      for (int e = threadIdx.x; e < nv; e += CG_T) p[e] = z[e] + beta * p[e];
      rz = nx;
      __syncthreads();
    }
  }
  if (threadIdx.x == 0) *out_residual = residual;
}

// returns the solution tensor (legs of rhs); residual left in device slot
static Tensor solve_core(Engine& E, const Tensor& normal, const Tensor& rhs, const Tensor& initial,
                         const FUOptions& o, int slot) {
  Tensor M = contiguous(E, normal), b = contiguous(E, rhs), x0 = contiguous(E, initial);
  int n = (int)(M.dims[0] * M.dims[1]);
  int P = (int)b.dims[2];
  if (M.dims[2] * M.dims[3] != n || b.dims[0] * b.dims[1] != n) throw Error(SPS_ERR_ARGUMENT, "solve_core: shape");
  Tensor x = E.empty(b.legs);
  Buf w = E.alloc(sizeof(double) * (n + 4 * n * P + 8));
  int tk = E.tic("cg");
  cg_kernel<<<1, CG_T, 0, E.stream>>>(M.ptr(), b.ptr(), x0.ptr(), x.ptr(), (double*)w->ptr, n, P,
                                      o.diagonal_shift, o.linear_max_iterations, o.linear_tolerance,
                                      E.dscal + slot);
  E.toc(tk);
  SPS_CUDA(cudaGetLastError());
  E.launches++;
  return x;
}

// ---------------------------------------------------------------------------
// FU pieces
// ---------------------------------------------------------------------------
static const std::array<int, 6> PA_H{0, 1, 5, 3, 2, 4}, PA_V{0, 1, 4, 3, 2, 5};
static const std::array<int, 6> PB_H{1, 4, 5, 3, 2, 0}, PB_V{0, 4, 5, 3, 2, 1};

static std::vector<int> invperm(const std::array<int, 6>& p) {
  std::vector<int> o(6);
  for (int i = 0; i < 6; ++i) o[p[i]] = i;
  return o;
}

struct Pair {
  Tensor Qa, Qb, target;
  std::array<int, 6> pa, pb;
  Tensor left, right, wt, wm, Li, Ri;
};

// _reduced_pair (full_update.jl:21-29)
static Pair reduced_pair(Engine& E, const Tensor& A, const Tensor& B, const Tensor& gate, bool horizontal) {
  Pair p;
  p.pa = horizontal ? PA_H : PA_V;
  p.pb = horizontal ? PB_H : PB_V;
  QRres a = qr(E, perm_view(A, {p.pa.begin(), p.pa.end()}), {0, 1, 2, 3}, {4, 5});
  QRres b = qr(E, perm_view(B, {p.pb.begin(), p.pb.end()}), {0, 1, 2, 3}, {4, 5});
  p.Qa = a.Q;
  p.Qb = b.Q;
  Tensor bb = perm_view(b.R, {2, 1, 0});
  Tensor X = ein(E, "ruk,kvs->ruvs", a.R, bb);
  p.target = ein(E, "ruvs,pquv->rpqs", X, gate);
  return p;
}

static Tensor concat_scale_leg(Engine& E, const Tensor& T, int axis, const std::vector<double> s[2],
                               bool root) {
  std::vector<double> v(s[0]);
  v.insert(v.end(), s[1].begin(), s[1].end());
  if (root)
    for (auto& x : v) x = std::sqrt(x);
  return scale_leg(E, T, axis, v);
}

// _fu_svd_initial (full_update.jl:31-42)
static void fu_svd_initial(Engine& E, const Tensor& target, int D, const int space[2], Tensor& left,
                           Tensor& right) {
  int64_t maxdim = *std::max_element(target.dims.begin(), target.dims.end());
  double cutoff = EPS * (double)maxdim * norm(E, target);
  Trunc tr;
  tr.chi = D;
  tr.space[0] = space[0];
  tr.space[1] = space[1];
  tr.atol = cutoff;
  SVDres f = svd(E, target, {0, 1}, {2, 3}, tr);
  if (f.S[0].size() + f.S[1].size() == 0) throw Error(SPS_ERR_NUMERIC, "gate produced a zero target");
  left = concat_scale_leg(E, f.U, 2, f.S, true);
  right = concat_scale_leg(E, f.V, 0, f.S, true);
}

// _fu_balance_bond (full_update.jl:45-52)
static void fu_balance_bond(Engine& E, const Tensor& QA, const Tensor& C, const Tensor& QB, Tensor& A,
                            Tensor& B) {
  SVDres f = svd(E, C, {0}, {1}, Trunc{});
  Tensor Ur = concat_scale_leg(E, f.U, 1, f.S, true);
  Tensor Vr = concat_scale_leg(E, f.V, 0, f.S, true);
  A = ein(E, "fpb,bk->fpk", QA, Ur);
  B = ein(E, "kb,bqs->kqs", Vr, QB);
}

// _fu_transform_metric (full_update.jl:55-62)
static Tensor fu_transform_metric(Engine& E, const Tensor& N, const Tensor& Li, const Tensor& Ri) {
  Tensor first = ein(E, "ijkl,ix->jklx", N, Li);
  Tensor second = ein(E, "jklx,jy->klxy", first, Ri);
  Tensor third = ein(E, "klxy,kz->lxyz", second, Li);
  return ein(E, "lxyz,lw->xyzw", third, Ri);
}

// _fu_environment_gauge (full_update.jl:72-106)
static void fu_environment_gauge(Engine& E, const Tensor& N, Pair& p) {
  if (!all_finite(E, N)) throw Error(SPS_ERR_NUMERIC, "nonfinite FU norm metric");
  double scale = norm(E, N);
  if (!(scale > 0)) throw Error(SPS_ERR_NUMERIC, "zero FU norm metric");
  Tensor NT = perm_view(N, {2, 3, 0, 1});
  Tensor H = axpby(E, 0.5 / scale, N, 0.5 / scale, NT);
  EIGres eg = eigh(E, H, {0, 1}, {2, 3});
  double spectral = 0;
  for (int c = 0; c < 2; ++c)
    for (double v : eg.w[c]) spectral = std::max(spectral, std::fabs(v));
  double relative_floor = std::max(std::sqrt(EPS), (double)(N.dims[2] * N.dims[3]) * EPS);
  if (spectral == 0) spectral = 1;
  double fl = relative_floor * spectral;
  std::vector<double> root;
  for (int c = 0; c < 2; ++c)
    for (double v : eg.w[c]) root.push_back(std::sqrt(std::max(v, fl)));
  Tensor Z = scale_leg(E, perm_view(eg.V, {2, 0, 1}), 0, root);   // (eig, rb, sb)
  Tensor left = qr(E, Z, {0, 2}, {1}).R;
  Tensor right = qr(E, Z, {0, 1}, {2}).R;
  p.Li = block_inverse(E, left);
  p.Ri = block_inverse(E, right);
  E.check_flag("fu_environment_gauge");
  p.wm = fu_transform_metric(E, N, p.Li, p.Ri);
  // working target: left on leg 0, right on leg 3
  Tensor t1 = ein(E, "xr,rpqs->xpqs", left, p.target);
  p.wt = ein(E, "rpqz,yz->rpqy", t1, right);
}

static void initialize_pair(Engine& E, Pair& p, const Tensor& N, int D, const int space[2]) {
  fu_environment_gauge(E, N, p);
  fu_svd_initial(E, p.wt, D, space, p.left, p.right);
}

static void original_cores(Engine& E, const Pair& p, const Tensor& A, const Tensor& B, Tensor& oA, Tensor& oB) {
  oA = ein(E, "xk,kpb->xpb", p.Li, A);
  oB = ein(E, "bqk,yk->bqy", B, p.Ri);
}

static void restore_pair(Engine& E, const Pair& p, const Tensor& A, const Tensor& B, Tensor& sa, Tensor& sb) {
  Tensor first = ein(E, "uvwar,rpb->uvwapb", p.Qa, A);
  Tensor second = ein(E, "uvwar,bpr->uvwapb", p.Qb, B);
  sa = perm(E, first, invperm(p.pa));
  sb = perm(E, second, invperm(p.pb));
}

// X contracted over its legs x1, x2 with the reduced layer of Q
// (_reduced_layer, full_update.jl:143-149: Q (x) Q over the auxiliary leg, the
// outer legs' (ket, bra) pairs fused) on Q's outer legs q1, q2: the ket Q, then
// the bra Q, never forming the d^3 r^2 layer.  Returns X's other legs in order,
// then the fused pair of Q's remaining outer leg, then (bra bond, ket bond).
// Q legs: three outer legs, auxiliary, reduced bond.
static Tensor reduced_apply(Engine& E, const Tensor& X, int x1, int x2, const Tensor& Q, int q1, int q2) {
  const int q3 = 3 - q1 - q2;
  const int hi = std::max(x1, x2), lo = std::min(x1, x2);
  const Par phi = Q.legs[hi == x1 ? q1 : q2], plo = Q.legs[lo == x1 ? q1 : q2];
  Tensor S = split(E, split(E, X, hi, {phi, phi}), lo, {plo, plo});
  auto ket_pos = [&](int x) { return x == lo ? lo : hi + 1; };   // bra half right after it
  const int k1 = ket_pos(x1), k2 = ket_pos(x2);
  std::string sx(S.rank(), '?'), fr;
  char c = 'a';
  for (int i = 0; i < S.rank(); ++i)
    if (i != k1 && i != k1 + 1 && i != k2 && i != k2 + 1) {
      sx[i] = c;
      fr += c;
      ++c;
    }
  sx[k1] = 'P';
  sx[k1 + 1] = 'Q';
  sx[k2] = 'R';
  sx[k2 + 1] = 'S';
  std::string qk(5, '?'), qb(5, '?');
  qk[q1] = 'P';
  qk[q2] = 'R';
  qk[q3] = 'T';
  qk[3] = 'U';
  qk[4] = 'K';
  qb[q1] = 'Q';
  qb[q2] = 'S';
  qb[q3] = 'V';
  qb[3] = 'U';
  qb[4] = 'B';
  const std::string y1 = fr + "QSTUK", y2 = fr + "TVBK";
  Tensor Y1 = ein(E, sx + "," + qk + "->" + y1, S, Q);
  Tensor Y2 = ein(E, y1 + "," + qb + "->" + y2, Y1, Q);
  return fuse(E, Y2, (int)fr.size(), 2);
}

struct BondEnv {
  Tensor left, right;
  std::vector<Tensor> top, bottom;
  std::vector<Par> outer;
  bool horizontal;
};

// _reduced_metric(::BondEnvironment) (full_update.jl:151-172), N[B,S,K,P]
// (bra bonds of a and b, ket bonds of a and b).  The reduced layers enter
// through reduced_apply; the vertical bond joins the right and bottom
// environments first (Rh) and contracts the upper and lower halves once,
// which is the same sum as the reference's order with far smaller GEMMs.
static Tensor reduced_metric(Engine& E, const BondEnv& env, const Tensor& Qa, const Tensor& Qb) {
  if (env.horizontal) {
    Tensor X = ein(E, "awb,anc->bncw", env.left, env.top[0]);
    Tensor Y = reduced_apply(E, X, 3, 1, Qa, 0, 1);                 // (b c s B K)
    Tensor L = ein(E, "bcsBK,bsf->cfBK", Y, env.bottom[0]);
    Tensor U = ein(E, "deg,cvd->cveg", env.right, env.top[1]);
    Tensor V = reduced_apply(E, U, 1, 2, Qb, 0, 1);                 // (c g t S P)
    Tensor R = ein(E, "cgtSP,ftg->cfSP", V, env.bottom[1]);
    return ein(E, "cfBK,cfSP->BSKP", L, R);
  }
  Tensor X = ein(E, "awvb,anc->wvbnc", env.left, env.top[0]);
  Tensor Y = reduced_apply(E, X, 0, 3, Qa, 0, 1);                   // (v b c e B K)
  Tensor RB = ein(E, "cefd,bsd->cefbs", env.right, env.bottom[0]);
  Tensor Rh = reduced_apply(E, RB, 2, 4, Qb, 1, 2);                 // (c e b v S P)
  return ein(E, "vbceBK,cebvSP->BSKP", Y, Rh);
}

// bond_hole (boundary_mps.jl:331-350): 12 legs (ket,bra) x 6
static Tensor bond_hole(Engine& E, const BondEnv& env) {
  Tensor H;
  if (env.horizontal) {
    Tensor X = ein(E, "awb,anc->wbnc", env.left, env.top[0]);
    Tensor L = ein(E, "wbnc,bsf->cwnfs", X, env.bottom[0]);
    Tensor Y = ein(E, "deg,cvd->cveg", env.right, env.top[1]);
    Tensor R = ein(E, "cveg,ftg->cveft", Y, env.bottom[1]);
    H = ein(E, "cwnfs,cveft->wnsvet", L, R);
  } else {
    Tensor L = ein(E, "awvb,anc->wvbnc", env.left, env.top[0]);
    Tensor R = ein(E, "bsd,cefd->bscef", env.bottom[0], env.right);
    H = ein(E, "wvbnc,bscef->wnevfs", L, R);
  }
  H = contiguous(E, H);
  for (int k = 5; k >= 0; --k) H = split(E, H, k, {env.outer[k], env.outer[k]});
  return H;
}

// _positive_reduced_metric (full_update.jl:278-340): PSD projection of the
// complete hole (scaled by its Frobenius norm), reduced with Qa and Qb.
static Tensor positive_reduced_metric(Engine& E, const Tensor& H, const Tensor& Qa, const Tensor& Qb) {
  if (!all_finite(E, H)) throw Error(SPS_ERR_NUMERIC, "nonfinite norm metric");
  double scale = norm(E, H);
  std::vector<int> bk{1, 3, 5, 7, 9, 11, 0, 2, 4, 6, 8, 10};
  Tensor Hm = contiguous(E, perm_view(H, bk));                     // (bras..., kets...)
  Tensor HmT = perm_view(Hm, {6, 7, 8, 9, 10, 11, 0, 1, 2, 3, 4, 5});
  double f = scale != 0 ? 0.5 / scale : 0.5;
  Tensor Hs = axpby(E, f, Hm, f, HmT);   // symmetric, Frobenius norm <= 1
  const std::vector<int> bras{0, 1, 2, 3, 4, 5}, kets{6, 7, 8, 9, 10, 11};
  int64_t half = 1;
  for (int k = 0; k < 6; ++k) half *= Hs.dims[k];
  // the parity blocks hold about half the fused states each
  EIGres eg = (half / 2 >= E.eigh_multi_min) ? eigh_unit_shifted(E, Hs, bras, kets) : eigh(E, Hs, bras, kets);
  std::vector<double> wpos;
  for (int c = 0; c < 2; ++c)
    for (double v : eg.w[c]) wpos.push_back(v > 0 ? v : 0.0);
  Tensor Vw = scale_leg(E, eg.V, 6, wpos);
  Tensor Hp = ein(E, "abcdefz,ABCDEFz->abcdefABCDEF", Vw, eg.V);   // (bras, kets)
  // N[rb,sb;rk,sk] = Hp[bras; kets] Qa(kets 1-3) Qa(bras 1-3) Qb(kets 4-6) Qb(bras 4-6)
  Tensor X1 = ein(E, "ABCDEFabcdef,abcuK->ABCDEFdefuK", Hp, Qa);
  Tensor X2 = ein(E, "ABCDEFdefuK,ABCuk->DEFdefKk", X1, Qa);
  Tensor X3 = ein(E, "DEFdefKk,defvS->DEFKkvS", X2, Qb);
  return ein(E, "DEFKkvS,DEFvs->ksKS", X3, Qb);
}

static Tensor apply_pair_metric(Engine& E, const Tensor& N, const Tensor& th) {
  return ein(E, "rstu,tpqu->rpqs", N, th);
}

static double residual_cost(Engine& E, const Tensor& N, const Tensor& A, const Tensor& B, const Tensor& target) {
  Tensor pr = ein(E, "rpb,bqs->rpqs", A, B);
  Tensor res = axpby(E, 1.0, pr, -1.0, target);
  return dot(E, res, apply_pair_metric(E, N, res));
}

static const char* repair_trigger(double raw, double target) {
  double scale = std::max(std::fabs(target), FLOATMIN);
  if (!(std::isfinite(raw) && std::isfinite(target))) throw Error(SPS_ERR_NUMERIC, "nonfinite FU residual/target");
  if (raw / scale < -RESIDUAL_ROUNDOFF_TOLERANCE) return "negative_residual";
  if (target < 0) return "negative_target_norm";
  return nullptr;
}

struct CostEval { double cost; bool fallback; double rel; };
static CostEval cost_evaluation(double raw, double target) {
  double rel = raw / std::max(std::fabs(target), FLOATMIN);
  if (!std::isfinite(rel)) throw Error(SPS_ERR_NUMERIC, "nonfinite relative FU residual");
  if (rel < -RESIDUAL_ROUNDOFF_TOLERANCE) throw Error(SPS_ERR_NUMERIC, "negative FU residual needs PSD repair");
  return {std::fabs(rel), rel < 0, rel};
}

static void left_normal_equation(Engine& E, const Tensor& metric, const Tensor& right, const Tensor& wt,
                                 Tensor& normal, Tensor& rhs) {
  Tensor X = ein(E, "fsgn,bps->fgnbp", metric, right);
  normal = ein(E, "fgnbp,opn->fbgo", X, right);
  rhs = perm(E, ein(E, "fpqs,bqs->fpb", wt, right), {0, 2, 1});
}

static void right_normal_equation(Engine& E, const Tensor& metric, const Tensor& left, const Tensor& wt,
                                  Tensor& normal, Tensor& rhs) {
  Tensor X = ein(E, "wsen,wpb->senpb", metric, left);
  normal = ein(E, "senpb,epo->bson", X, left);
  rhs = perm(E, ein(E, "wqps,wqb->bps", wt, left), {0, 2, 1});
}

struct Fit {
  const char* trigger = nullptr;
  Tensor left, right;
  BondReport rep;
};

// _optimize_pair (full_update.jl:418-482)
static Fit optimize_pair(Engine& E, const Pair& p, const Tensor& N, const FUOptions& o) {
  Fit fit;
  Tensor A = p.left, B = p.right;
  double target_norm = dot(E, p.target, apply_pair_metric(E, N, p.target));
  Tensor oA, oB;
  original_cores(E, p, A, B, oA, oB);
  double raw = residual_cost(E, N, oA, oB, p.target);
  fit.trigger = repair_trigger(raw, target_norm);
  if (fit.trigger) return fit;
  CostEval init = cost_evaluation(raw, target_norm);
  Tensor bestA = oA, bestB = oB;
  double best = init.cost, residual = 0;
  bool have_best = false;
  Tensor bQA, bC, bQB;
  int iterations = 0;
  bool limit = false;
  int stop = o.max_iterations == 0 ? 3 : 1;
  int fallbacks = 0;
  if (init.fallback) {
    stop = 2;
    fallbacks++;
  } else if (o.max_iterations > 0 && best <= o.error_tolerance) {
    stop = 0;
  } else if (o.max_iterations > 0) {
    Tensor wt = apply_pair_metric(E, p.wm, p.wt);
    for (int it = 1; it <= o.max_iterations; ++it) {
      Tensor MA, ya;
      left_normal_equation(E, p.wm, B, wt, MA, ya);
      Tensor sol = solve_core(E, MA, ya, perm_view(A, {0, 2, 1}), o, 20);
      QRres qa = qr(E, sol, {0, 2}, {1});
      Tensor right_initial = ein(E, "nb,bqs->nqs", qa.R, B);
      A = qa.Q;
      Tensor MB, yb;
      right_normal_equation(E, p.wm, A, wt, MB, yb);
      Tensor sol2 = solve_core(E, MB, yb, perm_view(right_initial, {0, 2, 1}), o, 21);
      LQres lb = lq(E, sol2, {0}, {2, 1});
      A = ein(E, "fpn,nm->fpm", qa.Q, lb.L);
      B = lb.Q;
      original_cores(E, p, A, B, oA, oB);
      raw = residual_cost(E, N, oA, oB, p.target);   // syncs; CG residuals are in slots 20, 21
      fit.trigger = repair_trigger(raw, target_norm);
      if (fit.trigger) return fit;
      CostEval ev = cost_evaluation(raw, target_norm);
      SPS_CUDA(cudaMemcpyAsync(E.hscal + 20, E.dscal + 20, 2 * sizeof(double), cudaMemcpyDeviceToHost, E.stream));
      E.sync();
      residual = std::max(E.hscal[20], E.hscal[21]);
      iterations = it;
      if (ev.fallback) {
        stop = 2;
        fallbacks++;
        break;
      }
      if (ev.cost <= best) {
        best = ev.cost;
        bestA = oA;
        bestB = oB;
        bQA = qa.Q;
        bC = lb.L;
        bQB = lb.Q;
        have_best = true;
      }
      if (best <= o.error_tolerance) {
        stop = 0;
        break;
      }
      limit = it == o.max_iterations;
    }
  }
  if (have_best) {
    Tensor A2, B2;
    fu_balance_bond(E, bQA, bC, bQB, A2, B2);
    original_cores(E, p, A2, B2, bestA, bestB);
  }
  fit.left = bestA;
  fit.right = bestB;
  fit.rep.initial_cost = init.cost;
  fit.rep.final_cost = best;
  fit.rep.residual = residual;
  fit.rep.iterations = iterations;
  fit.rep.iteration_limit_reached = limit;
  fit.rep.stop_reason = stop;
  fit.rep.fallbacks = fallbacks;
  return fit;
}

// update_bond! (full_update.jl:484-508)
BondReport update_bond_env(Engine& E, State& s, int ix, int iy, int jx, int jy, const Tensor& gate, int D,
                           const FUOptions& o, const PairEnv& env, const int space[2], bool force_repair) {
  Pair p = reduced_pair(E, s.at(ix, iy), s.at(jx, jy), gate, env.horizontal);
  Tensor N = env.metric(p.Qa, p.Qb);
  initialize_pair(E, p, N, D, space);
  Fit fit = optimize_pair(E, p, N, o);
  int repairs = 0;
  if (fit.trigger || force_repair) {
    Tensor Nr = positive_reduced_metric(E, env.hole(), p.Qa, p.Qb);
    repairs = 1;
    initialize_pair(E, p, Nr, D, space);
    fit = optimize_pair(E, p, Nr, o);
    if (fit.trigger) throw Error(SPS_ERR_REPAIR, "PSD repair did not remove the FU residual failure");
  }
  Tensor sa, sb;
  restore_pair(E, p, fit.left, fit.right, sa, sb);
  s.at(ix, iy) = sa;
  s.at(jx, jy) = sb;
  fit.rep.repairs = repairs;
  return fit.rep;
}

// update_bond! with a row bond environment
static BondReport update_bond(Engine& E, State& s, int ix, int iy, int jx, int jy, const Tensor& gate, int D,
                              const FUOptions& o, const BondEnv& hole, const int space[2], bool force_repair) {
  PairEnv env;
  env.horizontal = hole.horizontal;
  env.metric = [&](const Tensor& Qa, const Tensor& Qb) { return reduced_metric(E, hole, Qa, Qb); };
  env.hole = [&]() { return bond_hole(E, hole); };
  return update_bond_env(E, s, ix, iy, jx, jy, gate, D, o, env, space, force_repair);
}

void record_bond(StepReport& rep, const BondReport& br, const FUOptions& o) {
  rep.bond_updates++;
  if (br.iteration_limit_reached) {
    rep.iteration_limit_hits++;
    rep.max_iteration_limit_error = std::max(rep.max_iteration_limit_error, br.final_cost);
  }
  rep.stop_reasons[br.stop_reason]++;
  rep.max_state_truncation = std::max(rep.max_state_truncation, br.final_cost);
  rep.max_solver_residual = std::max(rep.max_solver_residual, br.residual);
  if (br.residual > o.linear_tolerance) rep.linear_unconverged++;
  rep.repairs += br.repairs;
  rep.fallbacks += br.fallbacks;
}

// _sweep! for the row method (full_update.jl:510-557)
static void sweep(Engine& E, State& s, const Model& m, double delta, int D, const FUOptions& o,
                  const BMPS& method, bool horizontal, bool reverse, const int space[2], Entropy* ent,
                  StepReport& rep, double& env_err, bool force_repair) {
  const int Lx = s.Lx, Ly = s.Ly;
  auto layers = row_layers(E, s);
  Envs env = boundary_environments(E, layers, Lx, Ly, method, reverse ? 1 : 2, ent);
  env_err = std::max(env_err, env.max_trunc);
  int ymax = horizontal ? Ly : Ly - 1;
  int xmax = horizontal ? Lx - 1 : Lx;
  for (int yi = 0; yi < ymax; ++yi) {
    int y = reverse ? ymax - 1 - yi : yi;
    const auto top = env.north[y].t;
    int lastrow = y + (horizontal ? 0 : 1);
    const auto bottom = env.south[lastrow + 1].t;
    std::vector<Layer> row(Lx);
    for (int x = 0; x < Lx; ++x) {
      row[x].a = layers[x + y * Lx];
      if (!horizontal) {
        row[x].b = layers[x + (y + 1) * Lx];
        row[x].slab = true;
      }
    }
    RowEnvs edges = row_environments(E, top, row, bottom, reverse ? 1 : 2);
    Tensor rolling = reverse ? edges.right[Lx] : edges.left[0];
    for (int xi = 0; xi < xmax; ++xi) {
      int x = reverse ? xmax - 1 - xi : xi;
      int jx = horizontal ? x + 1 : x, jy = horizontal ? y : y + 1;
      int finalx = horizontal ? x + 1 : x;
      BondEnv H;
      H.horizontal = horizontal;
      H.left = reverse ? edges.left[x] : rolling;
      H.right = reverse ? rolling : edges.right[finalx + 1];
      if (horizontal) {
        H.top = {top[x], top[x + 1]};
        H.bottom = {bottom[x], bottom[x + 1]};
        H.outer = {s.at(x, y).legs[0], s.at(x, y).legs[1], s.at(x, y).legs[5],
                   s.at(jx, jy).legs[1], s.at(jx, jy).legs[4], s.at(jx, jy).legs[5]};
      } else {
        H.top = {top[x]};
        H.bottom = {bottom[x]};
        H.outer = {s.at(x, y).legs[0], s.at(x, y).legs[1], s.at(x, y).legs[4],
                   s.at(jx, jy).legs[0], s.at(jx, jy).legs[4], s.at(jx, jy).legs[5]};
      }
      Tensor gate = trotter_gate(E, m, Lx, Ly, x, y, jx, jy, delta);
      double err = std::max(env.north[y].max_trunc, env.south[lastrow + 1].max_trunc);
      BondReport br = update_bond(E, s, x, y, jx, jy, gate, D, o, H, space, force_repair);
      br.max_env_trunc = err;
      record_bond(rep, br, o);
      layers[x + y * Lx] = double_layer(E, s.at(x, y), s.at(x, y));
      layers[jx + jy * Lx] = double_layer(E, s.at(jx, jy), s.at(jx, jy));
      int col = reverse ? finalx : x;
      if (x != (reverse ? 0 : xmax - 1)) {
        Layer Ec;
        Ec.a = layers[col + y * Lx];
        if (!horizontal) {
          Ec.b = layers[col + (y + 1) * Lx];
          Ec.slab = true;
        }
        rolling = reverse ? right_step(E, top[col], Ec, bottom[col], rolling)
                          : left_step(E, rolling, top[col], Ec, bottom[col]);
        safe_scale_inplace(E, rolling);
      }
    }
    std::vector<Tensor> rowt;
    if (reverse) {
      for (int x = 0; x < Lx; ++x) rowt.push_back(layers[x + lastrow * Lx]);
      env.south[lastrow] = absorb(E, env.south[lastrow + 1], rowt, method, false, ent, lastrow);
      env_err = std::max(env_err, env.south[lastrow].max_trunc);
    } else {
      for (int x = 0; x < Lx; ++x) rowt.push_back(layers[x + y * Lx]);
      env.north[y + 1] = absorb(E, env.north[y], rowt, method, true, ent, y + 1);
      env_err = std::max(env_err, env.north[y + 1].max_trunc);
    }
  }
}

// evolution_step! (full_update.jl:559-597)
StepReport evolution_step(Engine& E, State& s, const Model& m, double delta, int D, const FUOptions& o,
                          const BMPS& env_method, int order, const int space[2], bool record_entropy,
                          bool force_repair) {
  StepReport rep;
  double env_err = 0;
  Entropy ent;
  double gd = order == 2 ? delta / 2 : delta;
  if (s.Lx * s.Ly == 1) {
    // exp(-delta * (-h X)) on the physical leg
    const double h0 = m.field(0, 0, 1);
    double g[4] = {std::exp(delta * h0), 0, 0, std::exp(-delta * h0)};
    Par p2 = make_par(1, 1);
    Tensor G = E.upload({p2, p2}, g);
    s.sites[0] = ein(E, "pu,wnuaes->wnpaes", G, s.sites[0]);
  } else {
    struct SW { bool h, r; };
    std::vector<SW> sweeps = order == 2 ? std::vector<SW>{{true, false}, {false, false}, {false, true}, {true, true}}
                                        : std::vector<SW>{{true, false}, {false, false}};
    for (auto sw : sweeps) {
      if (sw.h && s.Lx < 2) continue;
      if (!sw.h && s.Ly < 2) continue;
      if (env_method.diagonal)
        sweep_diagonal(E, s, m, gd, D, o, env_method, sw.h, sw.r, space, record_entropy ? &ent : nullptr, rep,
                       env_err, force_repair || E.force_repair);
      else
        sweep(E, s, m, gd, D, o, env_method, sw.h, sw.r, space, record_entropy ? &ent : nullptr, rep, env_err,
              force_repair || E.force_repair);
    }
  }
  s.beta += 2 * delta;
  rep.log_normalizations = normalize_state(E, s);
  rep.beta = s.beta;
  rep.max_environment_truncation = env_err;
  rep.max_boundary_entropy = record_entropy ? ent.maximum : NAN;
  E.check_flag("evolution_step");
  return rep;
}

}  // namespace sps
