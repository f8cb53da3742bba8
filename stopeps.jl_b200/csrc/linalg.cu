// Dense FP64 factorizations of the Z2 parity blocks: Householder QR, one-sided
// (Hestenes) Jacobi SVD, two-sided cyclic Jacobi eigendecomposition and
// Gauss-Jordan inversion.  One CTA per block matrix; every loop is bounded and
// reports non-convergence through the engine's device flag instead of
// spinning.
//
// These replace LAPACK geqrf/orgqr (MatrixAlgebraKit left_orth/right_orth),
// gesdd (svd_compact/svd_trunc, src/states/svd.jl:2-33), syevd (eigh_full,
// src/evolution/full_update.jl:78) and getri (inv, full_update.jl:100).  The
// factors agree with LAPACK's up to the gauge freedom (column signs, the
// basis inside degenerate subspaces), which no reported scalar depends on.
#include "engine.h"
#include <cfloat>

namespace sps {
namespace la {

static constexpr int NT = 256;
static constexpr int NW = NT / 32;
static constexpr int FLAG_CONVERGENCE = 2;

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ double block_sum(double v, double* red) {
  v = warp_sum(v);
  int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) red[w] = v;
  __syncthreads();
  double t = 0;
  if (threadIdx.x < 32) {
    t = (l < NW) ? red[l] : 0.0;
    t = warp_sum(t);
    if (l == 0) red[NW] = t;
  }
  __syncthreads();
  return red[NW];
}

// ---------------------------------------------------------------------------
// Householder QR: a (m x n, col-major lda) -> q (m x k, ldq), r (k x n, ldr)
// tau stored in s[0..k).  LAPACK dlarfg/dorg2r conventions.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(NT) qr_kernel(const MatDesc* ds) {
  const MatDesc d = ds[blockIdx.x];
  const int m = d.m, n = d.n, lda = d.lda;
  const int k = min(m, n);
  if (k == 0) return;
  double* a = d.a;
  __shared__ double red[NW + 1];
  __shared__ double sh_tau;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int j = 0; j < k; ++j) {
    double* aj = a + (size_t)j * lda;
    double part = 0;
    for (int i = j + 1 + threadIdx.x; i < m; i += NT) part += aj[i] * aj[i];
    double sumsq = block_sum(part, red);
    if (threadIdx.x == 0) {
      double alpha = aj[j];
      double tau = 0.0;
      if (sumsq != 0.0) {
        double beta = -copysign(sqrt(alpha * alpha + sumsq), alpha);
        tau = (beta - alpha) / beta;
        aj[j] = beta;
        sh_tau = 1.0 / (alpha - beta);  // temporary: scale for v
      } else {
        sh_tau = 0.0;
      }
      d.s[j] = tau;
    }
    __syncthreads();
    double scal = sh_tau;
    if (scal != 0.0)
      for (int i = j + 1 + threadIdx.x; i < m; i += NT) aj[i] *= scal;
    __syncthreads();
    double tau = d.s[j];
    if (tau != 0.0) {
      for (int c = j + 1 + warp; c < n; c += NW) {
        double* ac = a + (size_t)c * lda;
        double w = 0;
        for (int i = j + 1 + lane; i < m; i += 32) w += aj[i] * ac[i];
        w = warp_sum(w);
        w = (w + ac[j]) * tau;
        if (lane == 0) ac[j] -= w;
        for (int i = j + 1 + lane; i < m; i += 32) ac[i] -= aj[i] * w;
      }
    }
    __syncthreads();
  }
  // R (k x n)
  for (int idx = threadIdx.x; idx < k * n; idx += NT) {
    int row = idx % k, col = idx / k;
    d.r[row + (size_t)col * d.ldr] = row <= col ? a[row + (size_t)col * lda] : 0.0;
  }
  // Q (m x k) = H_0 ... H_{k-1} [I; 0]
  for (int idx = threadIdx.x; idx < m * k; idx += NT) {
    int row = idx % m, col = idx / m;
    d.q[row + (size_t)col * d.ldq] = row == col ? 1.0 : 0.0;
  }
  __syncthreads();
  for (int j = k - 1; j >= 0; --j) {
    double tau = d.s[j];
    if (tau == 0.0) continue;
    const double* aj = a + (size_t)j * lda;
    for (int c = j + warp; c < k; c += NW) {
      double* qc = d.q + (size_t)c * d.ldq;
      double w = 0;
      for (int i = j + 1 + lane; i < m; i += 32) w += aj[i] * qc[i];
      w = warp_sum(w);
      w = (w + qc[j]) * tau;
      if (lane == 0) qc[j] -= w;
      for (int i = j + 1 + lane; i < m; i += 32) qc[i] -= aj[i] * w;
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// One-sided Jacobi SVD (m >= n): a (m x n, lda) is rotated in place until its
// columns are orthogonal; V accumulates in `work` (n x n).  Outputs sorted by
// descending singular value: q = U (m x n, ldq), r = V (n x n, ldr), s.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int rr_index(int i, int round, int np) {
  return i == 0 ? 0 : ((i - 1 + round) % (np - 1)) + 1;
}

__global__ void __launch_bounds__(NT) svd_kernel(const MatDesc* ds, double* work_base,
                                                 const size_t* work_off, int* flag, int max_sweeps) {
  const MatDesc d = ds[blockIdx.x];
  const int m = d.m, n = d.n, lda = d.lda;
  if (n == 0) return;
  double* U = d.a;
  double* V = work_base + work_off[blockIdx.x];   // n x n, ld n
  double* sig = V + (size_t)n * n;                // n scratch
  int* rank = (int*)(sig + n);                    // n ints
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int idx = threadIdx.x; idx < n * n; idx += NT) V[idx] = (idx % n == idx / n) ? 1.0 : 0.0;
  __shared__ int rotations;
  __syncthreads();
  const double tol = DBL_EPSILON * (double)max(m, 2);
  const int np = n + (n & 1);
  const int MAXSWEEP = max_sweeps;
  bool converged = (n == 1);
  for (int sweep = 0; sweep < MAXSWEEP && !converged; ++sweep) {
    if (threadIdx.x == 0) rotations = 0;
    __syncthreads();
    for (int round = 0; round < np - 1; ++round) {
      for (int pr = warp; pr < np / 2; pr += NW) {
        int p = rr_index(pr, round, np), q = rr_index(np - 1 - pr, round, np);
        if (p >= n || q >= n) continue;
        if (p > q) { int t = p; p = q; q = t; }
        double* up = U + (size_t)p * lda;
        double* uq = U + (size_t)q * lda;
        double al = 0, be = 0, ga = 0;
        for (int i = lane; i < m; i += 32) {
          double x = up[i], y = uq[i];
          al += x * x; be += y * y; ga += x * y;
        }
        al = warp_sum(al); be = warp_sum(be); ga = warp_sum(ga);
        // a column whose squared norm underflows counts as zero: rotating it
        // against a normal one is a no-op that would repeat every sweep
        if (!(al >= DBL_MIN && be >= DBL_MIN) || ga == 0.0 || !(fabs(ga) > tol * sqrt(al) * sqrt(be))) continue;
        double zeta = (be - al) / (2.0 * ga);
        double t = copysign(1.0, zeta) / (fabs(zeta) + hypot(1.0, zeta));
        double c = 1.0 / sqrt(1.0 + t * t), s = c * t;
        for (int i = lane; i < m; i += 32) {
          double x = up[i], y = uq[i];
          up[i] = c * x - s * y;
          uq[i] = s * x + c * y;
        }
        double* vp = V + (size_t)p * n;
        double* vq = V + (size_t)q * n;
        for (int i = lane; i < n; i += 32) {
          double x = vp[i], y = vq[i];
          vp[i] = c * x - s * y;
          vq[i] = s * x + c * y;
        }
        if (lane == 0) atomicAdd(&rotations, 1);
      }
      __syncthreads();
    }
    converged = (rotations == 0);
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    if (!converged) atomicOr(flag, FLAG_CONVERGENCE);
  }
  // singular values and descending order (stable by index)
  for (int c = warp; c < n; c += NW) {
    const double* uc = U + (size_t)c * lda;
    double v = 0;
    for (int i = lane; i < m; i += 32) v += uc[i] * uc[i];
    v = warp_sum(v);
    if (lane == 0) sig[c] = sqrt(v);
  }
  __syncthreads();
  for (int c = threadIdx.x; c < n; c += NT) {
    double sc = sig[c];
    int r = 0;
    for (int j = 0; j < n; ++j) {
      double sj = sig[j];
      r += (sj > sc) || (sj == sc && j < c);
    }
    rank[c] = r;
    d.s[r] = sc;
  }
  __syncthreads();
  for (int c = warp; c < n; c += NW) {
    int r = rank[c];
    double sc = sig[c];
    double inv = sc > 0 ? 1.0 / sc : 0.0;
    const double* uc = U + (size_t)c * lda;
    double* qo = d.q + (size_t)r * d.ldq;
    for (int i = lane; i < m; i += 32) qo[i] = uc[i] * inv;
    const double* vc = V + (size_t)c * n;
    double* ro = d.r + (size_t)r * d.ldr;
    for (int i = lane; i < n; i += 32) ro[i] = vc[i];
  }
}

// ---------------------------------------------------------------------------
// Two-sided parallel cyclic Jacobi for symmetric a (n x n, lda).  Eigenvalues
// ascending in s, eigenvectors in q (n x n, ldq).  `work` holds V and flags.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(NT) eigh_kernel(const MatDesc* ds, double* work_base,
                                                  const size_t* work_off, int* flag, int max_sweeps) {
  const MatDesc d = ds[blockIdx.x];
  const int n = d.n, lda = d.lda;
  if (n == 0) return;
  double* A = d.a;
  double* V = work_base + work_off[blockIdx.x];  // n x n
  const int np2 = n / 2 + 2;
  double* cs = V + (size_t)n * n;                 // cosines of the current round
  double* sn = cs + np2;                          // sines
  int* pp = (int*)(sn + np2);                     // pair p (np2 ints inside np2 doubles)
  int* qq = (int*)(sn + 2 * np2);                 // pair q
  double* ev = sn + 3 * np2;                      // n eigenvalues
  int* rank = (int*)(ev + n);
  __shared__ double red[NW + 1];
  __shared__ int rotations;
  for (int idx = threadIdx.x; idx < n * n; idx += NT) V[idx] = (idx % n == idx / n) ? 1.0 : 0.0;
  double part = 0;
  for (int idx = threadIdx.x; idx < n * n; idx += NT) {
    double x = A[(idx % n) + (size_t)(idx / n) * lda];
    part += x * x;
  }
  const double fro = sqrt(block_sum(part, red));
  // off-diagonals below eps ||A||_F are rounding noise (the backward error of
  // any symmetric eigensolver); rotating them would not end for nearly
  // rank-deficient matrices, whose diagonal is itself at noise level
  const double abs_floor = DBL_EPSILON * fro;
  const int np = n + (n & 1);
  const int npair = np / 2;
  bool converged = (n == 1) || fro == 0.0;
  const int MAXSWEEP = max_sweeps;
  for (int sweep = 0; sweep < MAXSWEEP && !converged; ++sweep) {
    if (threadIdx.x == 0) rotations = 0;
    __syncthreads();
    for (int round = 0; round < np - 1; ++round) {
      for (int pr = threadIdx.x; pr < npair; pr += NT) {
        int p = rr_index(pr, round, np), q = rr_index(np - 1 - pr, round, np);
        if (p > q) { int t = p; p = q; q = t; }
        pp[pr] = p; qq[pr] = q;
        double c = 1.0, s = 0.0;
        if (q < n) {
          double apq = A[p + (size_t)q * lda];
          double app = A[p + (size_t)p * lda], aqq = A[q + (size_t)q * lda];
          if (apq != 0.0 && fabs(apq) > DBL_EPSILON * sqrt(fabs(app * aqq)) && fabs(apq) > abs_floor) {
            double zeta = (aqq - app) / (2.0 * apq);
            double t = copysign(1.0, zeta) / (fabs(zeta) + hypot(1.0, zeta));
            c = 1.0 / sqrt(1.0 + t * t);
            s = c * t;
            atomicAdd(&rotations, 1);
          }
        }
        cs[pr] = c; sn[pr] = s;
      }
      __syncthreads();
      // A <- A J (columns), V <- V J
      for (int idx = threadIdx.x; idx < npair * n; idx += NT) {
        int pr = idx / n, i = idx % n;
        double s = sn[pr];
        if (s == 0.0) continue;
        double c = cs[pr];
        int p = pp[pr], q = qq[pr];
        double x = A[i + (size_t)p * lda], y = A[i + (size_t)q * lda];
        A[i + (size_t)p * lda] = c * x - s * y;
        A[i + (size_t)q * lda] = s * x + c * y;
        x = V[i + (size_t)p * n]; y = V[i + (size_t)q * n];
        V[i + (size_t)p * n] = c * x - s * y;
        V[i + (size_t)q * n] = s * x + c * y;
      }
      __syncthreads();
      // A <- J^T A (rows)
      for (int idx = threadIdx.x; idx < npair * n; idx += NT) {
        int pr = idx / n, j = idx % n;
        double s = sn[pr];
        if (s == 0.0) continue;
        double c = cs[pr];
        int p = pp[pr], q = qq[pr];
        double x = A[p + (size_t)j * lda], y = A[q + (size_t)j * lda];
        A[p + (size_t)j * lda] = c * x - s * y;
        A[q + (size_t)j * lda] = s * x + c * y;
      }
      __syncthreads();
    }
    converged = (rotations == 0);
    __syncthreads();
  }
  if (!converged && threadIdx.x == 0) atomicOr(flag, FLAG_CONVERGENCE);
  for (int c = threadIdx.x; c < n; c += NT) ev[c] = A[c + (size_t)c * lda];
  __syncthreads();
  for (int c = threadIdx.x; c < n; c += NT) {
    double e = ev[c];
    int r = 0;
    for (int j = 0; j < n; ++j) r += (ev[j] < e) || (ev[j] == e && j < c);
    rank[c] = r;
    d.s[r] = e;
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < n * n; idx += NT) {
    int i = idx % n, c = idx / n;
    d.q[i + (size_t)rank[c] * d.ldq] = V[i + (size_t)c * n];
  }
}

// ---------------------------------------------------------------------------
// Gauss-Jordan inverse with partial pivoting: a (n x n, lda) -> q (n x n, ldq)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(NT) inv_kernel(const MatDesc* ds, int* flag) {
  const MatDesc d = ds[blockIdx.x];
  const int n = d.n, lda = d.lda;
  if (n == 0) return;
  double* A = d.a;
  double* X = d.q;
  const int ldx = d.ldq;
  __shared__ int piv;
  __shared__ double pval[NT];
  __shared__ int pidx[NT];
  for (int idx = threadIdx.x; idx < n * n; idx += NT) {
    int i = idx % n, j = idx / n;
    X[i + (size_t)j * ldx] = (i == j) ? 1.0 : 0.0;
  }
  __syncthreads();
  for (int col = 0; col < n; ++col) {
    double best = -1.0;
    int bi = col;
    for (int i = col + threadIdx.x; i < n; i += NT) {
      double v = fabs(A[i + (size_t)col * lda]);
      if (v > best) { best = v; bi = i; }
    }
    pval[threadIdx.x] = best;
    pidx[threadIdx.x] = bi;
    __syncthreads();
    if (threadIdx.x == 0) {
      double b = -1.0;
      int bb = col;
      for (int t = 0; t < NT; ++t)
        if (pval[t] > b) { b = pval[t]; bb = pidx[t]; }
      piv = bb;
      if (!(b > 0.0)) atomicOr(flag, 1);
    }
    __syncthreads();
    int pr = piv;
    if (pr != col) {
      for (int j = threadIdx.x; j < n; j += NT) {
        double t = A[col + (size_t)j * lda];
        A[col + (size_t)j * lda] = A[pr + (size_t)j * lda];
        A[pr + (size_t)j * lda] = t;
        t = X[col + (size_t)j * ldx];
        X[col + (size_t)j * ldx] = X[pr + (size_t)j * ldx];
        X[pr + (size_t)j * ldx] = t;
      }
    }
    __syncthreads();
    double inv = 1.0 / A[col + (size_t)col * lda];
    __syncthreads();
    for (int j = threadIdx.x; j < n; j += NT) {
      A[col + (size_t)j * lda] *= inv;
      X[col + (size_t)j * ldx] *= inv;
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < n * n; idx += NT) {
      int i = idx % n, j = idx / n;
      if (i == col) continue;
      double f = A[i + (size_t)col * lda];
      if (f == 0.0) continue;
      // column `col` of A is read by every thread in this pass: defer its update
      if (j != col) A[i + (size_t)j * lda] -= f * A[col + (size_t)j * lda];
      X[i + (size_t)j * ldx] -= f * X[col + (size_t)j * ldx];
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += NT)
      if (i != col) A[i + (size_t)col * lda] = 0.0;
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------
static MatDesc* upload_desc(Engine& E, const std::vector<MatDesc>& d, Buf& keep) {
  keep = E.alloc(sizeof(MatDesc) * d.size());
  E.stage(d.data(), sizeof(MatDesc) * d.size(), keep->ptr);
  return (MatDesc*)keep->ptr;
}

void qr_batched(Engine& E, const std::vector<MatDesc>& d) {
  if (d.empty()) return;
  Buf kd;
  MatDesc* dd = upload_desc(E, d, kd);
  double fl = 0;
  for (auto& x : d) {
    double k = std::min(x.m, x.n);
    fl += 4.0 * x.m * x.n * k;
  }
  int tk = E.tic("qr_small");
  qr_kernel<<<(int)d.size(), NT, 0, E.stream>>>(dd);
  E.toc(tk, fl);
  SPS_CUDA(cudaGetLastError());
  E.launches++;
  E.flops += fl;
}

void svd_batched(Engine& E, const std::vector<MatDesc>& d) {
  if (d.empty()) return;
  Buf kd;
  MatDesc* dd = upload_desc(E, d, kd);
  std::vector<size_t> off(d.size());
  size_t tot = 0;
  for (size_t i = 0; i < d.size(); ++i) {
    off[i] = tot;
    size_t n = d[i].n;
    tot += n * n + n + (n + 1) / 2 + 8;
  }
  Buf w = E.alloc(std::max<size_t>(tot, 1) * sizeof(double));
  Buf ko = E.alloc(off.size() * sizeof(size_t));
  E.stage(off.data(), off.size() * sizeof(size_t), ko->ptr);
  int tk = E.tic("svd_small");
  svd_kernel<<<(int)d.size(), NT, 0, E.stream>>>(dd, (double*)w->ptr, (const size_t*)ko->ptr,
                                                E.dflag, E.sweep_cap > 0 ? E.sweep_cap : 80);
  E.toc(tk);
  SPS_CUDA(cudaGetLastError());
  E.launches++;
}

void eigh_batched(Engine& E, const std::vector<MatDesc>& d) {
  if (d.empty()) return;
  Buf kd;
  MatDesc* dd = upload_desc(E, d, kd);
  std::vector<size_t> off(d.size());
  size_t tot = 0;
  for (size_t i = 0; i < d.size(); ++i) {
    off[i] = tot;
    size_t n = d[i].n;
    tot += n * n + 4 * (n / 2 + 2) + 2 * n + 16;
  }
  Buf w = E.alloc(std::max<size_t>(tot, 1) * sizeof(double));
  Buf ko = E.alloc(off.size() * sizeof(size_t));
  E.stage(off.data(), off.size() * sizeof(size_t), ko->ptr);
  int tk = E.tic("eigh");
  eigh_kernel<<<(int)d.size(), NT, 0, E.stream>>>(dd, (double*)w->ptr, (const size_t*)ko->ptr,
                                                 E.dflag, E.sweep_cap > 0 ? E.sweep_cap : 80);
  E.toc(tk);
  SPS_CUDA(cudaGetLastError());
  E.launches++;
}

void inv_batched(Engine& E, const std::vector<MatDesc>& d) {
  if (d.empty()) return;
  Buf kd;
  MatDesc* dd = upload_desc(E, d, kd);
  inv_kernel<<<(int)d.size(), NT, 0, E.stream>>>(dd, E.dflag);
  SPS_CUDA(cudaGetLastError());
  E.launches++;
}

}  // namespace la
}  // namespace sps
