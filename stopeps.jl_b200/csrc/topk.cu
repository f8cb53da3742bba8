// Leading singular triplets of large parity blocks by block subspace
// iteration, for truncated SVDs that keep few vectors of a big block (the
// boundary-MPS compression keeps chi columns of (chi d) x (chi d) blocks,
// src/contraction/boundary_mps.jl:33-42 with truncrank & truncspace).
//
// One cooperative launch handles every parity block of a call; each block
// ("problem") owns a group of CTAs and its own software barrier, and every CTA
// owns a contiguous range of rows of the m- and n-sized iterates:
//
//   Q = orth(M Omega);  repeat  Z = orth(M^T Q),  Q = orth(M Z)
//
// (orthogonal iteration, block size b > k).  orth is a Cholesky QR: per-CTA
// Gram partials, reduced in a fixed order (deterministic), factored
// redundantly by every CTA, applied to the CTA's own rows; the iteration
// passes add the shift of shifted Cholesky QR (Fukaya, Kannan, Nakatsukasa,
// Yamamoto, Yanagisawa, SIAM J. Sci. Comput. 42 (2020)) so that they cannot
// break down.  Rayleigh-Ritz extraction: Q <- orth(Q) (plain pass),
// M^T Q = Qb Rb (shifted Cholesky QR3), Rb^T = Ub S J^T by one-sided Jacobi in
// one CTA, U = Q Ub, V = Qb J.  The extraction is accepted when
// ||M v_i - s_i u_i|| is at rounding level for every wanted i; otherwise two
// more iterations and a new extraction, up to a cap, after which the caller
// uses the full SVD.  Everything is FP64.
#include "engine.h"
#include "coop.cuh"
#include <cfloat>
#include <algorithm>

namespace sps {
namespace la {

namespace {

constexpr int TT = 256;           // threads per CTA
constexpr int TW = TT / 32;       // warps per CTA
constexpr int KMAXB = 80;         // largest block size b
constexpr int RMAX = 32;          // largest number of rows owned by one CTA
constexpr int KC = 32;            // contraction chunk of the row GEMM
constexpr int XLD = KC + 1;
constexpr int SLD = KMAXB + 4;
constexpr int YLD = KMAXB + 1;
constexpr int GLD = KMAXB + 1;
constexpr int OFF_X = 0;
constexpr int OFF_S = OFF_X + RMAX * XLD;
constexpr int OFF_Y = OFF_S + KC * SLD;
constexpr int OFF_G = OFF_Y + RMAX * YLD;
constexpr int OFF_V = OFF_G + KMAXB * GLD;
constexpr int OFF_R = OFF_V + 3 * KMAXB;
constexpr int SMEM_DOUBLES = OFF_R + 16 + KMAXB;
constexpr int JLD = KMAXB + 1;    // Jacobi arrays (CTA 0 only, overlays X..V)
constexpr int MAX_SWEEPS = 40;
static_assert(2 * KMAXB * JLD <= OFF_R, "Jacobi overlay exceeds the shared arena");
static_assert((RMAX / 2) * ((KMAXB + 3) / 4) * 8 <= OFF_Y, "GEMM reduction scratch exceeds X+S");

enum : int { ST_OK = 0, ST_BREAKDOWN = 1, ST_JACOBI = 2, ST_NOCONV = 3, ST_ZERO = 4 };

}  // namespace

struct TopkProb {
  const double* M;   // m x n, column-major, ld m (read-only in the kernel)
  const double* Mt;  // n x m, column-major, ld n (M transposed)
  int m, n, k, b, P, cta0;
  double* Q;     // m x b
  double* Z;     // n x b (Omega, Z iterates, Qb)
  double* Gp;    // P x KMAXB^2 Gram partials
  double* G;     // b x b
  double* Racc;  // b x b accumulated R of M^T Q (row-major)
  double* Ub;    // b x b left Ritz rotation (column-major)
  double* Jo;    // b x b right Ritz rotation (column-major)
  double* U;     // m x k out (ld m)
  double* V;     // n x k out (ld n)
  double* s;     // b Ritz values, descending
  double* fpart; // P partial squared Frobenius norms
  double* info;  // [status, iterations, ||M||_F^2, max residual / threshold, done]
  unsigned* bar; // 2 words
};

namespace {

struct Ctx {
  const TopkProb* p;
  int c;            // CTA index inside the problem
  int rm0, rm1;     // rows of m-sized iterates owned here
  int rn0, rn1;     // rows of n-sized iterates owned here
  double* sm;
  int* flag;
};

__device__ __forceinline__ void sync_group(const Ctx& x) { group_barrier(x.p->bar, (unsigned)x.p->P, x.flag); }

// Ys[r][j] = sum_t X[(r0+r)*ldx + t] * S[j*lds + t]   (r < r1-r0, j < bb, t < K)
// X is read-only for the whole launch; S is written by other CTAs (L2 loads).
__device__ void gemm_rows(const Ctx& x, const double* __restrict__ X, int ldx, int K, const double* S, int lds,
                          int bb, int r0, int r1) {
  double* Xs = x.sm + OFF_X;
  double* Ss = x.sm + OFF_S;
  double* Ys = x.sm + OFF_Y;
  const int R = r1 - r0;
  const int tr = (R + 1) / 2, tj = (bb + 3) / 4, ntile = tr * tj;
  int KG = 1;
  while (KG < 8 && KG * 2 * ntile <= TT) KG *= 2;
  const int TPG = TT / KG;
  const int g = threadIdx.x / TPG, lt = threadIdx.x % TPG;
  double acc[2][2][4];
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int r = 0; r < 2; ++r)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[a][r][q] = 0.0;
  int ri[2], ji[2];
#pragma unroll
  for (int a = 0; a < 2; ++a) {
    const int tl = lt + a * TPG;
    ri[a] = tl < ntile ? (tl / tj) * 2 : -1;
    ji[a] = tl < ntile ? (tl % tj) * 4 : 0;
  }
  for (int t0 = 0; t0 < K; t0 += KC) {
    const int kc = min(KC, K - t0);
    __syncthreads();
    for (int e = threadIdx.x; e < 2 * tr * KC; e += TT) {
      const int r = e / KC, t = e - r * KC;
      Xs[r * XLD + t] = (r < R && t < kc) ? X[(size_t)(r0 + r) * ldx + t0 + t] : 0.0;
    }
    for (int e = threadIdx.x; e < 4 * tj * KC; e += TT) {
      const int j = e / KC, t = e - j * KC;
      Ss[t * SLD + j] = (j < bb && t < kc) ? __ldcg(&S[(size_t)j * lds + t0 + t]) : 0.0;
    }
    __syncthreads();
    if (g < KG) {
      for (int t = g; t < KC; t += KG) {
#pragma unroll
        for (int a = 0; a < 2; ++a) {
          if (ri[a] < 0) continue;
          const double x0 = Xs[ri[a] * XLD + t], x1 = Xs[(ri[a] + 1) * XLD + t];
          const double* sr = Ss + t * SLD + ji[a];
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const double sv = sr[q];
            acc[a][0][q] = fma(x0, sv, acc[a][0][q]);
            acc[a][1][q] = fma(x1, sv, acc[a][1][q]);
          }
        }
      }
    }
  }
  __syncthreads();
  double* part = x.sm + OFF_X;   // KG x (2 tr) x (4 tj)
  const int pr = 2 * tr, pc = 4 * tj;
  if (g < KG) {
#pragma unroll
    for (int a = 0; a < 2; ++a) {
      if (ri[a] < 0) continue;
#pragma unroll
      for (int r = 0; r < 2; ++r)
#pragma unroll
        for (int q = 0; q < 4; ++q) part[(g * pr + ri[a] + r) * pc + ji[a] + q] = acc[a][r][q];
    }
  }
  __syncthreads();
  for (int e = threadIdx.x; e < R * bb; e += TT) {
    const int r = e / bb, j = e - r * bb;
    double v = 0.0;
    for (int q = 0; q < KG; ++q) v += part[(q * pr + r) * pc + j];
    Ys[r * YLD + j] = v;
  }
  __syncthreads();
}

// Load rows [r0, r1) of the column-major (ld) matrix A (bb columns) into Ys.
__device__ void load_rows(const Ctx& x, const double* A, int ld, int bb, int r0, int r1) {
  double* Ys = x.sm + OFF_Y;
  const int R = r1 - r0;
  __syncthreads();
  for (int e = threadIdx.x; e < R * bb; e += TT) {
    const int j = e / R, r = e - j * R;
    Ys[r * YLD + j] = __ldcg(&A[(size_t)j * ld + r0 + r]);
  }
  __syncthreads();
}

__device__ void store_rows(const Ctx& x, double* A, int ld, int bb, int r0, int r1) {
  const double* Ys = x.sm + OFF_Y;
  const int R = r1 - r0;
  for (int e = threadIdx.x; e < R * bb; e += TT) {
    const int j = e / R, r = e - j * R;
    A[(size_t)j * ld + r0 + r] = Ys[r * YLD + j];
  }
}

// Cholesky QR pass on the distributed rows held in Ys (rows [r0, r1) of an
// nrows x bb matrix).  racc: 0 none, 1 Racc = R, 2 Racc = R Racc (CTA 0).
// Returns false (uniformly over the group) on breakdown.
__device__ bool orth_pass(const Ctx& x, int bb, int r0, int r1, int nrows, bool shifted, int racc) {
  const TopkProb& p = *x.p;
  double* Ys = x.sm + OFF_Y;
  double* Gs = x.sm + OFF_G;
  double* sq = x.sm + OFF_V;              // sqrt of the pivots
  double* invd = sq + KMAXB;              // 1 / pivots
  const int R = r1 - r0;
  // partial Gram of the owned rows (upper triangle)
  double* gp = p.Gp + (size_t)x.c * KMAXB * KMAXB;
  for (int e = threadIdx.x; e < bb * bb; e += TT) {
    const int i = e / bb, j = e - i * bb;
    if (j < i) continue;
    double v = 0.0;
    for (int r = 0; r < R; ++r) v = fma(Ys[r * YLD + i], Ys[r * YLD + j], v);
    gp[e] = v;
  }
  sync_group(x);
  // reduce this CTA's slice of entries over the partials, in partial order
  {
    const int total = bb * bb;
    const int slice = (total + p.P - 1) / p.P;
    const int e0 = x.c * slice, e1 = min(total, e0 + slice);
    for (int e = e0 + threadIdx.x; e < e1; e += TT) {
      const int i = e / bb, j = e - i * bb;
      if (j < i) continue;
      double v = 0.0;
      for (int q = 0; q < p.P; ++q) v += __ldcg(&p.Gp[(size_t)q * KMAXB * KMAXB + e]);
      p.G[e] = v;
    }
  }
  sync_group(x);
  // factor G (+ shift) redundantly: G = U^T D U with U unit upper, kept as the
  // unscaled upper rows D U in Gs
  for (int e = threadIdx.x; e < bb * bb; e += TT) {
    const int i = e / bb, j = e - i * bb;
    if (j >= i) Gs[i * GLD + j] = __ldcg(&p.G[e]);
  }
  __syncthreads();
  if (shifted) {
    if (threadIdx.x == 0) {
      double tr = 0.0;
      for (int i = 0; i < bb; ++i) tr += Gs[i * GLD + i];
      const double sh = 11.0 * ((double)nrows * bb + (double)bb * (bb + 1)) * DBL_EPSILON * tr;
      for (int i = 0; i < bb; ++i) Gs[i * GLD + i] += sh;
    }
  }
  for (int j = 0; j < bb; ++j) {
    __syncthreads();
    const double d = Gs[j * GLD + j];
    if (!(d > 0.0) || !isfinite(d)) {
      if (x.c == 0 && threadIdx.x == 0) p.info[0] = ST_BREAKDOWN;
      return false;
    }
    const double inv = 1.0 / d;
    const int nt = bb - 1 - j;
    for (int e = threadIdx.x; e < nt * nt; e += TT) {
      const int i = j + 1 + e / nt, l = j + 1 + e % nt;
      if (l >= i) Gs[i * GLD + l] -= Gs[j * GLD + i] * Gs[j * GLD + l] * inv;
    }
  }
  __syncthreads();
  for (int j = threadIdx.x; j < bb; j += TT) {
    sq[j] = sqrt(Gs[j * GLD + j]);
    invd[j] = 1.0 / Gs[j * GLD + j];
  }
  __syncthreads();
  // unit upper U in place (diagonal kept as the pivot)
  for (int e = threadIdx.x; e < bb * bb; e += TT) {
    const int i = e / bb, j = e - i * bb;
    if (j > i) Gs[i * GLD + j] *= invd[i];
  }
  __syncthreads();
  if (racc && x.c == 0) {
    // R = diag(sq) U;  Racc <- R (racc 1) or R Racc (racc 2), via CTA 0's partial slot
    double* tmp = gp;
    for (int e = threadIdx.x; e < bb * bb; e += TT) {
      const int i = e / bb, j = e - i * bb;
      double v = 0.0;
      if (j >= i) {
        if (racc == 1) {
          v = (i == j) ? sq[i] : sq[i] * Gs[i * GLD + j];
        } else {
          for (int l = i; l <= j; ++l) {
            const double ril = (l == i) ? sq[i] : sq[i] * Gs[i * GLD + l];
            v = fma(ril, __ldcg(&p.Racc[l * bb + j]), v);
          }
        }
      }
      tmp[e] = v;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < bb * bb; e += TT) p.Racc[e] = tmp[e];
  }
  // rows: y <- y R^{-1}, R = diag(sq) U: forward substitution on the unit
  // upper factor, one column per step, then the diagonal scaling
  for (int j = 0; j < bb - 1; ++j) {
    const int nt = bb - 1 - j;
    for (int e = threadIdx.x; e < R * nt; e += TT) {
      const int r = e / nt, l = j + 1 + e % nt;
      Ys[r * YLD + l] -= Ys[r * YLD + j] * Gs[j * GLD + l];
    }
    __syncthreads();
  }
  for (int e = threadIdx.x; e < R * bb; e += TT) {
    const int r = e / bb, j = e - r * bb;
    Ys[r * YLD + j] /= sq[j];
  }
  __syncthreads();
  return true;
}

// One-sided Jacobi SVD of A = Racc^T (bb x bb) in CTA 0; sorted outputs to
// p.s, p.Ub (left vectors), p.Jo (right vectors).
__device__ void ritz_small(const Ctx& x, int bb) {
  const TopkProb& p = *x.p;
  double* A = x.sm;                 // column-major, JLD
  double* J = x.sm + KMAXB * JLD;   // column-major, JLD
  int* cnt = reinterpret_cast<int*>(x.sm + OFF_R);
  double* sig = x.sm + OFF_R + 16;  // not overlapping the Jacobi arrays (OFF_R >= 2 KMAXB JLD)
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int e = threadIdx.x; e < bb * bb; e += TT) {
    const int col = e / bb, row = e - col * bb;
    A[col * JLD + row] = __ldcg(&p.Racc[col * bb + row]);   // column col of Racc^T = row col of Racc
    J[col * JLD + row] = (row == col) ? 1.0 : 0.0;
  }
  __syncthreads();
  int sweep = 0;
  for (; sweep < MAX_SWEEPS; ++sweep) {
    if (threadIdx.x == 0) *cnt = 0;
    for (int round = 0; round < bb - 1; ++round) {
      __syncthreads();
      for (int pi = warp; pi < bb / 2; pi += TW) {
        int pp, qq;
        if (pi == 0) {
          pp = round;
          qq = bb - 1;
        } else {
          pp = (round + pi) % (bb - 1);
          qq = (round - pi + bb - 1) % (bb - 1);
        }
        double* ap = A + pp * JLD;
        double* aq = A + qq * JLD;
        double al = 0.0, be = 0.0, ga = 0.0;
        for (int r = lane; r < bb; r += 32) {
          const double u = ap[r], v = aq[r];
          al = fma(u, u, al);
          be = fma(v, v, be);
          ga = fma(u, v, ga);
        }
        al = wsum(al);
        be = wsum(be);
        ga = wsum(ga);
        if (ga != 0.0 && fabs(ga) > DBL_EPSILON * sqrt(al) * sqrt(be)) {
          const double zeta = (be - al) / (2.0 * ga);
          const double t = copysign(1.0, zeta) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
          const double cs = 1.0 / sqrt(1.0 + t * t), sn = cs * t;
          double* jp = J + pp * JLD;
          double* jq = J + qq * JLD;
          for (int r = lane; r < bb; r += 32) {
            const double u = ap[r], v = aq[r];
            ap[r] = cs * u - sn * v;
            aq[r] = sn * u + cs * v;
            const double ju = jp[r], jv = jq[r];
            jp[r] = cs * ju - sn * jv;
            jq[r] = sn * ju + cs * jv;
          }
          if (lane == 0) atomicAdd(cnt, 1);
        }
      }
    }
    __syncthreads();
    const int rotations = *cnt;
    __syncthreads();
    if (rotations == 0) break;
  }
  if (sweep == MAX_SWEEPS) {
    if (threadIdx.x == 0) p.info[0] = ST_JACOBI;
    return;
  }
  for (int col = warp; col < bb; col += TW) {
    double v = 0.0;
    for (int r = lane; r < bb; r += 32) v = fma(A[col * JLD + r], A[col * JLD + r], v);
    v = wsum(v);
    if (lane == 0) sig[col] = sqrt(v);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < bb; i += TT) {
    int rank = 0;
    for (int j = 0; j < bb; ++j) rank += (sig[j] > sig[i]) || (sig[j] == sig[i] && j < i);
    p.s[rank] = sig[i];
    const double inv = sig[i] > 0.0 ? 1.0 / sig[i] : 0.0;
    for (int r = 0; r < bb; ++r) {
      p.Ub[(size_t)rank * bb + r] = A[i * JLD + r] * inv;
      p.Jo[(size_t)rank * bb + r] = J[i * JLD + r];
    }
  }
}

// rows [r0, r1) of OUT (ld) = rows of A (ld_a, bb cols) times Rot[:, :k] (bb x bb col-major)
__device__ void rotate_rows(const Ctx& x, const double* A, int lda, const double* Rot, int bb, int k, double* out,
                            int ldo, int r0, int r1) {
  load_rows(x, A, lda, bb, r0, r1);
  double* Ys = x.sm + OFF_Y;
  double* Rs = x.sm + OFF_G;   // bb x k, column-major
  for (int e = threadIdx.x; e < bb * k; e += TT) Rs[e] = __ldcg(&Rot[e]);
  __syncthreads();
  const int R = r1 - r0;
  for (int e = threadIdx.x; e < R * k; e += TT) {
    const int i = e / R, r = e - i * R;
    double v = 0.0;
    for (int j = 0; j < bb; ++j) v = fma(Ys[r * YLD + j], Rs[i * bb + j], v);
    out[(size_t)i * ldo + r0 + r] = v;
  }
  __syncthreads();
}

__device__ __forceinline__ double omega(unsigned long long i) {
  unsigned long long z = i + 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  z ^= z >> 31;
  return (double)(z >> 11) * (2.0 / 9007199254740992.0) - 1.0;
}

}  // namespace

__global__ void __launch_bounds__(TT) topk_kernel(const TopkProb* __restrict__ probs, int nprob, int q0, int qstep,
                                                  int qmax, double tol, int* flag) {
  extern __shared__ double sm[];
  int pi = -1;
  for (int q = 0; q < nprob; ++q)
    if ((int)blockIdx.x >= probs[q].cta0 && (int)blockIdx.x < probs[q].cta0 + probs[q].P) pi = q;
  if (pi < 0) return;
  const TopkProb& p = probs[pi];
  Ctx x;
  x.p = &p;
  x.c = blockIdx.x - p.cta0;
  x.sm = sm;
  x.flag = flag;
  const int Rm = (p.m + p.P - 1) / p.P, Rn = (p.n + p.P - 1) / p.P;
  x.rm0 = min(p.m, x.c * Rm);
  x.rm1 = min(p.m, x.rm0 + Rm);
  x.rn0 = min(p.n, x.c * Rn);
  x.rn1 = min(p.n, x.rn0 + Rn);
  const int b = p.b, k = p.k;
  double* red = sm + OFF_R;

  // Omega into Z (owned n-rows) and the owned columns' share of ||M||_F^2
  {
    double f = 0.0;
    for (int e = threadIdx.x; e < (x.rn1 - x.rn0) * b; e += TT) {
      const int j = e / (x.rn1 - x.rn0), r = e - j * (x.rn1 - x.rn0);
      p.Z[(size_t)j * p.n + x.rn0 + r] = omega((unsigned long long)j * p.n + x.rn0 + r);
    }
    for (int col = x.rn0; col < x.rn1; ++col)
      for (int r = threadIdx.x; r < p.m; r += TT) {
        const double v = p.M[(size_t)col * p.m + r];
        f = fma(v, v, f);
      }
    f = wsum(f);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = f;
    __syncthreads();
    if (threadIdx.x == 0) {
      double s = 0.0;
      for (int w = 0; w < TW; ++w) s += red[w];
      p.fpart[x.c] = s;
    }
  }
  sync_group(x);
  if (x.c == 0 && threadIdx.x == 0) {
    double s = 0.0;
    for (int q = 0; q < p.P; ++q) s += __ldcg(&p.fpart[q]);
    p.info[2] = s;
  }
  gemm_rows(x, p.Mt, p.n, p.n, p.Z, p.n, b, x.rm0, x.rm1);
  if (!orth_pass(x, b, x.rm0, x.rm1, p.m, true, 0)) return;
  store_rows(x, p.Q, p.m, b, x.rm0, x.rm1);
  sync_group(x);

  int it = 0, target = q0;
  for (;;) {
    for (; it < target; ++it) {
      gemm_rows(x, p.M, p.m, p.m, p.Q, p.m, b, x.rn0, x.rn1);
      if (!orth_pass(x, b, x.rn0, x.rn1, p.n, true, 0)) return;
      store_rows(x, p.Z, p.n, b, x.rn0, x.rn1);
      sync_group(x);
      gemm_rows(x, p.Mt, p.n, p.n, p.Z, p.n, b, x.rm0, x.rm1);
      if (!orth_pass(x, b, x.rm0, x.rm1, p.m, true, 0)) return;
      store_rows(x, p.Q, p.m, b, x.rm0, x.rm1);
      sync_group(x);
    }
    // Rayleigh-Ritz: Q <- orth(Q); M^T Q = Qb Rb; Rb^T = Ub S J^T
    load_rows(x, p.Q, p.m, b, x.rm0, x.rm1);
    if (!orth_pass(x, b, x.rm0, x.rm1, p.m, false, 0)) return;
    store_rows(x, p.Q, p.m, b, x.rm0, x.rm1);
    sync_group(x);
    gemm_rows(x, p.M, p.m, p.m, p.Q, p.m, b, x.rn0, x.rn1);
    if (!orth_pass(x, b, x.rn0, x.rn1, p.n, true, 1)) return;
    if (!orth_pass(x, b, x.rn0, x.rn1, p.n, false, 2)) return;
    if (!orth_pass(x, b, x.rn0, x.rn1, p.n, false, 2)) return;
    store_rows(x, p.Z, p.n, b, x.rn0, x.rn1);
    sync_group(x);
    if (x.c == 0) ritz_small(x, b);
    sync_group(x);
    if (__ldcg(&p.info[0]) != ST_OK) return;
    rotate_rows(x, p.Q, p.m, p.Ub, b, k, p.U, p.m, x.rm0, x.rm1);
    rotate_rows(x, p.Z, p.n, p.Jo, b, k, p.V, p.n, x.rn0, x.rn1);
    sync_group(x);
    // residuals ||M v_i - s_i u_i||^2, partial over the owned m-rows
    gemm_rows(x, p.Mt, p.n, p.n, p.V, p.n, k, x.rm0, x.rm1);
    {
      const double* Ys = sm + OFF_Y;
      double* gp = p.Gp + (size_t)x.c * KMAXB * KMAXB;
      const int R = x.rm1 - x.rm0;
      for (int i = threadIdx.x; i < k; i += TT) {
        const double si = __ldcg(&p.s[i]);
        double v = 0.0;
        for (int r = 0; r < R; ++r) {
          const double d = Ys[r * YLD + i] - si * __ldcg(&p.U[(size_t)i * p.m + x.rm0 + r]);
          v = fma(d, d, v);
        }
        gp[i] = v;
      }
    }
    sync_group(x);
    if (x.c == 0 && threadIdx.x == 0) {
      const double s0 = __ldcg(&p.s[0]);
      const double fro = sqrt(__ldcg(&p.info[2]));
      const double thr = fmax(tol * s0, 8.0 * DBL_EPSILON * sqrt((double)max(p.m, p.n)) * fro);
      double worst = 0.0;
      bool zero = false;
      for (int i = 0; i < k; ++i) {
        double v = 0.0;
        for (int q = 0; q < p.P; ++q) v += __ldcg(&p.Gp[(size_t)q * KMAXB * KMAXB + i]);
        worst = fmax(worst, thr > 0.0 ? sqrt(v) / thr : 0.0);
        zero |= !(__ldcg(&p.s[i]) > 0.0);
      }
      p.info[1] = it;
      p.info[3] = worst;
      int done = 0;
      if (zero) {
        p.info[0] = ST_ZERO;
        done = 1;
      } else if (worst <= 1.0) {
        done = 1;
      } else if (it + qstep > qmax) {
        p.info[0] = ST_NOCONV;
        done = 1;
      }
      p.info[4] = done;
    }
    sync_group(x);
    if (__ldcg(&p.info[4]) != 0.0) return;
    target = it + qstep;
  }
}

// ---------------------------------------------------------------------------
// host driver
// ---------------------------------------------------------------------------

int topk_block_size(int k, int m, int n) {
  int b = k + std::max(16, std::min(k, 32));
  b = std::min(b, KMAXB);
  b += b & 1;
  if (b > KMAXB || 2 * b > std::min(m, n) || k < 1) return 0;
  return b;
}

bool topk_fits(int k, int m, int n, int nprob, Engine& E) {
  const int b = topk_block_size(k, m, n);
  if (b == 0) return false;
  const int P = (std::max(m, n) + RMAX - 1) / RMAX;
  return P * nprob <= E.num_sms;
}

void svd_topk(Engine& E, std::vector<TopkDesc>& ds, double tol) {
  if (ds.empty()) return;
  static bool attr = false;
  const size_t smem = sizeof(double) * SMEM_DOUBLES;
  if (!attr) {
    SPS_CUDA(cudaFuncSetAttribute(topk_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    attr = true;
  }
  int per_sm = 0;
  SPS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, topk_kernel, TT, smem));
  const int capacity = std::max(1, per_sm) * E.num_sms;
  const int nprob = (int)ds.size();
  std::vector<TopkProb> hp(nprob);
  std::vector<Buf> keep;
  int cta = 0;
  for (int i = 0; i < nprob; ++i) {
    TopkDesc& d = ds[i];
    const int m = d.m, n = d.n;
    d.b = topk_block_size(d.k, m, n);
    if (d.b == 0) throw Error(SPS_ERR_ARGUMENT, "svd_topk: block too small for subspace iteration");
    const int mx = std::max(m, n);
    int P = (mx + 11) / 12;                       // about 12 owned rows per CTA
    P = std::max(P, (mx + RMAX - 1) / RMAX);
    P = std::min(P, capacity / nprob);
    if ((mx + P - 1) / P > RMAX) throw Error(SPS_ERR_ARGUMENT, "svd_topk: block too large for the grid");
    const int b = d.b;
    const size_t nd = (size_t)n * m + (size_t)m * b + (size_t)n * b + (size_t)P * KMAXB * KMAXB + 4 * (size_t)b * b +
                      b + P + 8;
    Buf w = E.alloc(sizeof(double) * nd + 64);
    keep.push_back(w);
    double* base = (double*)w->ptr;
    TopkProb& p = hp[i];
    p.M = d.M;
    double* mt = base;
    p.Mt = mt;
    base += (size_t)n * m;
    p.m = m;
    p.n = n;
    p.k = d.k;
    p.b = b;
    p.P = P;
    p.cta0 = cta;
    cta += P;
    p.Q = base;
    base += (size_t)m * b;
    p.Z = base;
    base += (size_t)n * b;
    p.Gp = base;
    base += (size_t)P * KMAXB * KMAXB;
    p.G = base;
    base += (size_t)b * b;
    p.Racc = base;
    base += (size_t)b * b;
    p.Ub = base;
    base += (size_t)b * b;
    p.Jo = base;
    base += (size_t)b * b;
    p.s = base;
    base += b;
    p.fpart = base;
    base += P;
    p.info = base;
    base += 6;
    p.bar = (unsigned*)(base);
    p.U = d.U;
    p.V = d.V;
    SPS_CUDA(cudaMemsetAsync(p.info, 0, sizeof(double) * 6 + 8, E.stream));
    transpose_cm(E, d.M, m, n, m, mt, n);
  }
  Buf pb = E.alloc(sizeof(TopkProb) * nprob);
  keep.push_back(pb);
  E.stage(hp.data(), sizeof(TopkProb) * nprob, pb->ptr);
  const TopkProb* dp = (const TopkProb*)pb->ptr;
  int q0 = std::max(2, E.topk_hint), qstep = 2, qmax = 48;
  int* flag = E.dflag;
  void* args[] = {(void*)&dp, (void*)&nprob, (void*)&q0, (void*)&qstep, (void*)&qmax, (void*)&tol, (void*)&flag};
  const int tid = E.tic("svd_topk");
  SPS_CUDA(cudaLaunchCooperativeKernel((const void*)topk_kernel, dim3(cta), dim3(TT), args, smem, E.stream));
  E.launches++;
  // info and Ritz values to the host
  int off = 0;
  for (int i = 0; i < nprob; ++i) {
    SPS_CUDA(cudaMemcpyAsync(E.hscal + off, hp[i].info, sizeof(double) * 6, cudaMemcpyDeviceToHost, E.stream));
    SPS_CUDA(cudaMemcpyAsync(E.hscal + off + 6, hp[i].s, sizeof(double) * hp[i].b, cudaMemcpyDeviceToHost,
                             E.stream));
    off += 6 + hp[i].b;
  }
  if (off > Engine::NSCAL) throw Error(SPS_ERR_ARGUMENT, "svd_topk: too many values");
  E.sync();
  E.check_flag("svd_topk");
  off = 0;
  int qused = 0;
  for (int i = 0; i < nprob; ++i) {
    TopkDesc& d = ds[i];
    d.status = (int)E.hscal[off];
    d.iterations = (int)E.hscal[off + 1];
    d.fro2 = E.hscal[off + 2];
    d.residual = E.hscal[off + 3];
    d.s.assign(E.hscal + off + 6, E.hscal + off + 6 + d.b);
    qused = std::max(qused, d.iterations);
    off += 6 + d.b;
  }
  // work of the launch: 2 m n b flops per half-iteration, plus the extraction
  double fl = 0;
  for (auto& d : ds) fl += (4.0 * d.iterations + 6.0) * d.m * d.n * d.b;
  E.toc(tid, fl);
  // next starting count: the count that converged; after four first-check
  // successes in a row, one less
  if (qused > q0) {
    E.topk_hint = qused;
    E.topk_streak = 0;
  } else if (qused == q0 && ++E.topk_streak >= 4) {
    E.topk_hint = std::max(2, q0 - 1);
    E.topk_streak = 0;
  }
}

}  // namespace la
}  // namespace sps
