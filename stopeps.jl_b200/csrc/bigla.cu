// Multi-CTA factorizations for the large parity blocks of the boundary
// compression (e.g. 23328 x 648 and 648 x 648 at chi=36, D=6):
//
//  * blocked Householder QR: a cooperative panel kernel (one pass over the
//    panel rows per column, two grid barriers per column) and compact-WY
//    trailing updates / Q formation as dense FP64 GEMMs (dgemm.cu);
//  * one-sided Jacobi SVD with every column pair of a round rotated by its
//    own warp across the whole GPU and a grid barrier between rounds.
//
// Grid barriers are software barriers inside cooperative launches (all CTAs
// co-resident); every spin is bounded and reports through the device flag.
#include "engine.h"
#include "coop.cuh"
#include <cfloat>
#include <cstring>
#include <algorithm>
#include <initializer_list>
#include <mutex>
#include <set>

namespace sps {
namespace la {

static constexpr int BT = 256;
static constexpr int BW = BT / 32;

__device__ double bsum(double v, double* red) {
  v = wsum(v);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0;
    for (int w = 0; w < BW; ++w) s += red[w];
    red[BW] = s;
  }
  __syncthreads();
  return red[BW];
}

__device__ void grid_barrier(unsigned* bar, int* flag) { group_barrier(bar, gridDim.x, flag); }


// ---------------------------------------------------------------------------
// cooperative panel factorization
// ---------------------------------------------------------------------------
struct PanelArgs {
  double* A;
  int lda, m, j0, jb;
  double* tau;       // tau[j0 .. j0+jb)
  double* V;         // explicit V (m x n, ld m): panel columns written
  double* T;         // jb x jb (col-major) compact-WY factor of this panel
  double* acc;       // scratch: accn[jb], alpha[jb], accw[jb*jb], gram[jb*jb] (zeroed)
  unsigned* bar;
  int* flag;
  int rpc;           // rows per CTA
};

__global__ void __launch_bounds__(BT) panel_qr_kernel(PanelArgs p) {
  extern __shared__ double sm[];   // panel rows of this CTA, column-major: sm[c * ld + r]
  __shared__ double red[BW + 1];
  const int jb = p.jb;
  const int ld = p.rpc;
  const int r0 = p.j0 + blockIdx.x * p.rpc;
  const int r1 = min(p.m, r0 + p.rpc);
  const int nr = max(0, r1 - r0);
  double* accn = p.acc;
  double* alph = accn + jb;
  double* accw = alph + jb;
  double* gram = accw + jb * jb;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int e = threadIdx.x; e < nr * jb; e += BT) {
    int c = e / nr, r = e % nr;
    sm[c * ld + r] = p.A[(size_t)(r0 + r) + (size_t)(p.j0 + c) * p.lda];
  }
  __syncthreads();
  for (int jj = 0; jj < jb; ++jj) {
    const int j = p.j0 + jj;
    const bool owner = (j >= r0 && j < r1);
    const int rs = max(0, j + 1 - r0);   // first local row strictly below the pivot
    double* cj = sm + jj * ld;
    double part = 0;
    for (int r = rs + threadIdx.x; r < nr; r += BT) part += cj[r] * cj[r];
    part = bsum(part, red);
    if (threadIdx.x == 0) {
      if (part != 0.0) atomicAdd(&accn[jj], part);
      if (owner) alph[jj] = cj[j - r0];
    }
    grid_barrier(p.bar, p.flag);
    const double sumsq = __ldcg(&accn[jj]);
    const double alpha = __ldcg(&alph[jj]);
    double tau = 0.0, scal = 0.0, beta = alpha;
    if (sumsq != 0.0) {
      beta = -copysign(sqrt(alpha * alpha + sumsq), alpha);
      tau = (beta - alpha) / beta;
      scal = 1.0 / (alpha - beta);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) p.tau[j] = tau;
    if (tau != 0.0) {
      for (int r = rs + threadIdx.x; r < nr; r += BT) cj[r] *= scal;
      if (owner && threadIdx.x == 0) cj[j - r0] = beta;
      __syncthreads();
      for (int kk = jj + 1 + warp; kk < jb; kk += BW) {
        const double* ck = sm + kk * ld;
        double w = 0;
        for (int r = rs + lane; r < nr; r += 32) w += cj[r] * ck[r];
        if (owner && lane == 0) w += ck[j - r0];
        w = wsum(w);
        if (lane == 0 && w != 0.0) atomicAdd(&accw[jj * jb + kk], w);
      }
      grid_barrier(p.bar, p.flag);
      for (int kk = jj + 1 + warp; kk < jb; kk += BW) {
        double* ck = sm + kk * ld;
        const double w = __ldcg(&accw[jj * jb + kk]) * tau;
        for (int r = rs + lane; r < nr; r += 32) ck[r] -= cj[r] * w;
        if (owner && lane == 0) ck[j - r0] -= w;
      }
    }
    __syncthreads();
  }
  // write back, explicit V, partial Gram V^T V
  for (int e = threadIdx.x; e < nr * jb; e += BT) {
    int c = e / nr, r = e % nr;
    int gr = r0 + r, gc = p.j0 + c;
    double x = sm[c * ld + r];
    p.A[(size_t)gr + (size_t)gc * p.lda] = x;
    double v = gr < gc ? 0.0 : (gr == gc ? 1.0 : x);
    p.V[(size_t)gr + (size_t)gc * p.m] = v;
    sm[c * ld + r] = v;
  }
  __syncthreads();
  for (int pr = warp; pr < jb * jb; pr += BW) {
    int a = pr / jb, b = pr % jb;
    if (b < a) continue;
    const double* ca = sm + a * ld;
    const double* cb = sm + b * ld;
    double s = 0;
    for (int r = lane; r < nr; r += 32) s += ca[r] * cb[r];
    s = wsum(s);
    if (lane == 0 && s != 0.0) atomicAdd(&gram[a * jb + b], s);
  }
  grid_barrier(p.bar, p.flag);
  if (blockIdx.x == 0) {
    // T(i,i) = tau_i ; T(0:i, i) = -tau_i T(0:i,0:i) V(:,0:i)^T v_i  (dlarft, forward, columnwise),
    // built in shared memory: column i is a triangular mat-vec over the already built columns.
    double* Ts = sm;                  // jb x jb, column-major
    double* Gs = sm + jb * jb;        // Gram (upper part used)
    for (int e = threadIdx.x; e < jb * jb; e += BT) {
      Ts[e] = 0.0;
      int a = e / jb, b = e % jb;
      Gs[e] = a <= b ? __ldcg(&gram[a * jb + b]) : 0.0;   // Gs[a*jb + b] = (V^T V)(a,b), a <= b
    }
    __syncthreads();
    for (int i = 0; i < jb; ++i) {
      const double ti = __ldcg(&p.tau[p.j0 + i]);
      double v = 0;
      if (threadIdx.x < i) {
        const int a = threadIdx.x;
        for (int b = a; b < i; ++b) v += Ts[a + b * jb] * Gs[b * jb + i];
      }
      __syncthreads();
      if (threadIdx.x < i) Ts[threadIdx.x + i * jb] = -ti * v;
      if (threadIdx.x == 0) Ts[i + i * jb] = ti;
      __syncthreads();
    }
    for (int e = threadIdx.x; e < jb * jb; e += BT) p.T[e] = Ts[e];
  }
}

void copy_upper_and_identity(Engine& E, const double* a, int m, int n, int lda, double* r, int ldr, double* q,
                             int ldq);

// Allow a kernel the current device's full opt-in shared memory (once per
// device and kernel): a per-call attribute with the call's own size would race
// between host threads that launch the same kernel with different sizes.
static void allow_max_smem(const void* kernel) {
  int dev = 0, maxopt = 0;
  SPS_CUDA(cudaGetDevice(&dev));
  SPS_CUDA(cudaDeviceGetAttribute(&maxopt, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  cudaFuncAttributes fa;
  SPS_CUDA(cudaFuncGetAttributes(&fa, kernel));   // static shared memory counts against the limit
  set_max_dynamic_smem(kernel, maxopt - (int)fa.sharedSizeBytes);
}

static int coop_blocks(const void* kernel, int threads, size_t smem, Engine& E) {
  return E.coop_capacity(occupancy_per_sm(kernel, threads, smem));
}

// Householder QR of a (m x n, col-major lda), m >= n: q (m x n, ldq), r (n x n, ldr).
void qr_big(Engine& E, double* a, int m, int n, int lda, double* q, int ldq, double* r, int ldr) {
  qr_big_opt(E, a, m, n, lda, q, ldq, r, ldr, true);
}

void qr_big_opt(Engine& E, double* a, int m, int n, int lda, double* q, int ldq, double* r, int ldr, bool form_q) {
  const int jb_max = 32;
  const int np = (n + jb_max - 1) / jb_max;
  Buf vb = E.alloc(sizeof(double) * (size_t)m * n);
  Buf tb = E.alloc(sizeof(double) * (size_t)np * jb_max * jb_max);
  Buf taub = E.alloc(sizeof(double) * n);
  Buf accb = E.alloc(sizeof(double) * (size_t)np * (2 * jb_max + 2 * jb_max * jb_max));
  Buf barb = E.alloc(sizeof(unsigned) * 2 * np);
  Buf wb = E.alloc(sizeof(double) * (size_t)jb_max * n * 2);
  double* V = (double*)vb->ptr;
  double* T = (double*)tb->ptr;
  double* W = (double*)wb->ptr;
  double* W2 = W + (size_t)jb_max * n;
  SPS_CUDA(cudaMemsetAsync(accb->ptr, 0, sizeof(double) * (size_t)np * (2 * jb_max + 2 * jb_max * jb_max), E.stream));
  SPS_CUDA(cudaMemsetAsync(barb->ptr, 0, sizeof(unsigned) * 2 * np, E.stream));
  SPS_CUDA(cudaMemsetAsync(T, 0, sizeof(double) * (size_t)np * jb_max * jb_max, E.stream));
  for (int pi = 0; pi < np; ++pi) {
    int j0 = pi * jb_max, jb = std::min(jb_max, n - j0);
    int mrows = m - j0;
    int maxg = coop_blocks((const void*)panel_qr_kernel, BT, 0, E);
    int G = std::min({E.num_sms, maxg, std::max(1, (mrows + 63) / 64)});
    int rpc = (mrows + G - 1) / G;
    size_t smem = sizeof(double) * std::max((size_t)rpc * jb, (size_t)2 * jb * jb);
    if (smem > 200 * 1024) {
      G = std::min(maxg, (int)((mrows * (size_t)jb * 8 + 200 * 1024 - 1) / (200 * 1024)));
      rpc = (mrows + G - 1) / G;
      smem = sizeof(double) * std::max((size_t)rpc * jb, (size_t)2 * jb * jb);
      if (smem > 200 * 1024) throw Error(SPS_ERR_ARGUMENT, "qr_big: panel too tall for shared memory");
    }
    allow_max_smem((const void*)panel_qr_kernel);
    PanelArgs pa;
    pa.A = a;
    pa.lda = lda;
    pa.m = m;
    pa.j0 = j0;
    pa.jb = jb;
    pa.tau = (double*)taub->ptr;
    pa.V = V;
    pa.T = T + (size_t)pi * jb_max * jb_max;
    pa.acc = (double*)accb->ptr + (size_t)pi * (2 * jb_max + 2 * jb_max * jb_max);
    pa.bar = (unsigned*)barb->ptr + 2 * pi;
    pa.flag = E.dflag;
    pa.rpc = rpc;
    void* args[] = {&pa};
    int tk = E.tic("qr_panel");
    SPS_CUDA(cudaLaunchCooperativeKernel((const void*)panel_qr_kernel, dim3(G), dim3(BT), args, smem, E.stream));
    E.toc(tk, 2.0 * mrows * jb * (double)jb, 16.0 * mrows * jb);
    E.launches++;
    int n2 = n - j0 - jb;
    if (n2 > 0) {
      const double* Vp = V + j0 + (size_t)j0 * m;
      double* A2 = a + j0 + (size_t)(j0 + jb) * lda;
      dgemm_cm(E, true, jb, n2, mrows, 1.0, Vp, m, A2, lda, 0.0, W, jb);                      // W = V^T A2
      dgemm_cm(E, true, jb, n2, jb, 1.0, pa.T, jb, W, jb, 0.0, W2, jb);                       // W2 = T^T W
      dgemm_cm(E, false, mrows, n2, jb, -1.0, Vp, m, W2, jb, 1.0, A2, lda);                   // A2 -= V W2
    }
  }
  // R (upper triangle of a) and Q = H_1 ... H_np [I; 0]
  copy_upper_and_identity(E, a, m, n, lda, r, ldr, form_q ? q : nullptr, ldq);
  if (!form_q) return;
  for (int pi = np - 1; pi >= 0; --pi) {
    int j0 = pi * jb_max, jb = std::min(jb_max, n - j0);
    int mrows = m - j0, nc = n - j0;
    const double* Vp = V + j0 + (size_t)j0 * m;
    const double* Tp = T + (size_t)pi * jb_max * jb_max;
    double* Q2 = q + j0 + (size_t)j0 * ldq;
    dgemm_cm(E, true, jb, nc, mrows, 1.0, Vp, m, Q2, ldq, 0.0, W, jb);       // W = V^T Q2
    dgemm_cm(E, false, jb, nc, jb, 1.0, Tp, jb, W, jb, 0.0, W2, jb);         // W2 = T W
    dgemm_cm(E, false, mrows, nc, jb, -1.0, Vp, m, W2, jb, 1.0, Q2, ldq);    // Q2 -= V W2
  }
}

__global__ void upper_identity_kernel(const double* a, int m, int n, int lda, double* r, int ldr, double* q, int ldq) {
  size_t tr = (size_t)n * n, tq = (size_t)m * n;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < tr + tq; e += (size_t)gridDim.x * blockDim.x) {
    if (e < tr) {
      int i = (int)(e % n), j = (int)(e / n);
      r[i + (size_t)j * ldr] = i <= j ? a[i + (size_t)j * lda] : 0.0;
    } else if (q) {
      size_t f = e - tr;
      int i = (int)(f % m), j = (int)(f / m);
      q[i + (size_t)j * ldq] = i == j ? 1.0 : 0.0;
    }
  }
}

void copy_upper_and_identity(Engine& E, const double* a, int m, int n, int lda, double* r, int ldr, double* q,
                             int ldq) {
  size_t total = (size_t)n * n + (q ? (size_t)m * n : 0);
  int g = (int)std::min<size_t>((total + 255) / 256, 8192);
  upper_identity_kernel<<<g, 256, 0, E.stream>>>(a, m, n, lda, r, ldr, q, ldq);
  SPS_CUDA(cudaGetLastError());
  E.launches++;
}

// ---------------------------------------------------------------------------
// cooperative one-sided Jacobi SVD over several problems (m >= n each)
// ---------------------------------------------------------------------------
struct JacProb {
  double* U;     // m x n (ld m), rotated in place
  double* V;     // n x n (ld n) workspace
  double* q;     // output U sorted (ld m)
  double* r;     // output V sorted (ld n)
  double* s;     // output singular values (descending)
  double* sig;   // n scratch
  int* rank;     // n scratch
  int m, n;
  int pair_base; // first global pair index of this problem
};

__device__ __forceinline__ int rr_idx(int i, int round, int np) {
  return i == 0 ? 0 : ((i - 1 + round) % (np - 1)) + 1;
}

__global__ void __launch_bounds__(BT) jacobi_coop_kernel(const JacProb* probs, int nprob, int total_pairs,
                                                         int max_rounds, unsigned* bar, int* counters, int* flag) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int gw = blockIdx.x * BW + warp, TW = gridDim.x * BW;
  // V = I
  for (int pi = 0; pi < nprob; ++pi) {
    const JacProb P = probs[pi];
    size_t nn = (size_t)P.n * P.n;
    for (size_t e = blockIdx.x * (size_t)BT + threadIdx.x; e < nn; e += (size_t)gridDim.x * BT)
      P.V[e] = (e % P.n == e / P.n) ? 1.0 : 0.0;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    counters[0] = 0;
    counters[1] = 0;
    counters[2] = 0;
  }
  grid_barrier(bar, flag);
  const int MAXSWEEP = 80;
  bool converged = false;
  for (int sweep = 0; sweep < MAXSWEEP; ++sweep) {
    int* cnt = counters + (sweep % 3);
    if (blockIdx.x == 0 && threadIdx.x == 0) counters[(sweep + 1) % 3] = 0;
    for (int round = 0; round < max_rounds; ++round) {
      for (int t = gw; t < total_pairs; t += TW) {
        int pi = 0;
        while (pi + 1 < nprob && t >= probs[pi + 1].pair_base) ++pi;
        const JacProb& P = probs[pi];
        const int np = P.n + (P.n & 1);
        if (round >= np - 1) continue;
        int pr = t - P.pair_base;
        int p = rr_idx(pr, round, np), qd = rr_idx(np - 1 - pr, round, np);
        if (p >= P.n || qd >= P.n) continue;
        if (p > qd) { int tt = p; p = qd; qd = tt; }
        double* up = P.U + (size_t)p * P.m;
        double* uq = P.U + (size_t)qd * P.m;
        double al = 0, be = 0, ga = 0;
        for (int i = lane; i < P.m; i += 32) {
          double x = up[i], y = uq[i];
          al += x * x;
          be += y * y;
          ga += x * y;
        }
        al = wsum(al);
        be = wsum(be);
        ga = wsum(ga);
        const double tol = DBL_EPSILON * (double)max(P.m, 2);
        if (!(al >= DBL_MIN && be >= DBL_MIN) || ga == 0.0 || !(fabs(ga) > tol * sqrt(al) * sqrt(be))) continue;
        double zeta = (be - al) / (2.0 * ga);
        double tt = copysign(1.0, zeta) / (fabs(zeta) + hypot(1.0, zeta));
        double c = 1.0 / sqrt(1.0 + tt * tt), s = c * tt;
        for (int i = lane; i < P.m; i += 32) {
          double x = up[i], y = uq[i];
          up[i] = c * x - s * y;
          uq[i] = s * x + c * y;
        }
        double* vp = P.V + (size_t)p * P.n;
        double* vq = P.V + (size_t)qd * P.n;
        for (int i = lane; i < P.n; i += 32) {
          double x = vp[i], y = vq[i];
          vp[i] = c * x - s * y;
          vq[i] = s * x + c * y;
        }
        if (lane == 0) atomicAdd(cnt, 1);
      }
      grid_barrier(bar, flag);
    }
    int rot = *(volatile int*)cnt;
    if (rot == 0) {
      converged = true;
      break;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    if (!converged) atomicOr(flag, FLAG_CONV);
    atomicMax(flag + 1, 1000 + 0);   // marks the element-pair kernel
  }
  // singular values
  for (int pi = 0; pi < nprob; ++pi) {
    const JacProb P = probs[pi];
    for (int c = gw; c < P.n; c += TW) {
      const double* uc = P.U + (size_t)c * P.m;
      double v = 0;
      for (int i = lane; i < P.m; i += 32) v += uc[i] * uc[i];
      v = wsum(v);
      if (lane == 0) P.sig[c] = sqrt(v);
    }
  }
  grid_barrier(bar, flag);
  for (int pi = 0; pi < nprob; ++pi) {
    const JacProb P = probs[pi];
    for (int c = blockIdx.x * BT + threadIdx.x; c < P.n; c += gridDim.x * BT) {
      double sc = __ldcg(&P.sig[c]);
      int rk = 0;
      for (int j = 0; j < P.n; ++j) {
        double sj = __ldcg(&P.sig[j]);
        rk += (sj > sc) || (sj == sc && j < c);
      }
      P.rank[c] = rk;
      P.s[rk] = sc;
    }
  }
  grid_barrier(bar, flag);
  for (int pi = 0; pi < nprob; ++pi) {
    const JacProb P = probs[pi];
    for (int c = gw; c < P.n; c += TW) {
      int rk = __ldcg(&P.rank[c]);
      double sc = __ldcg(&P.sig[c]);
      double inv = sc > 0 ? 1.0 / sc : 0.0;
      const double* uc = P.U + (size_t)c * P.m;
      double* qo = P.q + (size_t)rk * P.m;
      for (int i = lane; i < P.m; i += 32) qo[i] = uc[i] * inv;
      const double* vc = P.V + (size_t)c * P.n;
      double* ro = P.r + (size_t)rk * P.n;
      for (int i = lane; i < P.n; i += 32) ro[i] = vc[i];
    }
  }
}

// ---------------------------------------------------------------------------
// block one-sided Jacobi: columns in blocks of BJW; each round pairs blocks
// and one CTA orthogonalizes the 2*BJW columns of its pair in shared memory
// (inner one-sided Jacobi sweeps), then applies the accumulated 2BJW x 2BJW
// rotation to V.  A grid barrier separates rounds (nblk-1 per sweep).
// ---------------------------------------------------------------------------
static constexpr int BJW = 16;
static constexpr int BJ2 = 2 * BJW;

__global__ void __launch_bounds__(BT) bjacobi_kernel(const JacProb* probs, int nprob, int total_pairs,
                                                     int max_rounds, unsigned* bar, int* counters, int* flag,
                                                     int* sweeps_out) {
  extern __shared__ double smem[];
  double* W = smem;                 // BJ2 x BJ2, column-major
  double* Ub = smem + BJ2 * BJ2;    // m x BJ2, column-major (ld m)
  __shared__ int inner_rot;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int pi = 0; pi < nprob; ++pi) {
    const JacProb P = probs[pi];
    size_t nn = (size_t)P.n * P.n;
    for (size_t e = blockIdx.x * (size_t)BT + threadIdx.x; e < nn; e += (size_t)gridDim.x * BT)
      P.V[e] = (e % P.n == e / P.n) ? 1.0 : 0.0;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    counters[0] = 0;
    counters[1] = 0;
    counters[2] = 0;
  }
  grid_barrier(bar, flag);
  const int MAXSWEEP = 60;
  bool converged = false;
  int sweep = 0;
  for (; sweep < MAXSWEEP; ++sweep) {
    int* cnt = counters + (sweep % 3);
    if (blockIdx.x == 0 && threadIdx.x == 0) counters[(sweep + 1) % 3] = 0;
    for (int round = 0; round < max_rounds; ++round) {
      for (int t = blockIdx.x; t < total_pairs; t += gridDim.x) {
        int pi = 0;
        while (pi + 1 < nprob && t >= probs[pi + 1].pair_base) ++pi;
        const JacProb& P = probs[pi];
        const int nb = (P.n + BJW - 1) / BJW;
        const int nbp = nb + (nb & 1);
        if (round >= nbp - 1) continue;
        const int pr = t - P.pair_base;
        int bi = rr_idx(pr, round, nbp), bj = rr_idx(nbp - 1 - pr, round, nbp);
        if (bi >= nb || bj >= nb) continue;
        if (bi > bj) { int tt = bi; bi = bj; bj = tt; }
        const int c0 = bi * BJW, w1 = min(BJW, P.n - c0);
        const int c1 = bj * BJW, w2 = min(BJW, P.n - c1);
        const int wt = w1 + w2, m = P.m;
        // load the two column blocks and W = I
        for (int e = threadIdx.x; e < wt * m; e += BT) {
          int k = e / m, i = e % m;
          int gc = k < w1 ? c0 + k : c1 + (k - w1);
          Ub[i + (size_t)k * m] = P.U[i + (size_t)gc * m];
        }
        for (int e = threadIdx.x; e < BJ2 * BJ2; e += BT) W[e] = (e % BJ2 == e / BJ2) ? 1.0 : 0.0;
        __syncthreads();
        const double tol = DBL_EPSILON * (double)max(m, 2);
        const int wtp = wt + (wt & 1);
        bool any = false;
        for (int inner = 0; inner < 12; ++inner) {
          if (threadIdx.x == 0) inner_rot = 0;
          __syncthreads();
          for (int ir = 0; ir < wtp - 1; ++ir) {
            for (int q = warp; q < wtp / 2; q += BW) {
              int a = rr_idx(q, ir, wtp), b = rr_idx(wtp - 1 - q, ir, wtp);
              if (a >= wt || b >= wt) continue;
              if (a > b) { int tt = a; a = b; b = tt; }
              double* ua = Ub + (size_t)a * m;
              double* ub = Ub + (size_t)b * m;
              double al = 0, be = 0, ga = 0;
              for (int i = lane; i < m; i += 32) {
                double x = ua[i], y = ub[i];
                al += x * x;
                be += y * y;
                ga += x * y;
              }
              al = wsum(al);
              be = wsum(be);
              ga = wsum(ga);
              if (!(al >= DBL_MIN && be >= DBL_MIN) || ga == 0.0 || !(fabs(ga) > tol * sqrt(al) * sqrt(be))) continue;
              double zeta = (be - al) / (2.0 * ga);
              double tt = copysign(1.0, zeta) / (fabs(zeta) + hypot(1.0, zeta));
              double c = 1.0 / sqrt(1.0 + tt * tt), s = c * tt;
              for (int i = lane; i < m; i += 32) {
                double x = ua[i], y = ub[i];
                ua[i] = c * x - s * y;
                ub[i] = s * x + c * y;
              }
              if (lane < wt) {
                double x = W[lane + a * BJ2], y = W[lane + b * BJ2];
                W[lane + a * BJ2] = c * x - s * y;
                W[lane + b * BJ2] = s * x + c * y;
              }
              if (lane == 0) inner_rot = 1;
            }
            __syncthreads();
          }
          bool rot = inner_rot != 0;
          __syncthreads();
          if (!rot) break;
          any = true;
        }
        if (any) {
          if (threadIdx.x == 0) atomicAdd(cnt, 1);
          for (int e = threadIdx.x; e < wt * m; e += BT) {
            int k = e / m, i = e % m;
            int gc = k < w1 ? c0 + k : c1 + (k - w1);
            P.U[i + (size_t)gc * m] = Ub[i + (size_t)k * m];
          }
          // V[:, cols] <- V[:, cols] W : one warp per row, lane c owns output column c
          for (int i = warp; i < P.n; i += BW) {
            double vi = 0;
            if (lane < wt) {
              int gc = lane < w1 ? c0 + lane : c1 + (lane - w1);
              vi = P.V[i + (size_t)gc * P.n];
            }
            double out = 0;
            for (int k = 0; k < wt; ++k) {
              double vk = __shfl_sync(0xffffffffu, vi, k);
              if (lane < wt) out += vk * W[k + lane * BJ2];
            }
            if (lane < wt) {
              int gc = lane < w1 ? c0 + lane : c1 + (lane - w1);
              P.V[i + (size_t)gc * P.n] = out;
            }
          }
        }
        __syncthreads();
      }
      grid_barrier(bar, flag);
    }
    int rot = *(volatile int*)cnt;
    if (rot == 0) {
      converged = true;
      break;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    if (!converged) atomicOr(flag, FLAG_CONV);
    atomicMax(sweeps_out, sweep + 1);
    atomicMax(flag + 1, sweep + 1);
  }
  // singular values, order, outputs (as in jacobi_coop_kernel)
  const int gw = blockIdx.x * BW + warp, TW = gridDim.x * BW;
  for (int pi = 0; pi < nprob; ++pi) {
    const JacProb P = probs[pi];
    for (int c = gw; c < P.n; c += TW) {
      const double* uc = P.U + (size_t)c * P.m;
      double v = 0;
      for (int i = lane; i < P.m; i += 32) v += uc[i] * uc[i];
      v = wsum(v);
      if (lane == 0) P.sig[c] = sqrt(v);
    }
  }
  grid_barrier(bar, flag);
  for (int pi = 0; pi < nprob; ++pi) {
    const JacProb P = probs[pi];
    for (int c = blockIdx.x * BT + threadIdx.x; c < P.n; c += gridDim.x * BT) {
      double sc = __ldcg(&P.sig[c]);
      int rk = 0;
      for (int j = 0; j < P.n; ++j) {
        double sj = __ldcg(&P.sig[j]);
        rk += (sj > sc) || (sj == sc && j < c);
      }
      P.rank[c] = rk;
      P.s[rk] = sc;
    }
  }
  grid_barrier(bar, flag);
  for (int pi = 0; pi < nprob; ++pi) {
    const JacProb P = probs[pi];
    for (int c = gw; c < P.n; c += TW) {
      int rk = __ldcg(&P.rank[c]);
      double sc = __ldcg(&P.sig[c]);
      double inv = sc > 0 ? 1.0 / sc : 0.0;
      const double* uc = P.U + (size_t)c * P.m;
      double* qo = P.q + (size_t)rk * P.m;
      for (int i = lane; i < P.m; i += 32) qo[i] = uc[i] * inv;
      const double* vc = P.V + (size_t)c * P.n;
      double* ro = P.r + (size_t)rk * P.n;
      for (int i = lane; i < P.n; i += 32) ro[i] = vc[i];
    }
  }
}

// ---------------------------------------------------------------------------
// U-only one-sided Jacobi: rotates the columns of X (m x n, ld m) until they
// are orthogonal, then writes the normalized columns sorted by descending
// norm (the left singular vectors of X) and the norms (singular values).
// No right factor is accumulated: callers recover what they need by one GEMM
// with the original matrix.  One warp per column pair, the pair's two columns
// held in registers; a grid barrier between rounds.
// ---------------------------------------------------------------------------
static constexpr int JR = 24;   // registers per lane per column: m <= 32*JR

struct JUProb {
  double* X;      // m x n (ld m), rotated in place
  double* q;      // output: sorted normalized columns (m x n, ld m)
  double* s;      // output: sorted norms (n)
  double* sig;    // scratch n
  int* rank;      // scratch n
  int m, n;
  int pair_base;
};

template <bool REG>
__global__ void __launch_bounds__(BT) jacobi_u_kernel(const JUProb* probs, int nprob, int total_pairs,
                                                      int max_rounds, unsigned* bar, int* counters, int* flag) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int gw = blockIdx.x * BW + warp, TW = gridDim.x * BW;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    counters[0] = 0;
    counters[1] = 0;
    counters[2] = 0;
  }
  grid_barrier(bar, flag);
  const int MAXSWEEP = 80;
  bool converged = false;
  int sweep = 0;
  for (; sweep < MAXSWEEP; ++sweep) {
    int* cnt = counters + (sweep % 3);
    if (blockIdx.x == 0 && threadIdx.x == 0) counters[(sweep + 1) % 3] = 0;
    for (int round = 0; round < max_rounds; ++round) {
      for (int t = gw; t < total_pairs; t += TW) {
        int pi = 0;
        while (pi + 1 < nprob && t >= probs[pi + 1].pair_base) ++pi;
        const JUProb& P = probs[pi];
        const int np = P.n + (P.n & 1);
        if (round >= np - 1) continue;
        const int pr = t - P.pair_base;
        int p = rr_idx(pr, round, np), qd = rr_idx(np - 1 - pr, round, np);
        if (p >= P.n || qd >= P.n) continue;
        if (p > qd) { int tt = p; p = qd; qd = tt; }
        double* up = P.X + (size_t)p * P.m;
        double* uq = P.X + (size_t)qd * P.m;
        const int m = P.m;
        const double tol = DBL_EPSILON * (double)max(m, 2);
        if (REG) {
          double x[JR], y[JR];
          double al = 0, be = 0, ga = 0;
#pragma unroll
          for (int k = 0; k < JR; ++k) {
            int i = lane + 32 * k;
            x[k] = i < m ? up[i] : 0.0;
            y[k] = i < m ? uq[i] : 0.0;
            al += x[k] * x[k];
            be += y[k] * y[k];
            ga += x[k] * y[k];
          }
          al = wsum(al);
          be = wsum(be);
          ga = wsum(ga);
          if (!(al >= DBL_MIN && be >= DBL_MIN) || ga == 0.0 || !(fabs(ga) > tol * sqrt(al) * sqrt(be))) continue;
          double zeta = (be - al) / (2.0 * ga);
          double tt = copysign(1.0, zeta) / (fabs(zeta) + hypot(1.0, zeta));
          double c = 1.0 / sqrt(1.0 + tt * tt), sn = c * tt;
#pragma unroll
          for (int k = 0; k < JR; ++k) {
            int i = lane + 32 * k;
            if (i < m) {
              up[i] = c * x[k] - sn * y[k];
              uq[i] = sn * x[k] + c * y[k];
            }
          }
        } else {
          double al = 0, be = 0, ga = 0;
          for (int i = lane; i < m; i += 32) {
            double a = up[i], b = uq[i];
            al += a * a;
            be += b * b;
            ga += a * b;
          }
          al = wsum(al);
          be = wsum(be);
          ga = wsum(ga);
          if (!(al >= DBL_MIN && be >= DBL_MIN) || ga == 0.0 || !(fabs(ga) > tol * sqrt(al) * sqrt(be))) continue;
          double zeta = (be - al) / (2.0 * ga);
          double tt = copysign(1.0, zeta) / (fabs(zeta) + hypot(1.0, zeta));
          double c = 1.0 / sqrt(1.0 + tt * tt), sn = c * tt;
          for (int i = lane; i < m; i += 32) {
            double a = up[i], b = uq[i];
            up[i] = c * a - sn * b;
            uq[i] = sn * a + c * b;
          }
        }
        if (lane == 0) atomicAdd(cnt, 1);
      }
      grid_barrier(bar, flag);
    }
    int rot = *(volatile int*)cnt;
    if (rot == 0) {
      converged = true;
      break;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    if (!converged) atomicOr(flag, FLAG_CONV);
    atomicMax(flag + 1, sweep + 1);
  }
  for (int pi = 0; pi < nprob; ++pi) {
    const JUProb P = probs[pi];
    for (int c = gw; c < P.n; c += TW) {
      const double* uc = P.X + (size_t)c * P.m;
      double v = 0;
      for (int i = lane; i < P.m; i += 32) v += uc[i] * uc[i];
      v = wsum(v);
      if (lane == 0) P.sig[c] = sqrt(v);
    }
  }
  grid_barrier(bar, flag);
  for (int pi = 0; pi < nprob; ++pi) {
    const JUProb P = probs[pi];
    for (int c = blockIdx.x * BT + threadIdx.x; c < P.n; c += gridDim.x * BT) {
      double sc = __ldcg(&P.sig[c]);
      int rk = 0;
      for (int j = 0; j < P.n; ++j) {
        double sj = __ldcg(&P.sig[j]);
        rk += (sj > sc) || (sj == sc && j < c);
      }
      P.rank[c] = rk;
      P.s[rk] = sc;
    }
  }
  grid_barrier(bar, flag);
  for (int pi = 0; pi < nprob; ++pi) {
    const JUProb P = probs[pi];
    for (int c = gw; c < P.n; c += TW) {
      int rk = __ldcg(&P.rank[c]);
      double sc = __ldcg(&P.sig[c]);
      double inv = sc > 0 ? 1.0 / sc : 0.0;
      const double* uc = P.X + (size_t)c * P.m;
      double* qo = P.q + (size_t)rk * P.m;
      for (int i = lane; i < P.m; i += 32) qo[i] = uc[i] * inv;
    }
  }
}

// ---------------------------------------------------------------------------
// U-only block one-sided Jacobi: blocks of UBW columns; each round one CTA
// takes a block pair (2*UBW columns) into shared memory, runs one inner
// one-sided Jacobi sweep over its column pairs (shared-memory rounds, no grid
// barrier) and writes the pair back.  nblk-1 grid barriers per sweep.
// ---------------------------------------------------------------------------
static constexpr int UBW = 4;
static constexpr int UB2 = 2 * UBW;

__global__ void __launch_bounds__(BT) jacobi_ub_kernel(const JUProb* probs, int nprob, int total_pairs,
                                                       int max_rounds, unsigned* bar, int* counters, int* flag) {
  extern __shared__ double Ub[];   // m x UB2, column-major (ld m)
  __shared__ int any_rot;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    counters[0] = 0;
    counters[1] = 0;
    counters[2] = 0;
  }
  grid_barrier(bar, flag);
  const int MAXSWEEP = 80;
  bool converged = false;
  int sweep = 0;
  for (; sweep < MAXSWEEP; ++sweep) {
    int* cnt = counters + (sweep % 3);
    if (blockIdx.x == 0 && threadIdx.x == 0) counters[(sweep + 1) % 3] = 0;
    for (int round = 0; round < max_rounds; ++round) {
      for (int t = blockIdx.x; t < total_pairs; t += gridDim.x) {
        int pi = 0;
        while (pi + 1 < nprob && t >= probs[pi + 1].pair_base) ++pi;
        const JUProb& P = probs[pi];
        const int nb = (P.n + UBW - 1) / UBW;
        const int nbp = nb + (nb & 1);
        if (round >= nbp - 1) continue;
        const int pr = t - P.pair_base;
        int bi = rr_idx(pr, round, nbp), bj = rr_idx(nbp - 1 - pr, round, nbp);
        if (bi >= nb || bj >= nb) continue;
        if (bi > bj) { int tt = bi; bi = bj; bj = tt; }
        const int c0 = bi * UBW, w1 = min(UBW, P.n - c0);
        const int c1 = bj * UBW, w2 = min(UBW, P.n - c1);
        const int wt = w1 + w2, m = P.m;
        for (int e = threadIdx.x; e < wt * m; e += BT) {
          int k = e / m, i = e % m;
          int gc = k < w1 ? c0 + k : c1 + (k - w1);
          Ub[i + (size_t)k * m] = P.X[i + (size_t)gc * m];
        }
        if (threadIdx.x == 0) any_rot = 0;
        __syncthreads();
        const double tol = DBL_EPSILON * (double)max(m, 2);
        const int wtp = wt + (wt & 1);
        for (int ir = 0; ir < wtp - 1; ++ir) {
          for (int q = warp; q < wtp / 2; q += BW) {
            int a = rr_idx(q, ir, wtp), b = rr_idx(wtp - 1 - q, ir, wtp);
            if (a >= wt || b >= wt) continue;
            if (a > b) { int tt = a; a = b; b = tt; }
            double* ua = Ub + (size_t)a * m;
            double* ub = Ub + (size_t)b * m;
            double al = 0, be = 0, ga = 0;
            for (int i = lane; i < m; i += 32) {
              double x = ua[i], y = ub[i];
              al += x * x;
              be += y * y;
              ga += x * y;
            }
            al = wsum(al);
            be = wsum(be);
            ga = wsum(ga);
            if (!(al >= DBL_MIN && be >= DBL_MIN) || ga == 0.0 || !(fabs(ga) > tol * sqrt(al) * sqrt(be))) continue;
            double zeta = (be - al) / (2.0 * ga);
            double tt = copysign(1.0, zeta) / (fabs(zeta) + hypot(1.0, zeta));
            double c = 1.0 / sqrt(1.0 + tt * tt), sn = c * tt;
            for (int i = lane; i < m; i += 32) {
              double x = ua[i], y = ub[i];
              ua[i] = c * x - sn * y;
              ub[i] = sn * x + c * y;
            }
            if (lane == 0) any_rot = 1;
          }
          __syncthreads();
        }
        if (any_rot) {
          if (threadIdx.x == 0) atomicAdd(cnt, 1);
          for (int e = threadIdx.x; e < wt * m; e += BT) {
            int k = e / m, i = e % m;
            int gc = k < w1 ? c0 + k : c1 + (k - w1);
            P.X[i + (size_t)gc * m] = Ub[i + (size_t)k * m];
          }
        }
        __syncthreads();
      }
      grid_barrier(bar, flag);
    }
    int rot = *(volatile int*)cnt;
    if (rot == 0) {
      converged = true;
      break;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    if (!converged) atomicOr(flag, FLAG_CONV);
    atomicMax(flag + 1, sweep + 1);
  }
  const int gw = blockIdx.x * BW + warp, TW = gridDim.x * BW;
  for (int pi = 0; pi < nprob; ++pi) {
    const JUProb P = probs[pi];
    for (int c = gw; c < P.n; c += TW) {
      const double* uc = P.X + (size_t)c * P.m;
      double v = 0;
      for (int i = lane; i < P.m; i += 32) v += uc[i] * uc[i];
      v = wsum(v);
      if (lane == 0) P.sig[c] = sqrt(v);
    }
  }
  grid_barrier(bar, flag);
  for (int pi = 0; pi < nprob; ++pi) {
    const JUProb P = probs[pi];
    for (int c = blockIdx.x * BT + threadIdx.x; c < P.n; c += gridDim.x * BT) {
      double sc = __ldcg(&P.sig[c]);
      int rk = 0;
      for (int j = 0; j < P.n; ++j) {
        double sj = __ldcg(&P.sig[j]);
        rk += (sj > sc) || (sj == sc && j < c);
      }
      P.rank[c] = rk;
      P.s[rk] = sc;
    }
  }
  grid_barrier(bar, flag);
  for (int pi = 0; pi < nprob; ++pi) {
    const JUProb P = probs[pi];
    for (int c = gw; c < P.n; c += TW) {
      int rk = __ldcg(&P.rank[c]);
      double sc = __ldcg(&P.sig[c]);
      double inv = sc > 0 ? 1.0 / sc : 0.0;
      const double* uc = P.X + (size_t)c * P.m;
      double* qo = P.q + (size_t)rk * P.m;
      for (int i = lane; i < P.m; i += 32) qo[i] = uc[i] * inv;
    }
  }
}

// problems: (x = m x n ld m rotated in place, q = sorted left vectors m x n ld m, s = values n)
void jacobi_left(Engine& E, const std::vector<MatDesc>& d) {
  if (d.empty()) return;
  std::vector<JUProb> ps;
  int pairs = 0, max_rounds = 0, mmax = 0;
  size_t ws = 0;
  for (auto& x : d) ws += 2 * (size_t)x.n + 8;
  Buf wb = E.alloc(sizeof(double) * ws);
  double* w = (double*)wb->ptr;
  for (auto& x : d) {
    JUProb P;
    P.X = x.a;
    P.q = x.q;
    P.s = x.s;
    P.m = x.m;
    P.n = x.n;
    P.sig = w;
    w += x.n;
    P.rank = (int*)w;
    w += x.n + 8;
    P.pair_base = pairs;
    int np = x.n + (x.n & 1);
    pairs += np / 2;
    max_rounds = std::max(max_rounds, np - 1);
    mmax = std::max(mmax, x.m);
    ps.push_back(P);
  }
  Buf pb = E.alloc(sizeof(JUProb) * ps.size());
  E.stage(ps.data(), sizeof(JUProb) * ps.size(), pb->ptr);
  Buf bb = E.alloc(sizeof(unsigned) * 2 + sizeof(int) * 4);
  SPS_CUDA(cudaMemsetAsync(bb->ptr, 0, sizeof(unsigned) * 2 + sizeof(int) * 4, E.stream));
  size_t ubsmem = sizeof(double) * (size_t)mmax * UB2;
  const bool blocked = ubsmem <= 200 * 1024;
  if (blocked) {
    int bpairs = 0, brounds = 0;
    for (auto& P : ps) {
      int nb = (P.n + UBW - 1) / UBW;
      int nbp = nb + (nb & 1);
      P.pair_base = bpairs;
      bpairs += nbp / 2;
      brounds = std::max(brounds, nbp - 1);
    }
    pairs = bpairs;
    max_rounds = brounds;
    E.stage(ps.data(), sizeof(JUProb) * ps.size(), pb->ptr);
  }
  const bool reg = mmax <= 32 * JR;
  const void* kfn = blocked ? (const void*)jacobi_ub_kernel
                            : (reg ? (const void*)jacobi_u_kernel<true> : (const void*)jacobi_u_kernel<false>);
  size_t smem = blocked ? ubsmem : 0;
  if (blocked)
    allow_max_smem(kfn);
  int maxg = coop_blocks(kfn, BT, smem, E);
  int G = blocked ? std::min(maxg, std::max(1, pairs))
                  : std::min({E.num_sms, maxg, std::max(1, (pairs + BW - 1) / BW)});
  const JUProb* dp = (const JUProb*)pb->ptr;
  int nprob = (int)ps.size();
  unsigned* bar = (unsigned*)bb->ptr;
  int* counters = (int*)(bar + 2);
  void* args[] = {&dp, &nprob, &pairs, &max_rounds, &bar, &counters, &E.dflag};
  int tk = E.tic("svd_jacobi_left");
  SPS_CUDA(cudaLaunchCooperativeKernel(kfn, dim3(G), dim3(BT), args, smem, E.stream));
  E.toc(tk);
  E.launches++;
  if (E.profile) {
    // algorithmic work: per sweep every column pair costs 3 dot products and a rotation (6m flops)
    int sweeps = 0;
    SPS_CUDA(cudaMemcpyAsync(&sweeps, E.dflag + 1, sizeof(int), cudaMemcpyDeviceToHost, E.stream));
    E.sync();
    SPS_CUDA(cudaMemsetAsync(E.dflag + 1, 0, sizeof(int), E.stream));
    double fl = 0, by = 0;
    for (auto& x : d) {
      fl += 6.0 * x.m * 0.5 * x.n * (x.n - 1) * sweeps;
      by += 32.0 * x.m * 0.5 * x.n * (x.n - 1) * sweeps / 2;   // each round reads and writes every column once
    }
    E.set_work(tk, fl, by);
  }
}

__global__ void transpose_cm_kernel(const double* __restrict__ src, int m, int n, int lds, double* __restrict__ dst,
                                    int ldd) {
  size_t total = (size_t)m * n;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    int i = (int)(e % m), j = (int)(e / m);
    dst[j + (size_t)i * ldd] = src[i + (size_t)j * lds];
  }
}

// dst (n x m, ld ldd) = src^T, src (m x n, ld lds), both column-major
void transpose_cm(Engine& E, const double* src, int m, int n, int lds, double* dst, int ldd) {
  size_t total = (size_t)m * n;
  if (!total) return;
  int g = (int)std::min<size_t>((total + 255) / 256, 8192);
  transpose_cm_kernel<<<g, 256, 0, E.stream>>>(src, m, n, lds, dst, ldd);
  SPS_CUDA(cudaGetLastError());
  E.launches++;
}

// problems: (a = U in/out workspace m x n ld m, q out m x n ld m, r out n x n ld n, s out n)
void svd_big(Engine& E, const std::vector<MatDesc>& d) {
  if (d.empty()) return;
  std::vector<JacProb> ps;
  int pairs = 0, max_rounds = 0;
  size_t ws = 0;
  for (auto& x : d) ws += (size_t)x.n * x.n + 2 * (size_t)x.n + 8;
  Buf wb = E.alloc(sizeof(double) * ws);
  double* w = (double*)wb->ptr;
  for (auto& x : d) {
    if (x.lda != x.m || x.ldq != x.m || x.ldr != x.n) throw Error(SPS_ERR_ARGUMENT, "svd_big: leading dimensions");
    JacProb P;
    P.U = x.a;
    P.q = x.q;
    P.r = x.r;
    P.s = x.s;
    P.m = x.m;
    P.n = x.n;
    P.V = w;
    w += (size_t)x.n * x.n;
    P.sig = w;
    w += x.n;
    P.rank = (int*)w;
    w += x.n + 8;
    P.pair_base = pairs;
    int np = x.n + (x.n & 1);
    pairs += np / 2;
    max_rounds = std::max(max_rounds, np - 1);
    ps.push_back(P);
  }
  int mmax = 0;
  for (auto& x : d) mmax = std::max(mmax, x.m);
  size_t bsmem = sizeof(double) * ((size_t)BJ2 * BJ2 + (size_t)mmax * BJ2);
  const bool blocked = bsmem <= 200 * 1024;
  if (blocked) {
    int bpairs = 0, brounds = 0;
    for (auto& P : ps) {
      int nb = (P.n + BJW - 1) / BJW;
      int nbp = nb + (nb & 1);
      P.pair_base = bpairs;
      bpairs += nbp / 2;
      brounds = std::max(brounds, nbp - 1);
    }
    pairs = bpairs;
    max_rounds = brounds;
  }
  Buf pb = E.alloc(sizeof(JacProb) * ps.size());
  E.stage(ps.data(), sizeof(JacProb) * ps.size(), pb->ptr);
  Buf bb = E.alloc(sizeof(unsigned) * 2 + sizeof(int) * 6);
  SPS_CUDA(cudaMemsetAsync(bb->ptr, 0, sizeof(unsigned) * 2 + sizeof(int) * 6, E.stream));
  if (blocked) {
    allow_max_smem((const void*)bjacobi_kernel);
    const int per_sm = occupancy_per_sm((const void*)bjacobi_kernel, BT, bsmem);
    int G = std::min({E.coop_capacity(per_sm), std::max(1, pairs)});
    const JacProb* dp = (const JacProb*)pb->ptr;
    int nprob = (int)ps.size();
    unsigned* bar = (unsigned*)bb->ptr;
    int* counters = (int*)(bar + 2);
    int* sweeps = counters + 4;
    void* args[] = {&dp, &nprob, &pairs, &max_rounds, &bar, &counters, &E.dflag, &sweeps};
    int tk = E.tic("svd_block_jacobi");
    SPS_CUDA(cudaLaunchCooperativeKernel((const void*)bjacobi_kernel, dim3(G), dim3(BT), args, bsmem, E.stream));
    E.toc(tk);
    E.launches++;
    return;
  }
  int maxg = coop_blocks((const void*)jacobi_coop_kernel, BT, 0, E);
  int G = std::min({E.num_sms, maxg, std::max(1, (pairs + BW - 1) / BW)});
  const JacProb* dp = (const JacProb*)pb->ptr;
  int nprob = (int)ps.size();
  unsigned* bar = (unsigned*)bb->ptr;
  int* counters = (int*)(bar + 2);
  void* args[] = {&dp, &nprob, &pairs, &max_rounds, &bar, &counters, &E.dflag};
  int tk = E.tic("svd_jacobi_coop");
  SPS_CUDA(cudaLaunchCooperativeKernel((const void*)jacobi_coop_kernel, dim3(G), dim3(BT), args, 0, E.stream));
  E.toc(tk);
  E.launches++;
}

}  // namespace la
}  // namespace sps
