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
// one CTA, U = Q Ub, V = Qb J.  When a plain pass meets a non-positive pivot
// (trailing columns of the iterate at the rounding level, as a fast-decaying
// spectrum leaves them, most of all on M M^T) it is redone with the shift and
// followed by two deflating passes that zero those columns.  If fewer than k
// columns survive on M M^T, the launch stops with status 4 (the caller then
// iterates on M); on M the extraction goes on, and a converged extraction with
// zero values among the wanted ones reports status 4 (the caller completes
// their vectors).  The extraction is accepted when
// ||M v_i - s_i u_i|| is within the requested relative residual (rounding
// level unless the caller asks for less) for every wanted i; otherwise two
// more iterations and a new extraction, up to a cap, after which the caller
// uses the full SVD.  Everything is FP64.
#include "engine.h"
#include "coop.cuh"
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cfloat>
#include <algorithm>
#include <mutex>

namespace sps {
namespace la {

namespace {

constexpr int TT = 256;           // threads per CTA
constexpr int TW = TT / 32;       // warps per CTA
constexpr int KMAXB = 80;         // largest block size b
constexpr int RMAX = 96;          // largest number of rows owned by one CTA
constexpr int KC = 32;            // contraction chunk of the row GEMM
constexpr int NST = 2;            // stage budget of the row GEMM, in stages of the largest tile
constexpr int MAXST = 8;          // most stages (and stage barriers) of the row GEMM
constexpr int XLD = KC + 4;       // row stride of the staged operands: a fragment load is 2 wavefronts
constexpr int STAGE = (RMAX + KMAXB) * XLD;
constexpr int YLD = KMAXB + 1;
constexpr int GLD = KMAXB + 1;
constexpr int OFF_X = 0;
constexpr int STG_PAD = 128;      // the stages start at the first 1024-byte boundary of the arena
constexpr int OFF_Y = OFF_X + NST * STAGE + STG_PAD;
constexpr int OFF_G = OFF_Y + RMAX * YLD;
constexpr int OFF_V = OFF_G + KMAXB * GLD;
constexpr int OFF_R = OFF_V + 3 * KMAXB;
constexpr int SMEM_DOUBLES = OFF_R + 16 + KMAXB;
constexpr int JLD = KMAXB + 1;    // Jacobi arrays (CTA 0 only, overlays X..V)
constexpr int MAX_SWEEPS = 40;
static_assert(2 * KMAXB * JLD <= OFF_R, "Jacobi overlay exceeds the shared arena");
constexpr int MAXT = ((RMAX / 8) * (KMAXB / 8) + TW - 1) / TW;   // 8 x 8 output tiles per warp
static_assert(RMAX % 8 == 0 && KMAXB % 8 == 0 && KC % 4 == 0 && XLD % 2 == 0, "tiling");
static_assert(TT >= 256, "the 16 x 16 thread grid of the small factorizations needs 256 threads");
static_assert(KC == 32 && MAXT <= 15, "the row GEMM's chunk is 8 k-steps; its tile dispatch covers 15 tiles per warp");
static_assert(MAXT * TW * 64 <= NST * STAGE, "k-part partial sums exceed the staging area");
static_assert(2 * (RMAX / 8 + KMAXB / 8) * 128 <= STAGE, "a stage of the largest tile exceeds the budget");
static_assert(2 * (RMAX / 8 + KMAXB / 8) * 128 < 65536, "packed fragment offsets are 16-bit");

enum : int { ST_OK = 0, ST_BREAKDOWN = 1, ST_JACOBI = 2, ST_NOCONV = 3, ST_ZERO = 4 };

}  // namespace

struct TopkProb {
  // TMA maps of the row-GEMM operands (16 x rows boxes, 128-byte swizzle):
  // M (box Rn rows), M^T and M M^T (box Rm rows), Q and Z (box b), Vi (box k)
  CUtensorMap tM, tMt, tGm, tQ, tZ, tVi;
  const double* M;   // m x n, column-major, ld ldm (read-only in the kernel)
  const double* Mt;  // n x m, column-major, ld ldn (M transposed)
  int m, n, k, b, P, cta0;
  int ldm, ldn;      // m and n rounded up to even (16-byte row strides)
  int Rm, Rn;        // rows of the m- and n-sized iterates owned by one CTA (the last may own fewer)
  double* Q;     // m x b (ld ldm)
  double* Z;     // n x b (ld ldn): Omega, Z iterates, Qb
  double* Vi;    // n x k (ld ldn): right vectors
  const double* Gm;  // m x m (ld ldm): M M^T when iterating on the Gram matrix, else null
  double* Gp;    // P x KMAXB^2 Gram partials
  double* G;     // b x b
  double* Racc;  // b x b accumulated R of M^T Q (row-major)
  double* Ub;    // b x b left Ritz rotation (column-major)
  double* Jo;    // b x b right Ritz rotation (column-major)
  double* U;     // m x k out (ld m)
  double* s;     // b Ritz values, descending
  double* fpart; // P partial squared Frobenius norms
  double* info;  // [status, iterations, ||M||_F^2, max residual / threshold, done, Ritz Jacobi sweeps]
  unsigned* bar; // 2 words
};

namespace {

struct Ctx {
  const TopkProb* p;
  int c;            // CTA index inside the problem
  int rm0, rm1;     // rows of m-sized iterates owned here
  int rn0, rn1;     // rows of n-sized iterates owned here
  double* sm;
  double* stg;                 // the row GEMM's stages: 1024-byte aligned, NST * STAGE doubles
  int* flag;
  unsigned long long* trace;   // profile mode: [count, (phase, clock) ...], CTA 0 only
  unsigned* trace_n;           // its count (shared memory)
  unsigned long long* mbar;    // MAXST stage barriers (shared memory)
  unsigned phase;              // bit s: parity of stage barrier s's next completion
};

// phases of the profile-mode trace (interval ending at the record)
enum : int { PH_START = 0, PH_INIT, PH_GEMM, PH_GRAM, PH_REDUCE, PH_CHOL, PH_APPLY, PH_STORE, PH_JACOBI, PH_ROTATE,
             PH_RESID, PH_GISSUE, PH_GWAIT, PH_GMMA, PH_COUNT };
constexpr int TRACE_CAP = 2048;

__device__ __forceinline__ void trace_mark(const Ctx& x, int phase) {
  if (x.trace && x.c == 0 && threadIdx.x == 0) {
    const unsigned n = *x.trace_n;
    if (n < TRACE_CAP) {
      x.trace[1 + 2 * n] = phase;
      x.trace[2 + 2 * n] = clock64();
      x.trace[0] = n + 1;
      *x.trace_n = n + 1;
    }
  }
}

// every global write before a group barrier may be read by a bulk copy after it
__device__ __forceinline__ void sync_group(const Ctx& x) {
  asm volatile("fence.proxy.async.global;" ::: "memory");
  group_barrier(x.p->bar, (unsigned)x.p->P, x.flag);
}

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

// Stage barriers: one mbarrier per shared-memory stage, armed with the bytes
// its bulk copies deliver, completed by the copies themselves.
__device__ __forceinline__ void stage_expect(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}
// one 16 x rows box of a row-major view (x0: first element of the row, even;
// y0: first row); elements outside the matrix arrive as zeros
__device__ __forceinline__ void tma_load(double* dst, const CUtensorMap* map, int x0, int y0, unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          smem_addr(dst)),
      "l"(reinterpret_cast<unsigned long long>(map)), "r"(x0), "r"(y0), "r"(smem_addr(bar))
      : "memory");
}
__device__ __forceinline__ bool stage_try(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// bounded: after the cap the copy flag is raised and the data is not trusted
__device__ __forceinline__ void stage_wait(const Ctx& x, unsigned long long* bar, unsigned parity) {
  long long spins = 0;
  while (!stage_try(bar, parity))
    if (++spins > (1ll << 24)) {
      if (threadIdx.x == 0) atomicOr(x.flag, FLAG_COPY);
      break;
    }
}
// orders this thread's generic-proxy shared-memory accesses before later TMA
// writes to the same bytes (async proxy)
__device__ __forceinline__ void proxy_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// NQ output tiles of this warp over KSN k-steps of one staged chunk.  A
// staged operand row is 16 doubles (128 bytes) per half-chunk, its 16-byte
// pieces permuted by the 128-byte swizzle: piece u of row r sits at u ^ (r % 8).
// off[q] packs the fragment offsets of item q: X row in the low 16 bits, S
// row in the high 16 bits (doubles from the stage start).
template <int NQ, int KSN>
__device__ __forceinline__ void mma_chunk(double (&acc)[MAXT][2], const double* st, const unsigned (&off)[MAXT],
                                          const int (&cx)[4], int hx, int hs) {
#pragma unroll
  for (int ks = 0; ks < KSN; ++ks) {
    const int h = ks >> 2;
#pragma unroll
    for (int q = 0; q < NQ; ++q)
      dmma(acc[q][0], acc[q][1], st[(off[q] & 0xffffu) + h * hx + cx[ks & 3]],
           st[(off[q] >> 16) + h * hs + cx[ks & 3]]);
  }
}

// Ys[r][j] = sum_t X[r0 + r][t] * S[j][t]   (r < r1 - r0, j < bb, t < K), X
// and S row-major views given by their TMA maps (boxes of 16 x rbox and
// 16 x bb), on the FP64 tensor cores.  Chunks of 32 along t stream through as
// many shared-memory stages as fit (up to MAXST): lane 0 of warps 4-7 issues
// one box load each per chunk (two halves of X and of S), completing on the
// stage's mbarrier (warp 4 arms it with the chunk's byte count; a load that
// lands first leaves the count negative, and the phase cannot complete before
// that single arrival); rows and columns past the matrices arrive as zeros.  Work items
// are (8 x 8 output tile, half of the chunk's k-steps) when splitting the
// k-steps evens out the warps' tile counts; the halves are then added in a
// fixed order at the end.
__device__ __noinline__ void gemm_rows(Ctx& x, const CUtensorMap* tX, int rbox, const CUtensorMap* tS, int bb, int K,
                                       int r0, int r1) {
  double* Ys = x.sm + OFF_Y;
  const int R = r1 - r0;
  const int mt = (rbox + 7) / 8, nt = (bb + 7) / 8, ntiles = mt * nt;
  const int per1 = (ntiles + TW - 1) / TW, per2 = (2 * ntiles + TW - 1) / TW;
  const int parts = (per2 <= MAXT && per2 * 4 < per1 * 8) ? 2 : 1;
  const int items = ntiles * parts;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, fr = lane >> 2, fc = lane & 3;
  const int nq = warp < items ? (items - warp + TW - 1) / TW : 0;
  const int hx = mt * 128, hs = nt * 128;   // doubles of one half-chunk region of X and of S
  const int stage = 2 * (hx + hs);
  int cx[4];
#pragma unroll
  for (int u = 0; u < 4; ++u) cx[u] = ((((u << 1) | (fc >> 1)) ^ fr) << 1) | (fc & 1);
  double acc[MAXT][2];
  unsigned off[MAXT];
#pragma unroll
  for (int q = 0; q < MAXT; ++q) {
    acc[q][0] = acc[q][1] = 0.0;
    const int item = warp + q * TW;
    const int tile = item % ntiles, part = item / ntiles;
    const unsigned ao = q < nq ? part * hx + ((tile / nt) * 8 + fr) * 16 : 0;
    const unsigned bo = q < nq ? 2 * hx + part * hs + ((tile % nt) * 8 + fr) * 16 : 0;
    off[q] = ao | (bo << 16);
  }
  const int nst = max(2, min(MAXST, (NST * STAGE) / stage));
  const int nch = (K + KC - 1) / KC;
  const unsigned bytes = 2u * 128u * (unsigned)(rbox + bb);
  const int role = (lane == 0 && warp >= TW - 4) ? warp - (TW - 4) : -1;   // which of the four boxes
  auto issue = [&](int c) {
    double* st = x.stg + (c % nst) * stage;
    unsigned long long* bar = x.mbar + (c % nst);
    const int t0 = c * KC;
    if (role == 0) {
      stage_expect(bar, bytes);
      tma_load(st, tX, t0, r0, bar);
    } else if (role == 1) {
      tma_load(st + hx, tX, t0 + 16, r0, bar);
    } else if (role == 2) {
      tma_load(st + 2 * hx, tS, t0, 0, bar);
    } else {
      tma_load(st + 2 * hx + hs, tS, t0 + 16, 0, bar);
    }
  };
  proxy_fence();
  __syncthreads();   // the stages may still be read by the previous phase
  if (role >= 0)
    for (int c = 0; c < nst - 1 && c < nch; ++c) issue(c);
  trace_mark(x, PH_GISSUE);
  for (int c = 0; c < nch; ++c) {
    stage_wait(x, x.mbar + (c % nst), (x.phase >> (c % nst)) & 1u);
    x.phase ^= 1u << (c % nst);
    __syncthreads();   // every warp is done with chunk c - 1: its stage is free
    trace_mark(x, PH_GWAIT);
    if (role >= 0 && c + nst - 1 < nch) issue(c + nst - 1);
    const double* st = x.stg + (c % nst) * stage;
    if (parts == 1) {
      switch (nq) {
#define SPS_TOPK_MMA(N) \
  case N:               \
    mma_chunk<N, 8>(acc, st, off, cx, hx, hs); \
    break;
        SPS_TOPK_MMA(1) SPS_TOPK_MMA(2) SPS_TOPK_MMA(3) SPS_TOPK_MMA(4) SPS_TOPK_MMA(5)
        SPS_TOPK_MMA(6) SPS_TOPK_MMA(7) SPS_TOPK_MMA(8) SPS_TOPK_MMA(9) SPS_TOPK_MMA(10)
        SPS_TOPK_MMA(11) SPS_TOPK_MMA(12) SPS_TOPK_MMA(13) SPS_TOPK_MMA(14) SPS_TOPK_MMA(15)
#undef SPS_TOPK_MMA
        default:
          break;
      }
    } else {
      switch (nq) {
#define SPS_TOPK_MMA(N) \
  case N:               \
    mma_chunk<N, 4>(acc, st, off, cx, hx, hs); \
    break;
        SPS_TOPK_MMA(1) SPS_TOPK_MMA(2) SPS_TOPK_MMA(3) SPS_TOPK_MMA(4) SPS_TOPK_MMA(5)
        SPS_TOPK_MMA(6) SPS_TOPK_MMA(7) SPS_TOPK_MMA(8) SPS_TOPK_MMA(9) SPS_TOPK_MMA(10)
        SPS_TOPK_MMA(11) SPS_TOPK_MMA(12) SPS_TOPK_MMA(13) SPS_TOPK_MMA(14) SPS_TOPK_MMA(15)
#undef SPS_TOPK_MMA
        default:
          break;
      }
    }
    trace_mark(x, PH_GMMA);
  }
  __syncthreads();   // the stages are free: partial sums of the halves go there
  // accumulator fragment: row fr, columns 2 fc + {0, 1} of the tile
  if (parts == 1) {
#pragma unroll
    for (int q = 0; q < MAXT; ++q) {
      if (q >= nq) break;
      const int tile = warp + q * TW;
      const int r = (tile / nt) * 8 + fr, j = (tile % nt) * 8 + 2 * fc;
      if (r < R) {
        if (j < bb) Ys[r * YLD + j] = acc[q][0];
        if (j + 1 < bb) Ys[r * YLD + j + 1] = acc[q][1];
      }
    }
  } else {
    double* part = x.stg;   // [item][64]
#pragma unroll
    for (int q = 0; q < MAXT; ++q) {
      if (q >= nq) break;
      const int item = warp + q * TW;
      part[item * 64 + fr * 8 + 2 * fc] = acc[q][0];
      part[item * 64 + fr * 8 + 2 * fc + 1] = acc[q][1];
    }
    __syncthreads();
    for (int e = threadIdx.x; e < ntiles * 64; e += TT) {
      const int tile = e >> 6, w = e & 63;
      const int r = (tile / nt) * 8 + (w >> 3), j = (tile % nt) * 8 + (w & 7);
      const double v = part[tile * 64 + w] + part[(ntiles + tile) * 64 + w];
      if (r < R && j < bb) Ys[r * YLD + j] = v;
    }
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
// mode OP_SHIFT: shifted Cholesky QR (never meets a non-positive pivot);
// OP_PLAIN: plain Cholesky QR, redone with the shift when a pivot is not
// positive (the iterate's trailing columns fell to the rounding level of G);
// OP_DEFLATE: plain, dropping every column whose pivot is at the rounding
// level of G (a zero column of the result, a zero row of R).
// Returns -1 on breakdown, else bit 0 = redone with the shift (plain) or a
// column left short of unit norm (shifted), bits 1.. = the number of dropped
// columns; the value is the same in every CTA of the group (each factors the
// same reduced G).
enum : int { OP_SHIFT = 0, OP_PLAIN = 1, OP_DEFLATE = 2 };
__device__ __noinline__ int orth_pass(const Ctx& x, int bb, int r0, int r1, int nrows, int mode, int racc) {
  const TopkProb& p = *x.p;
  double* Ys = x.sm + OFF_Y;
  double* Gs = x.sm + OFF_G;
  double* sq = x.sm + OFF_V;              // sqrt of the pivots
  double* invd = sq + KMAXB;              // 1 / pivots
  double* defl = sq + 2 * KMAXB;          // 1: column dropped
  const int R = r1 - r0;
  // partial Gram of the owned rows (upper triangle)
  double* gp = p.Gp + (size_t)x.c * KMAXB * KMAXB;
  const int ty = threadIdx.x >> 4, tx = threadIdx.x & 15;   // 16 x 16 thread grid
  for (int i = ty; i < bb; i += 16)
    for (int j = i + tx; j < bb; j += 16) {
      double v = 0.0;
      for (int r = 0; r < R; ++r) v = fma(Ys[r * YLD + i], Ys[r * YLD + j], v);
      gp[i * bb + j] = v;
    }
  sync_group(x);
  trace_mark(x, PH_GRAM);
  // reduce this CTA's slice of entries over the partials: thread groups take
  // interleaved partials, then the groups are summed in order (deterministic)
  {
    const int total = bb * bb;
    const int slice = (total + p.P - 1) / p.P;
    const int e0 = min(total, x.c * slice), e1 = min(total, e0 + slice);
    double* red2 = x.sm + OFF_X;   // TT doubles (the GEMM staging area is free here)
    for (int base = e0; base < e1; base += TT) {
      const int ns = min(TT, e1 - base), ng = TT / ns;
      const int el = threadIdx.x % ns, q0 = threadIdx.x / ns;
      if (q0 < ng) {
        double v = 0.0;
        for (int q = q0; q < p.P; q += ng) v += __ldcg(&p.Gp[(size_t)q * KMAXB * KMAXB + base + el]);
        red2[q0 * ns + el] = v;
      }
      __syncthreads();
      if (threadIdx.x < ns) {
        double v = 0.0;
        for (int q = 0; q < ng; ++q) v += red2[q * ns + threadIdx.x];
        const int e = base + threadIdx.x, i = e / bb, j = e - i * bb;
        if (j >= i) p.G[e] = v;
      }
      __syncthreads();
    }
  }
  sync_group(x);
  trace_mark(x, PH_REDUCE);
  // factor G (+ shift) redundantly: G = U^T D U with U unit upper, kept as the
  // unscaled upper rows D U in Gs
  int retried = 0;
  for (int attempt = 0; attempt < 2; ++attempt) {
    __syncthreads();
    for (int i = ty; i < bb; i += 16)
      for (int j = i + tx; j < bb; j += 16) Gs[i * GLD + j] = __ldcg(&p.G[i * bb + j]);
    for (int j = threadIdx.x; j < bb; j += TT) defl[j] = 0.0;
    __syncthreads();
    // the rounding level of G's pivots: a deflating pass drops the columns at
    // or below it, a plain pass is redone with the shift when it meets one
    const bool deflating = mode == OP_DEFLATE, plain = mode == OP_PLAIN && attempt == 0;
    double delta = 0.0;
    if (deflating || plain) {
      double mx = 0.0;
      for (int i = 0; i < bb; ++i) mx = fmax(mx, Gs[i * GLD + i]);
      delta = 32.0 * bb * DBL_EPSILON * mx;
    } else {
      if (threadIdx.x < 32) {   // trace by one warp, then the shift of shifted Cholesky QR on the diagonal
        double tr = 0.0;
        for (int i = threadIdx.x; i < bb; i += 32) tr += Gs[i * GLD + i];
        tr = wsum(tr);
        const double sh = 11.0 * ((double)nrows * bb + (double)bb * (bb + 1)) * DBL_EPSILON * tr;
        __syncwarp();
        for (int i = threadIdx.x; i < bb; i += 32) Gs[i * GLD + i] += sh;
      }
    }
    bool ok = true;
    for (int j = 0; j < bb; ++j) {
      __syncthreads();
      const double d = Gs[j * GLD + j];
      if (deflating && d <= delta) {   // dropped: no elimination by row j
        if (threadIdx.x == 0) defl[j] = 1.0;
        continue;
      }
      if (!(d > (plain ? delta : 0.0)) || !isfinite(d)) {
        ok = false;
        break;
      }
      const double inv = 1.0 / d;
      const double* gj = Gs + j * GLD;
      for (int i = j + 1 + ty; i < bb; i += 16) {
        const double gji = gj[i] * inv;
        for (int l = i + tx; l < bb; l += 16) Gs[i * GLD + l] -= gji * gj[l];
      }
    }
    if (ok) break;
    if (mode != OP_PLAIN || attempt == 1) {
      if (x.c == 0 && threadIdx.x == 0) p.info[0] = ST_BREAKDOWN;
      return -1;
    }
    retried = 1;
  }
  __syncthreads();
  int dropped = 0;
  for (int j = 0; j < bb; ++j) dropped += defl[j] != 0.0;
  // a shifted pass whose pivot stayed below twice the shift left that column
  // short of unit norm (its part of the iterate was below the shift's scale)
  int under = 0;
  if (mode == OP_SHIFT) {
    double tr = 0.0;
    for (int i = 0; i < bb; ++i) tr += __ldcg(&p.G[i * bb + i]);
    const double sh2 = 22.0 * ((double)nrows * bb + (double)bb * (bb + 1)) * DBL_EPSILON * tr;
    for (int j = 0; j < bb; ++j) under |= Gs[j * GLD + j] < sh2;
  }
  for (int j = threadIdx.x; j < bb; j += TT) {
    const bool dj = defl[j] != 0.0;
    sq[j] = dj ? 0.0 : sqrt(Gs[j * GLD + j]);
    invd[j] = dj ? 0.0 : 1.0 / Gs[j * GLD + j];
  }
  __syncthreads();
  // unit upper U in place (diagonal kept as the pivot)
  for (int i = ty; i < bb; i += 16)
    for (int j = i + 1 + tx; j < bb; j += 16) Gs[i * GLD + j] *= invd[i];
  __syncthreads();
  if (racc && x.c == 0) {
    // R = diag(sq) U;  Racc <- R (racc 1) or R Racc (racc 2), via CTA 0's partial slot;
    // the previous Racc is staged in shared memory (the GEMM stages are free here)
    double* tmp = gp;
    double* old = x.sm + OFF_X;
    if (racc == 2) {
      for (int e = threadIdx.x; e < bb * bb; e += TT) old[e] = __ldcg(&p.Racc[e]);
      __syncthreads();
    }
    for (int e = threadIdx.x; e < bb * bb; e += TT) {
      const int i = e / bb, j = e - i * bb;
      double v = 0.0;
      if (j >= i) {
        if (racc == 1) {
          v = (i == j) ? sq[i] : sq[i] * Gs[i * GLD + j];
        } else {
          for (int l = i; l <= j; ++l) {
            const double ril = (l == i) ? sq[i] : sq[i] * Gs[i * GLD + l];
            v = fma(ril, old[l * bb + j], v);
          }
        }
      }
      tmp[e] = v;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < bb * bb; e += TT) p.Racc[e] = tmp[e];
  }
  trace_mark(x, PH_CHOL);
  // rows: y <- y R^{-1}, R = diag(sq) U: forward substitution on the unit
  // upper factor, one column per step, then the diagonal scaling
  for (int j = 0; j < bb - 1; ++j) {
    for (int r = ty; r < R; r += 16) {
      const double yj = Ys[r * YLD + j];
      for (int l = j + 1 + tx; l < bb; l += 16) Ys[r * YLD + l] -= yj * Gs[j * GLD + l];
    }
    __syncthreads();
  }
  for (int r = ty; r < R; r += 16)
    for (int j = tx; j < bb; j += 16) Ys[r * YLD + j] = sq[j] > 0.0 ? Ys[r * YLD + j] / sq[j] : 0.0;
  __syncthreads();
  trace_mark(x, PH_APPLY);
  return retried | under | (dropped << 1);
}

// The orthonormalisation of an iteration step: a shifted pass, repeated once
// when it left a column short of unit norm (without the repeat, a column whose
// singular value is below the shift's scale, about 5e-5 of the largest, shrinks
// by that factor at every step until it reaches the rounding level).
__device__ __forceinline__ int orth_iter(const Ctx& x, int bb, int r0, int r1, int nrows) {
  const int f = orth_pass(x, bb, r0, r1, nrows, OP_SHIFT, 0);
  if (f < 0 || !(f & 1)) return f;
  return orth_pass(x, bb, r0, r1, nrows, OP_SHIFT, 0);
}

// One-sided Jacobi SVD of A = Racc^T (bb x bb) in CTA 0; sorted outputs to
// p.s, p.Ub (left vectors), p.Jo (right vectors).
__device__ __noinline__ void ritz_small(const Ctx& x, int bb) {
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
  const double tol_rot = DBL_EPSILON * bb;   // stop rotating pairs orthogonal to rounding level
  int sweep = 0;
  for (; sweep < MAX_SWEEPS; ++sweep) {
    if (threadIdx.x == 0) *cnt = 0;
    for (int round = 0; round < bb - 1; ++round) {
      __syncthreads();
      // 8 threads per column pair: 32 pairs at a time
      const int grp = threadIdx.x >> 3, sub = threadIdx.x & 7;
      // every lane runs the same number of passes so that the shuffles are convergent
      for (int base = 0; base < bb / 2; base += TT / 8) {
        const int pi = base + grp;
        const bool active = pi < bb / 2;
        int pp = 0, qq = 1;
        if (!active) {
        } else if (pi == 0) {
          pp = round;
          qq = bb - 1;
        } else {
          pp = (round + pi) % (bb - 1);
          qq = (round - pi + bb - 1) % (bb - 1);
        }
        double* ap = A + pp * JLD;
        double* aq = A + qq * JLD;
        double al = 0.0, be = 0.0, ga = 0.0;
        for (int r = sub; active && r < bb; r += 8) {
          const double u = ap[r], v = aq[r];
          al = fma(u, u, al);
          be = fma(v, v, be);
          ga = fma(u, v, ga);
        }
#pragma unroll
        for (int o = 4; o > 0; o >>= 1) {
          al += __shfl_xor_sync(0xffffffffu, al, o);
          be += __shfl_xor_sync(0xffffffffu, be, o);
          ga += __shfl_xor_sync(0xffffffffu, ga, o);
        }
        if (active && al >= DBL_MIN && be >= DBL_MIN && ga != 0.0 && fabs(ga) > tol_rot * sqrt(al) * sqrt(be)) {
          const double zeta = (be - al) / (2.0 * ga);
          const double t = copysign(1.0, zeta) / (fabs(zeta) + hypot(1.0, zeta));
          const double cs = 1.0 / sqrt(1.0 + t * t), sn = cs * t;
          double* jp = J + pp * JLD;
          double* jq = J + qq * JLD;
          for (int r = sub; r < bb; r += 8) {
            const double u = ap[r], v = aq[r];
            ap[r] = cs * u - sn * v;
            aq[r] = sn * u + cs * v;
            const double ju = jp[r], jv = jq[r];
            jp[r] = cs * ju - sn * jv;
            jq[r] = sn * ju + cs * jv;
          }
          if (sub == 0) atomicAdd(cnt, 1);
        }
      }
    }
    __syncthreads();
    const int rotations = *cnt;
    __syncthreads();
    if (rotations == 0) break;
  }
  if (threadIdx.x == 0) p.info[5] += sweep + 1;
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

__global__ void __launch_bounds__(TT, 1) topk_kernel(const TopkProb* __restrict__ probs, int nprob, int q0, int qstep,
                                                  int qmax, double tol, int* flag, unsigned long long* trace) {
  extern __shared__ __align__(128) double sm[];
  __shared__ unsigned long long stage_bar[MAXST];
  __shared__ unsigned trace_count;
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
  x.trace = (pi == 0) ? trace : nullptr;
  x.mbar = stage_bar;
  x.phase = 0;
  x.trace_n = &trace_count;
  x.stg = sm + ((1024u - (smem_addr(sm) & 1023u)) & 1023u) / sizeof(double);
  if (threadIdx.x == 0) {
    // the maps were written through the generic proxy (a host copy into
    // pooled memory that earlier launches may have used for other maps)
    // (the Gram map exists only when iterating on M M^T)
    const CUtensorMap* maps[6] = {&p.tM, &p.tMt, &p.tQ, &p.tZ, &p.tVi, &p.tGm};
    for (int i = 0; i < (p.Gm ? 6 : 5); ++i) {
      asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(maps[i]) : "memory");
      asm volatile("prefetch.tensormap [%0];" ::"l"(maps[i]) : "memory");
    }
    trace_count = 0;
    for (int st = 0; st < MAXST; ++st)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(stage_bar + st)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  trace_mark(x, PH_START);
  x.rm0 = min(p.m, x.c * p.Rm);
  x.rm1 = min(p.m, x.rm0 + p.Rm);
  x.rn0 = min(p.n, x.c * p.Rn);
  x.rn1 = min(p.n, x.rn0 + p.Rn);
  const int b = p.b, k = p.k;
  double* red = sm + OFF_R;

  // Omega into Z (owned n-rows) and the owned columns' share of ||M||_F^2
  {
    double f = 0.0;
    for (int e = threadIdx.x; e < (x.rn1 - x.rn0) * b; e += TT) {
      const int j = e / (x.rn1 - x.rn0), r = e - j * (x.rn1 - x.rn0);
      p.Z[(size_t)j * p.ldn + x.rn0 + r] = omega((unsigned long long)j * p.n + x.rn0 + r);
    }
    for (int col = x.rn0; col < x.rn1; ++col)
      for (int r = threadIdx.x; r < p.m; r += TT) {
        const double v = p.M[(size_t)col * p.ldm + r];
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
  trace_mark(x, PH_INIT);
  if (x.c == 0 && threadIdx.x == 0) {
    double s = 0.0;
    for (int q = 0; q < p.P; ++q) s += __ldcg(&p.fpart[q]);
    p.info[2] = s;
  }
  gemm_rows(x, &p.tMt, p.Rm, &p.tZ, b, p.n, x.rm0, x.rm1);
  trace_mark(x, PH_GEMM);
  if (orth_iter(x, b, x.rm0, x.rm1, p.m) < 0) return;
  store_rows(x, p.Q, p.ldm, b, x.rm0, x.rm1);
  sync_group(x);
  trace_mark(x, PH_STORE);

  int it = 0, target = q0;
  for (;;) {
    for (; it < target && p.Gm; ++it) {   // Gram iteration: Q = orth(M M^T Q)
      gemm_rows(x, &p.tGm, p.Rm, &p.tQ, b, p.m, x.rm0, x.rm1);
      trace_mark(x, PH_GEMM);
      if (orth_iter(x, b, x.rm0, x.rm1, p.m) < 0) return;
      store_rows(x, p.Q, p.ldm, b, x.rm0, x.rm1);
      sync_group(x);
      trace_mark(x, PH_STORE);
    }
    for (; it < target; ++it) {
      gemm_rows(x, &p.tM, p.Rn, &p.tQ, b, p.m, x.rn0, x.rn1);
      trace_mark(x, PH_GEMM);
      if (orth_iter(x, b, x.rn0, x.rn1, p.n) < 0) return;
      store_rows(x, p.Z, p.ldn, b, x.rn0, x.rn1);
      sync_group(x);
      trace_mark(x, PH_STORE);
      gemm_rows(x, &p.tMt, p.Rm, &p.tZ, b, p.n, x.rm0, x.rm1);
      trace_mark(x, PH_GEMM);
      if (orth_iter(x, b, x.rm0, x.rm1, p.m) < 0) return;
      store_rows(x, p.Q, p.ldm, b, x.rm0, x.rm1);
      sync_group(x);
      trace_mark(x, PH_STORE);
    }
    // Rayleigh-Ritz: Q <- orth(Q); M^T Q = Qb Rb; Rb^T = Ub S J^T
    // (a plain pass that had to be redone with the shift means columns at the
    // rounding level: two deflating passes then make Q orthonormal with those
    // columns zero; fewer than k columns left means the iteration lost wanted
    // directions, ST_ZERO)
    load_rows(x, p.Q, p.ldm, b, x.rm0, x.rm1);
    int fq = orth_pass(x, b, x.rm0, x.rm1, p.m, OP_PLAIN, 0);
    if (fq < 0) return;
    if (fq & 1)
      for (int pass = 0; pass < 2; ++pass)
        if ((fq = orth_pass(x, b, x.rm0, x.rm1, p.m, OP_DEFLATE, 0)) < 0) return;
    store_rows(x, p.Q, p.ldm, b, x.rm0, x.rm1);
    sync_group(x);
    trace_mark(x, PH_STORE);
    gemm_rows(x, &p.tM, p.Rn, &p.tQ, b, p.m, x.rn0, x.rn1);
    trace_mark(x, PH_GEMM);
    if (orth_pass(x, b, x.rn0, x.rn1, p.n, OP_SHIFT, 1) < 0) return;
    int fz = 0, redone = 0;
    for (int pass = 0; pass < 2; ++pass) {
      if ((fz = orth_pass(x, b, x.rn0, x.rn1, p.n, OP_PLAIN, 2)) < 0) return;
      redone |= fz & 1;
    }
    if (redone)
      for (int pass = 0; pass < 2; ++pass)
        if ((fz = orth_pass(x, b, x.rn0, x.rn1, p.n, OP_DEFLATE, 2)) < 0) return;
    if (p.Gm && (b - (fq >> 1) < k || b - (fz >> 1) < k)) {
      // on M M^T: wanted directions below its rounding level; the caller
      // iterates on M.  (On M, fewer than k surviving columns means fewer than
      // k singular values above the rounding level: the extraction goes on and
      // reports the missing ones as zero, status 4.)
      if (x.c == 0 && threadIdx.x == 0) {
        p.info[0] = ST_ZERO;
        p.info[1] = it;
      }
      return;
    }
    store_rows(x, p.Z, p.ldn, b, x.rn0, x.rn1);
    sync_group(x);
    trace_mark(x, PH_STORE);
    if (x.c == 0) ritz_small(x, b);
    sync_group(x);
    trace_mark(x, PH_JACOBI);
    if (__ldcg(&p.info[0]) != ST_OK) return;
    rotate_rows(x, p.Q, p.ldm, p.Ub, b, k, p.U, p.m, x.rm0, x.rm1);
    rotate_rows(x, p.Z, p.ldn, p.Jo, b, k, p.Vi, p.ldn, x.rn0, x.rn1);
    sync_group(x);
    trace_mark(x, PH_ROTATE);
    // residuals ||M v_i - s_i u_i||^2, partial over the owned m-rows
    gemm_rows(x, &p.tMt, p.Rm, &p.tVi, k, p.n, x.rm0, x.rm1);
    trace_mark(x, PH_GEMM);
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
    if (x.c == 0) {
      // squared residual of vector i summed over the partials, one thread per i
      double* res2 = sm + OFF_R + 16;
      for (int i = threadIdx.x; i < k; i += TT) {
        double v = 0.0;
        for (int q = 0; q < p.P; ++q) v += __ldcg(&p.Gp[(size_t)q * KMAXB * KMAXB + i]);
        res2[i] = v;
      }
      __syncthreads();
    }
    if (x.c == 0 && threadIdx.x == 0) {
      const double s0 = __ldcg(&p.s[0]);
      const double fro = sqrt(__ldcg(&p.info[2]));
      const double thr = fmax(tol * s0, 8.0 * DBL_EPSILON * sqrt((double)max(p.m, p.n)) * fro);
      const double* res2 = sm + OFF_R + 16;
      double worst = 0.0;
      bool zero = false;
      for (int i = 0; i < k; ++i) {
        worst = fmax(worst, thr > 0.0 ? sqrt(res2[i]) / thr : 0.0);
        zero |= !(__ldcg(&p.s[i]) > 0.0);
      }
      p.info[1] = it;
      p.info[3] = worst;
      int done = 0;
      if (worst <= 1.0) {
        done = 1;
        if (zero) p.info[0] = ST_ZERO;   // converged, with zero values among the wanted ones
      } else if (it + qstep > qmax) {
        p.info[0] = ST_NOCONV;
        done = 1;
      }
      p.info[4] = done;
    }
    sync_group(x);
    trace_mark(x, PH_RESID);
    if (__ldcg(&p.info[4]) != 0.0) return;
    target = it + qstep;
  }
}

// ---------------------------------------------------------------------------
// host driver
// ---------------------------------------------------------------------------

namespace {

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    SPS_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q));
    if (q != cudaDriverEntryPointSuccess || !f) throw Error(SPS_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
    fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
  });
  return fn;
}

// TMA map of a matrix seen as `rows` rows of `len` contiguous doubles, row
// stride ld (even); boxes of 16 x box_rows, 128-byte swizzle, zero fill
void encode_rows(CUtensorMap* map, const double* base, int len, int rows, int ld, int box_rows) {
  const cuuint64_t dims[2] = {(cuuint64_t)len, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)ld * sizeof(double)};
  const cuuint32_t box[2] = {16u, (cuuint32_t)box_rows};
  const cuuint32_t es[2] = {1u, 1u};
  const CUresult r = encode_fn()(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<double*>(base), dims, strides, box,
                                 es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                 CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) throw Error(SPS_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
}

}  // namespace

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
  return P * nprob <= E.num_sms;   // one CTA per SM; the whole GPU (see svd_topk)
}

void svd_topk(Engine& E, std::vector<TopkDesc>& ds, double tol) {
  if (ds.empty()) return;
  const size_t smem = sizeof(double) * SMEM_DOUBLES;
  set_max_dynamic_smem((const void*)topk_kernel, (int)smem);
  const int per_sm = occupancy_per_sm((const void*)topk_kernel, TT, smem);
  // the engine's share of the GPU is a target: a problem that needs more CTAs
  // than its share gets the minimum it needs (the cooperative launch then
  // waits for free SMs), up to the whole GPU
  const int capacity = E.coop_capacity(per_sm);
  const int capacity_full = std::max(1, per_sm) * E.num_sms;
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
    P = std::min(P, std::max(1, capacity / nprob));
    P = std::max(P, (mx + RMAX - 1) / RMAX);
    if (P * nprob > capacity_full || (mx + P - 1) / P > RMAX)
      throw Error(SPS_ERR_ARGUMENT, "svd_topk: block too large for the grid");
    const int b = d.b;
    const int ldm = m + (m & 1), ldn = n + (n & 1);
    // even leading dimensions: the TMA maps' row strides are multiples of 16
    // bytes and every buffer starts 16-byte aligned
    const size_t nd = (size_t)ldn * m + (size_t)ldm * b + (size_t)ldn * b + (size_t)ldn * d.k +
                      (d.gram ? (size_t)ldm * m : 0) +
                      ((m & 1) ? (size_t)ldm * n : 0) + (size_t)P * KMAXB * KMAXB + 4 * (size_t)b * b + b + P + 8;
    Buf w = E.alloc(sizeof(double) * nd + 64);
    keep.push_back(w);
    double* base = (double*)w->ptr;
    TopkProb& p = hp[i];
    double* mt = base;
    p.Mt = mt;
    base += (size_t)ldn * m;
    p.m = m;
    p.n = n;
    p.ldm = ldm;
    p.ldn = ldn;
    p.k = d.k;
    p.b = b;
    p.P = P;
    p.cta0 = cta;
    cta += P;
    p.Q = base;
    base += (size_t)ldm * b;
    p.Z = base;
    base += (size_t)ldn * b;
    // right vectors straight into the caller's buffer when its layout suits
    // the TMA maps (even n, 16-byte aligned), else via Vi
    if (ldn == n && reinterpret_cast<uintptr_t>(d.V) % 16 == 0) {
      p.Vi = d.V;
    } else {
      p.Vi = base;
    }
    base += (size_t)ldn * d.k;
    double* g = nullptr;
    if (d.gram) {
      g = base;
      base += (size_t)ldm * m;
    }
    p.Gm = g;
    if (m & 1) {   // odd leading dimension: an even-ld copy of M
      SPS_CUDA(cudaMemcpy2DAsync(base, sizeof(double) * ldm, d.M, sizeof(double) * m, sizeof(double) * m, n,
                                 cudaMemcpyDeviceToDevice, E.stream));
      p.M = base;
      base += (size_t)ldm * n;
    } else {
      if (reinterpret_cast<uintptr_t>(d.M) % 16) throw Error(SPS_ERR_ARGUMENT, "svd_topk: matrix not 16-byte aligned");
      p.M = d.M;
    }
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
    p.Rm = (m + P - 1) / P;
    p.Rn = (n + P - 1) / P;
    encode_rows(&p.tM, p.M, m, n, ldm, p.Rn);
    encode_rows(&p.tMt, p.Mt, n, m, ldn, p.Rm);
    if (g) encode_rows(&p.tGm, g, m, m, ldm, p.Rm);
    encode_rows(&p.tQ, p.Q, m, b, ldm, b);
    encode_rows(&p.tZ, p.Z, n, b, ldn, b);
    encode_rows(&p.tVi, p.Vi, n, d.k, ldn, d.k);
    SPS_CUDA(cudaMemsetAsync(p.info, 0, sizeof(double) * 6 + 8, E.stream));
    transpose_cm(E, d.M, m, n, m, mt, ldn);
    if (g) dgemm_cm(E, false, m, m, n, 1.0, p.M, ldm, mt, ldn, 0.0, g, ldm, true);   // G = M M^T
  }
  if (cta > capacity_full) throw Error(SPS_ERR_ARGUMENT, "svd_topk: blocks too large for one cooperative grid");
  Buf pb = E.alloc(sizeof(TopkProb) * nprob);
  keep.push_back(pb);
  E.stage(hp.data(), sizeof(TopkProb) * nprob, pb->ptr);
  const TopkProb* dp = (const TopkProb*)pb->ptr;
  int q0 = std::max(2, E.topk_hint), qstep = 2, qmax = 48;
  int* flag = E.dflag;
  // profile mode: phase trace of the first problem's CTA 0
  Buf tb;
  unsigned long long* trace = nullptr;
  if (E.profile) {
    tb = E.alloc(sizeof(unsigned long long) * (1 + 2 * TRACE_CAP));
    trace = (unsigned long long*)tb->ptr;
    SPS_CUDA(cudaMemsetAsync(trace, 0, sizeof(unsigned long long), E.stream));
  }
  void* args[] = {(void*)&dp,   (void*)&nprob, (void*)&q0,   (void*)&qstep,
                  (void*)&qmax, (void*)&tol,   (void*)&flag, (void*)&trace};
  const int tid = E.tic("svd_topk");
  SPS_CUDA(cudaLaunchCooperativeKernel((const void*)topk_kernel, dim3(cta), dim3(TT), args, smem, E.stream));
  E.toc(tid);
  E.launches++;
  // right vectors into the caller's layout, info and Ritz values to the host
  for (int i = 0; i < nprob; ++i)
    if (hp[i].Vi != ds[i].V)
      SPS_CUDA(cudaMemcpy2DAsync(ds[i].V, sizeof(double) * hp[i].n, hp[i].Vi, sizeof(double) * hp[i].ldn,
                                 sizeof(double) * hp[i].n, hp[i].k, cudaMemcpyDeviceToDevice, E.stream));
  int off = 0;
  for (int i = 0; i < nprob; ++i) {
    SPS_CUDA(cudaMemcpyAsync(E.hscal + off, hp[i].info, sizeof(double) * 6, cudaMemcpyDeviceToHost, E.stream));
    SPS_CUDA(cudaMemcpyAsync(E.hscal + off + 6, hp[i].s, sizeof(double) * hp[i].b, cudaMemcpyDeviceToHost,
                             E.stream));
    off += 6 + hp[i].b;
  }
  if (off + 1 > Engine::NSCAL) throw Error(SPS_ERR_ARGUMENT, "svd_topk: too many values");
  // the device flag travels with the values: one synchronisation
  int* hflag = reinterpret_cast<int*>(E.hscal + off);
  SPS_CUDA(cudaMemcpyAsync(hflag, E.dflag, sizeof(int), cudaMemcpyDeviceToHost, E.stream));
  E.sync();
  E.raise_flag(*hflag, "svd_topk");
  off = 0;
  int qused = 0;
  for (int i = 0; i < nprob; ++i) {
    TopkDesc& d = ds[i];
    d.status = (int)E.hscal[off];
    d.iterations = (int)E.hscal[off + 1];
    d.fro2 = E.hscal[off + 2];
    d.residual = E.hscal[off + 3];
    if (E.profile) E.add_stat("svd_topk.sweeps", 0.0, (long long)E.hscal[off + 5]);
    d.s.assign(E.hscal + off + 6, E.hscal + off + 6 + d.b);
    qused = std::max(qused, d.iterations);
    off += 6 + d.b;
  }
  if (trace) {
    std::vector<unsigned long long> h(1 + 2 * TRACE_CAP);
    SPS_CUDA(cudaMemcpy(h.data(), trace, sizeof(unsigned long long) * h.size(), cudaMemcpyDeviceToHost));
    int khz = 0;
    SPS_CUDA(cudaDeviceGetAttribute(&khz, cudaDevAttrClockRate, E.device));
    static const char* names[PH_COUNT] = {"start",  "init",   "gemm",     "gram",       "reduce",
                                          "cholesky", "apply", "store",   "jacobi",     "rotate",
                                          "residual", "gemm_issue", "gemm_wait", "gemm_mma"};
    const unsigned long long n = std::min<unsigned long long>(h[0], TRACE_CAP);
    for (unsigned long long i = 1; i < n; ++i) {
      const int ph = (int)h[1 + 2 * i];
      const double cyc = (double)(h[2 + 2 * i] - h[2 + 2 * (i - 1)]);
      if (ph > 0 && ph < PH_COUNT && khz > 0) E.add_stat(std::string("svd_topk.") + names[ph], cyc / khz);
    }
  }
  // work of the launch: the start M Omega, 2 m n b flops per half-iteration
  // (2 m^2 b per Gram iteration; M M^T itself is dgemm_cm's), and per
  // extraction M^T Q and the residual products M V
  double fl = 0;
  for (auto& d : ds) {
    const double ext = 1.0 + std::max(0, d.iterations - q0) / qstep;
    fl += d.gram ? 2.0 * d.m * d.m * d.iterations * d.b + 2.0 * d.m * d.n * d.b +
                       ext * (2.0 * d.m * d.n * d.b + 2.0 * d.m * d.n * d.k)
                 : 4.0 * d.iterations * d.m * d.n * d.b + 2.0 * d.m * d.n * d.b +
                       ext * (2.0 * d.m * d.n * d.b + 2.0 * d.m * d.n * d.k);
  }
  E.set_work(tid, fl);
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
