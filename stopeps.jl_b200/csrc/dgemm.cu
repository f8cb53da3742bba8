// Dense FP64 GEMM on the FP64 tensor cores: C = alpha op(A) B + beta C, all
// column-major, op(A) = A or A^T.  This is the compact-WY / Q-formation /
// Gram / subspace GEMM of the boundary compression (23328 x 648 x 648 blocks
// at chi=36, D=6).
//
// The FP64 tensor-core instruction on sm_100a is the warp-level
// mma.sync.m8n8k4.f64 (tcgen05 has no FP64 kind).  CTA tile 128 x 64 x 16,
// 8 warps as 4 (M) x 2 (N), warp tile 32 x 32 = 4 x 4 mma tiles; operands are
// staged global -> registers -> shared memory (double-buffered, so any
// alignment and leading dimension works), k-major in shared memory with row
// strides chosen so that a fragment load is two conflict-free wavefronts.
// Split-K writes FP64 partials that a second kernel reduces in a fixed order.
#include "engine.h"
#include <algorithm>
#include <mutex>

namespace sps {
namespace la {

namespace {

constexpr int TM = 128, TN = 64, TK = 16, NT = 256;
constexpr int ALD = TM + 8;   // 136 doubles: consecutive k rows land on opposite bank halves
constexpr int BLD = TN + 8;   // 72 doubles
constexpr int A_PER = TM * TK / NT;   // 8 elements of A per thread per tile
constexpr int B_PER = TN * TK / NT;   // 4 elements of B per thread per tile
constexpr size_t SMEM = sizeof(double) * 2 * TK * (ALD + BLD);

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

template <bool TA>
__device__ __forceinline__ void load_tile(const double* __restrict__ A, int lda, const double* __restrict__ B,
                                          int ldb, int M, int N, int i0, int j0, int k0, int kend, double (&ra)[A_PER],
                                          double (&rb)[B_PER]) {
  const int t = threadIdx.x;
  if (TA) {
    // op(A)(i,k) = A[k + i lda]: each thread reads 8 consecutive k of one row i
    const int i = i0 + (t >> 1), kb = k0 + (t & 1) * 8;
#pragma unroll
    for (int u = 0; u < A_PER; ++u) {
      const int k = kb + u;
      ra[u] = (i < M && k < kend) ? __ldg(&A[k + (size_t)i * lda]) : 0.0;
    }
  } else {
    // A[i + k lda]: each thread reads row i = t % 128 of 8 columns k
    const int i = i0 + (t & 127), kb = k0 + (t >> 7);
#pragma unroll
    for (int u = 0; u < A_PER; ++u) {
      const int k = kb + 2 * u;
      ra[u] = (i < M && k < kend) ? __ldg(&A[i + (size_t)k * lda]) : 0.0;
    }
  }
  // B[k + j ldb]: each thread reads 4 consecutive k of one column j
  const int j = j0 + (t >> 2), kb = k0 + (t & 3) * 4;
#pragma unroll
  for (int u = 0; u < B_PER; ++u) {
    const int k = kb + u;
    rb[u] = (j < N && k < kend) ? __ldg(&B[k + (size_t)j * ldb]) : 0.0;
  }
}

template <bool TA>
__device__ __forceinline__ void store_tile(double* As, double* Bs, const double (&ra)[A_PER],
                                           const double (&rb)[B_PER]) {
  const int t = threadIdx.x;
  if (TA) {
    const int i = t >> 1, kb = (t & 1) * 8;
#pragma unroll
    for (int u = 0; u < A_PER; ++u) As[(kb + u) * ALD + i] = ra[u];
  } else {
    const int i = t & 127, kb = t >> 7;
#pragma unroll
    for (int u = 0; u < A_PER; ++u) As[(kb + 2 * u) * ALD + i] = ra[u];
  }
  const int j = t >> 2, kb = (t & 3) * 4;
#pragma unroll
  for (int u = 0; u < B_PER; ++u) Bs[(kb + u) * BLD + j] = rb[u];
}

// symmetric results (sym): a tile wholly below the diagonal is not computed;
// its elements come from the mirrored elements of computed tiles
__host__ __device__ __forceinline__ bool tile_skipped(int i, int j) { return (i / TM) * TM >= (j / TN) * TN + TN; }

template <bool TA>
__global__ void __launch_bounds__(NT, 2) dgemm_tc_kernel(int M, int N, int K, const double* __restrict__ A, int lda,
                                                         const double* __restrict__ B, int ldb,
                                                         double* __restrict__ C, int ldc, double alpha, double beta,
                                                         int kchunk, double* __restrict__ partial, int sym) {
  extern __shared__ __align__(16) double gsm[];
  double* const As = gsm;                  // two buffers of TK x ALD
  double* const Bs = gsm + 2 * TK * ALD;   // two buffers of TK x BLD
  const int i0 = blockIdx.y * TM, j0 = blockIdx.x * TN;
  if (sym && tile_skipped(i0, j0)) return;
  const int kbeg = blockIdx.z * kchunk, kend = min(K, kbeg + kchunk);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wm = (warp & 3) * 32, wn = (warp >> 2) * 32;
  const int fr = lane >> 2, fc = lane & 3;   // fragment row / k index
  double acc[4][4][2];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;
  double ra[A_PER], rb[B_PER];
  int buf = 0;
  if (kbeg < kend) {
    load_tile<TA>(A, lda, B, ldb, M, N, i0, j0, kbeg, kend, ra, rb);
    store_tile<TA>(As, Bs, ra, rb);
  }
  __syncthreads();
  for (int k0 = kbeg; k0 < kend; k0 += TK) {
    const bool more = k0 + TK < kend;
    if (more) load_tile<TA>(A, lda, B, ldb, M, N, i0, j0, k0 + TK, kend, ra, rb);
    const double* as = As + buf * TK * ALD;
    const double* bs = Bs + buf * TK * BLD;
#pragma unroll
    for (int ks = 0; ks < TK; ks += 4) {
      double fa[4], fb[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) fa[a] = as[(ks + fc) * ALD + wm + a * 8 + fr];
#pragma unroll
      for (int b = 0; b < 4; ++b) fb[b] = bs[(ks + fc) * BLD + wn + b * 8 + fr];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) dmma(acc[a][b][0], acc[a][b][1], fa[a], fb[b]);
    }
    if (more) {
      store_tile<TA>(As + (buf ^ 1) * TK * ALD, Bs + (buf ^ 1) * TK * BLD, ra, rb);
      buf ^= 1;
    }
    __syncthreads();
  }
  // accumulator fragment: row fr, columns 2 fc + {0, 1} of each 8 x 8 tile
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const int i = i0 + wm + a * 8 + fr;
    if (i >= M) continue;
#pragma unroll
    for (int b = 0; b < 4; ++b)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int j = j0 + wn + b * 8 + 2 * fc + e;
        if (j >= N) continue;
        if (partial) {
          partial[(size_t)blockIdx.z * M * N + i + (size_t)j * M] = acc[a][b][e];
        } else {
          double* c = C + i + (size_t)j * ldc;
          *c = alpha * acc[a][b][e] + (beta == 0.0 ? 0.0 : beta * *c);
          if (sym && tile_skipped(j, i)) {   // the mirror's own tile is not computed
            double* cm = C + j + (size_t)i * ldc;
            *cm = alpha * acc[a][b][e] + (beta == 0.0 ? 0.0 : beta * *cm);
          }
        }
      }
  }
}

__global__ void splitk_reduce_kernel(int M, int N, int splits, const double* __restrict__ partial, double* C, int ldc,
                                     double alpha, double beta, int sym) {
  const size_t total = (size_t)M * N;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(e % M), j = (int)(e / M);
    // a skipped tile's element sums the partials of its mirror (whose tile is computed)
    const size_t src = (sym && tile_skipped(i, j)) ? (size_t)j + (size_t)i * M : e;
    double s = 0;
    for (int z = 0; z < splits; ++z) s += partial[(size_t)z * total + src];
    double* c = C + i + (size_t)j * ldc;
    *c = alpha * s + (beta == 0.0 ? 0.0 : beta * *c);
  }
}

}  // namespace

void dgemm_cm(Engine& E, bool ta, int M, int N, int K, double alpha, const double* A, int lda, const double* B,
              int ldb, double beta, double* C, int ldc, bool symmetric) {
  if (M <= 0 || N <= 0) return;
  if (symmetric && M != N) throw Error(SPS_ERR_ARGUMENT, "dgemm_cm: a symmetric product must be square");
  const int sym = symmetric ? 1 : 0;
  const int tiles = ((M + TM - 1) / TM) * ((N + TN - 1) / TN);
  int splits = 1, kchunk = std::max(K, 0);
  // split K when the output tiles alone cannot fill two CTAs per SM
  if (K > 4 * TK && tiles < 2 * E.num_sms) {
    splits = std::min((K + 63) / 64, std::max(1, (2 * E.num_sms + tiles - 1) / tiles));
    kchunk = (K + splits - 1) / splits;
    kchunk = ((kchunk + TK - 1) / TK) * TK;
    splits = (K + kchunk - 1) / kchunk;
  }
  dim3 grid((N + TN - 1) / TN, (M + TM - 1) / TM, splits);
  Buf part;
  double* partial = nullptr;
  if (splits > 1) {
    part = E.alloc(sizeof(double) * (size_t)splits * M * N);
    partial = (double*)part->ptr;
  }
  set_max_dynamic_smem((const void*)dgemm_tc_kernel<true>, (int)SMEM);
  set_max_dynamic_smem((const void*)dgemm_tc_kernel<false>, (int)SMEM);
  const int tk = E.tic("dgemm_cm");
  if (ta)
    dgemm_tc_kernel<true><<<grid, NT, SMEM, E.stream>>>(M, N, K, A, lda, B, ldb, C, ldc, alpha, beta, kchunk, partial,
                                                         sym);
  else
    dgemm_tc_kernel<false><<<grid, NT, SMEM, E.stream>>>(M, N, K, A, lda, B, ldb, C, ldc, alpha, beta, kchunk, partial,
                                                          sym);
  const double fl = sym ? (double)M * (M + 1) * (double)K : 2.0 * M * N * (double)K;
  E.toc(tk, fl, 8.0 * ((double)M * K + (double)K * N + 2.0 * M * N));
  SPS_CUDA(cudaGetLastError());
  E.launches++;
  if (splits > 1) {
    const size_t total = (size_t)M * N;
    const int g = (int)std::min<size_t>((total + 255) / 256, 4096);
    splitk_reduce_kernel<<<g, 256, 0, E.stream>>>(M, N, splits, partial, C, ldc, alpha, beta, sym);
    SPS_CUDA(cudaGetLastError());
    E.launches++;
  }
  E.flops += fl;
}

}  // namespace la
}  // namespace sps
