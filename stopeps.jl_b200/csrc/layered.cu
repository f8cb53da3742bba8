// One row step of the double layer in a single kernel: the environment X
// (w, b, n, c) contracted over (w, n) with double_layer(ket, ket), giving
// (b, c, e_ket, e_bra, s_ket, s_bra) — the ket step and the bra step of
// _left_step (src/contraction/boundary_mps.jl:216-231) fused, so the
// (chi^2 D^2) x (P A D^2) intermediate never goes to global memory.
//
// The tensors are dense (parity-forbidden entries are stored zeros), so the
// kernel contracts them densely: per (b, c) the two steps are D^2 x D^2 x
// (P A D^2) products, exact zeros contribute exact zeros, and the result is
// the block-sparse contraction's to rounding.  One CTA owns one b and a chunk
// of CC values of c: it copies the ket and its slice of X into shared memory,
// forms Y[(c,y,v), (p,a,e,f)] = sum_(x,u) X[c,x,y,u,v] ket[(x,u),(p,a,e,f)] in
// shared memory, then Z[(c,e,f), (g,h)] = sum_(y,v,p,a) Y ket[(y,v,p,a),(g,h)]
// straight to the output.  Both products run on the FP64 tensor cores
// (mma.m8n8k4.f64): a warp owns a strip of up to four 8 x 8 output tiles that
// share one A fragment per k-step, operands read from shared memory through
// row and k offset tables.
#include "pipeline.h"
#include <algorithm>
#include <mutex>
#include <string>

namespace sps {

namespace {

constexpr int LT = 256;
constexpr size_t LW_SMEM_TWO = 110 * 1024;   // two CTAs per SM
constexpr size_t LW_SMEM_ONE = 200 * 1024;

struct LayerWN {
  const double* X;                 // (x, y, b, u, v, c) view of the environment
  int64_t sx, sy, sb, su, sv, sc;  // its element strides
  const double* K;                 // ket, dense row-major (x, u, p, a, e, f)
  double* Z;                       // (b, c, e, g, f, h), dense row-major
  int B, C, Dw, Dn, PA, De, Ds, CC;
};

// 8-byte asynchronous copy global -> shared (bytes = 0 writes a zero)
__device__ __forceinline__ void cp_async8_lw(double* dst, const double* src, int bytes) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(a), "l"(src), "r"(bytes) : "memory");
}

__device__ __forceinline__ void dmma_lw(double& d0, double& d1, double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
      : "+d"(d0), "+d"(d1)
      : "d"(a), "d"(b));
}

// C[r][n] = sum_k A[rowoff[r] + koff[k]] Bm[k ldb + n] for r < R, n < N on the
// FP64 tensor cores; k ascending in every sum (deterministic).  Rows and
// columns past the edges are clamped copies whose results are dropped; k
// past K reads zeros.
template <class Store>
__device__ __forceinline__ void mma_gemm(int R, int N, int K, const double* A, const int* rowoff, const int* koff,
                                         const double* Bm, int ldb, Store store) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, fr = lane >> 2, fc = lane & 3;
  const int RT = (R + 7) >> 3, NT = (N + 7) >> 3, NS = (NT + 3) >> 2;
  for (int s = warp; s < RT * NS; s += LT / 32) {
    const int rt = s / NS, ns = s - rt * NS;
    const int ntl = min(4, NT - ns * 4);   // n-tiles in this strip (warp-uniform)
    const int ro = rowoff[min(rt * 8 + fr, R - 1)];
    int nb[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) nb[j] = min((ns * 4 + j) * 8 + fr, N - 1);
    double acc[4][2];
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[j][0] = acc[j][1] = 0.0;
    for (int k0 = 0; k0 < K; k0 += 4) {
      const int k = k0 + fc;
      const bool kin = k < K;
      const int kk = kin ? k : 0;
      const double a = kin ? A[ro + koff[kk]] : 0.0;
      const double* bk = Bm + kk * ldb;
#pragma unroll
      for (int j = 0; j < 4; ++j)
        if (j < ntl) dmma_lw(acc[j][0], acc[j][1], a, kin ? bk[nb[j]] : 0.0);
    }
    // accumulator fragment: row fr, columns 2 fc + {0, 1} of each tile
    const int r = rt * 8 + fr;
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int n = (ns * 4 + j) * 8 + 2 * fc + e;
        if (j < ntl && r < R && n < N) store(r, n, acc[j][e]);
      }
  }
}

// DW, DN, DE, DS: the bond dimensions when known at compile time (0: read
// from d), so that the index arithmetic needs no runtime division; CC is a
// power of two (lgc = log2 CC).
template <int DW, int DN, int DE, int DS>
__global__ void __launch_bounds__(LT) layer_wn_kernel(LayerWN d, int lgc) {
  extern __shared__ __align__(16) double sm[];
  const int Dw = DW ? DW : d.Dw, Dn = DN ? DN : d.Dn, De = DE ? DE : d.De, Ds = DS ? DS : d.Ds;
  const int PA = d.PA, CC = 1 << lgc;
  const int K1 = Dw * Dn, N2 = De * Ds, N1 = PA * N2, X4 = K1 * K1;
  const int b = blockIdx.y, c0 = blockIdx.x * CC, cn = min(CC, d.C - c0);
  double* Ks = sm;                     // K1 x N1
  double* Xs = Ks + K1 * N1;           // [c][x][y][u][v]
  double* Ys = Xs + CC * X4;           // [c][y][v][p a][e][f]
  int* ro1 = reinterpret_cast<int*>(Ys + CC * K1 * N1);
  int* ko1 = ro1 + CC * K1;
  int* ro2 = ko1 + K1;
  int* ko2 = ro2 + CC * N2;
  const int t = threadIdx.x;
  // every copy of the ket and of the X slice in flight at once
  for (int e = t; e < K1 * N1; e += LT) cp_async8_lw(Ks + e, d.K + e, 8);
  const double* Xb = d.X + (int64_t)b * d.sb + (int64_t)c0 * d.sc;
  for (int e = t; e < CC * X4; e += LT) {   // c fastest: consecutive threads read consecutive c
    const int c = e & (CC - 1);
    int q = e >> lgc;
    const int v = q % Dn;
    q /= Dn;
    const int u = q % Dn;
    q /= Dn;
    const int y = q % Dw, x = q / Dw;
    const bool ok = c < cn;
    cp_async8_lw(Xs + c * X4 + ((x * Dw + y) * Dn + u) * Dn + v,
                 ok ? Xb + c * d.sc + x * d.sx + y * d.sy + u * d.su + v * d.sv : d.K, ok ? 8 : 0);
  }
  asm volatile("cp.async.commit_group;" ::: "memory");
  for (int r = t; r < CC * K1; r += LT) {   // r = (c, y, v)
    const int c = r / K1, y = (r % K1) / Dn, v = r % Dn;
    ro1[r] = c * X4 + y * Dn * Dn + v;
  }
  for (int k = t; k < K1; k += LT) ko1[k] = (k / Dn) * Dw * Dn * Dn + (k % Dn) * Dn;   // k = (x, u)
  for (int r = t; r < CC * N2; r += LT) ro2[r] = (r / N2) * K1 * N1 + r % N2;          // r = (c, e, f)
  for (int k = t; k < K1 * PA; k += LT) ko2[k] = k * N2;                                // k = (y, v, p a)
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  __syncthreads();
  mma_gemm(CC * K1, N1, K1, Xs, ro1, ko1, Ks, N1, [&](int r, int n, double v) { Ys[r * N1 + n] = v; });
  __syncthreads();
  double* Zb = d.Z + ((int64_t)b * d.C + c0) * N2 * N2;
  mma_gemm(CC * N2, N2, K1 * PA, Ys, ro2, ko2, Ks, N2, [&](int r, int n, double v) {
    const int c = r / N2, ef = r % N2, e = ef / Ds, f = ef % Ds, g = n / Ds, h = n % Ds;
    if (c < cn) Zb[(int64_t)c * N2 * N2 + ((e * De + g) * Ds + f) * Ds + h] = v;
  });
}

size_t layer_wn_smem(int CC, int K1, int N1, int N2, int PA) {
  const size_t dbl = (size_t)K1 * N1 + (size_t)CC * ((size_t)K1 * K1 + (size_t)K1 * N1);
  const size_t ints = (size_t)CC * K1 + K1 + (size_t)CC * N2 + (size_t)K1 * PA;
  return sizeof(double) * dbl + sizeof(int) * ints;
}

}  // namespace

bool layer_wn_fused(Engine& E, const Tensor& X5, const Tensor& ket0, Tensor& Z) {
  if (X5.rank() != 6 || ket0.rank() != 6) return false;
  const int Dw = (int)ket0.dims[0], Dn = (int)ket0.dims[1], PA = (int)(ket0.dims[2] * ket0.dims[3]);
  const int De = (int)ket0.dims[4], Ds = (int)ket0.dims[5];
  if (X5.dims[0] != Dw || X5.dims[1] != Dw || X5.dims[3] != Dn || X5.dims[4] != Dn) return false;
  const int B = (int)X5.dims[2], C = (int)X5.dims[5];
  const int K1 = Dw * Dn, N2 = De * Ds, N1 = PA * N2;
  // measured to beat the two table-driven contractions up to D = 6 (D^2 <= 36 on
  // each side); at D = 8 the tiles need one SM each and the dense products
  // (twice the block-sparse flops) no longer pay
  if (K1 > 36 || N2 > 36) return false;
  // the largest chunk of c that keeps two CTAs per SM (else one), shrunk
  // while the grid is under eight CTAs per SM (small CTAs cut the last wave
  // and, at 52 KB, four of them share an SM)
  int CC = 8;
  while (CC > 1 && (CC > C || layer_wn_smem(CC, K1, N1, N2, PA) > LW_SMEM_TWO)) CC >>= 1;
  while (CC > 1 && (long long)((C + CC - 1) / CC) * B < 8LL * E.num_sms) CC >>= 1;
  int lgc = 0;
  while ((1 << lgc) < CC) ++lgc;
  const size_t smem = layer_wn_smem(CC, K1, N1, N2, PA);
  if (smem > LW_SMEM_ONE || B == 0 || C == 0) return false;
  Tensor ket = contiguous(E, ket0);
  Z = E.empty({X5.legs[2], X5.legs[5], ket.legs[4], ket.legs[4], ket.legs[5], ket.legs[5]});
  set_max_dynamic_smem((const void*)layer_wn_kernel<6, 6, 6, 6>, (int)LW_SMEM_ONE);
  set_max_dynamic_smem((const void*)layer_wn_kernel<0, 0, 0, 0>, (int)LW_SMEM_ONE);
  LayerWN d;
  d.X = X5.ptr();
  d.sx = X5.strides[0];
  d.sy = X5.strides[1];
  d.sb = X5.strides[2];
  d.su = X5.strides[3];
  d.sv = X5.strides[4];
  d.sc = X5.strides[5];
  d.K = ket.ptr();
  d.Z = Z.ptr();
  d.B = B;
  d.C = C;
  d.Dw = Dw;
  d.Dn = Dn;
  d.PA = PA;
  d.De = De;
  d.Ds = Ds;
  d.CC = CC;
  dim3 grid((C + CC - 1) / CC, B);
  const double fl = 2.0 * B * C * ((double)K1 * K1 * N1 + (double)N2 * K1 * PA * N2);
  const double by = 8.0 * ((double)X5.size() + (double)Z.size());
  const int tk = E.tic("layer_wn");
  int tshape = -1;
  if (E.profile > 1) {
    const std::string nm = "layer_wn " + std::to_string(B) + "x" + std::to_string(C) + " D" + std::to_string(Dw) + "." +
                           std::to_string(Dn) + "." + std::to_string(De) + "." + std::to_string(Ds) + " cc" +
                           std::to_string(CC) + " g" + std::to_string(grid.x * grid.y);
    tshape = E.tic(nm.c_str());
  }
  if (Dw == 6 && Dn == 6 && De == 6 && Ds == 6)
    layer_wn_kernel<6, 6, 6, 6><<<grid, LT, smem, E.stream>>>(d, lgc);
  else
    layer_wn_kernel<0, 0, 0, 0><<<grid, LT, smem, E.stream>>>(d, lgc);
  E.toc(tk, fl, by);
  E.toc(tshape, fl, by);
  SPS_CUDA(cudaGetLastError());
  E.launches++;
  E.flops += fl;
  return true;
}

}  // namespace sps
