// sps_la_svd_noalloc: the one-sided Jacobi SVD of one small matrix for callers
// that cannot allocate device memory.
//
// Who needs it: code that runs where cudaMalloc is not available or not
// allowed -- a host callback or a library entered while another component
// owns the device allocator, a memory-capped embedding, or a caller that
// must not disturb its own allocator's pool.  Such a caller passes device
// buffers for the input and the outputs; every scratch byte the kernel needs
// lives in one file-scope __device__ array of fixed size below, so the call
// allocates nothing (no cudaMalloc, no cudaFree, no allocating library call).
//
// Results: a = u diag(s) vt with s descending; u and vt have orthonormal
// columns / rows even where singular values are zero (the factor is completed
// to an orthonormal set there).  NaN or Inf in a, or overflow in the column
// norms, returns SPS_ERR_NUMERIC with the outputs unspecified.
//
// Limits and sharing: max(m, n) <= SPS_NOALLOC_MAX_DIM and
// min(m, n) <= SPS_NOALLOC_MAX_RANK; larger problems are rejected with
// SPS_ERR_ARGUMENT.  The array is shared by every call on a device and keeps
// the contents of the last call (each call clears the words that must start at
// zero), so calls whose kernels overlap on the GPU race with each other:
// serialise them (one stream, or wait between calls).  Every GPU that loads
// the library holds the array until the process exits.
#include <cuda_runtime.h>
#include <cfloat>
#include <cstdint>
#include <cstring>
#include <mutex>

#include "stopeps_gpu.h"

namespace {

constexpr int SPS_NOALLOC_MAX_DIM = 256;
constexpr int SPS_NOALLOC_MAX_RANK = 128;
constexpr int MAXDEV = 64;
constexpr int NT = 256;
constexpr int NW = NT / 32;
// working U (MAX_DIM x MAX_RANK) + V (MAX_RANK^2) + sigma (MAX_RANK) + rank (MAX_RANK ints)
// + flag words
constexpr size_t SCRATCH_DOUBLES = (size_t)SPS_NOALLOC_MAX_DIM * SPS_NOALLOC_MAX_RANK +
                                   (size_t)SPS_NOALLOC_MAX_RANK * SPS_NOALLOC_MAX_RANK + 2 * SPS_NOALLOC_MAX_RANK + 32;

__device__ __align__(256) double g_noalloc_scratch[SCRATCH_DOUBLES];

std::mutex g_setup_mutex;
double* g_scratch_ptr[MAXDEV] = {nullptr};

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ int rr_index(int i, int round, int np) {
  return i == 0 ? 0 : ((i - 1 + round) % (np - 1)) + 1;
}

// a: m x n column-major (device, read only).  Works on X = a (m >= n) or a^T.
// u: m x k, s: k, vt: k x n (column-major), k = min(m, n).
__global__ void __launch_bounds__(NT) svd_noalloc_kernel(const double* __restrict__ a, int m, int n,
                                                         double* __restrict__ u, double* __restrict__ s,
                                                         double* __restrict__ vt, double* scratch) {
  const bool tall = m >= n;
  const int mm = tall ? m : n, nn = tall ? n : m;
  double* U = scratch;                                                   // mm x nn
  double* V = U + (size_t)SPS_NOALLOC_MAX_DIM * SPS_NOALLOC_MAX_RANK;    // nn x nn
  double* sig = V + (size_t)SPS_NOALLOC_MAX_RANK * SPS_NOALLOC_MAX_RANK;
  int* rank = (int*)(sig + SPS_NOALLOC_MAX_RANK);
  int* flag = (int*)(sig + 2 * SPS_NOALLOC_MAX_RANK);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __shared__ int rotations, nonfinite;
  if (threadIdx.x == 0) {
    *flag = 0;
    nonfinite = 0;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < mm * nn; e += NT) {
    int i = e % mm, j = e / mm;
    const double x = tall ? a[i + (size_t)j * m] : a[j + (size_t)i * m];
    if (!isfinite(x)) nonfinite = 1;
    U[e] = x;
  }
  for (int e = threadIdx.x; e < nn * nn; e += NT) V[e] = (e % nn == e / nn) ? 1.0 : 0.0;
  __syncthreads();
  if (nonfinite) {   // a NaN or Inf entry: no rotation test is meaningful, write nothing
    if (threadIdx.x == 0) *flag = 2;
    return;
  }
  const double tol = DBL_EPSILON * (double)max(mm, 2);
  const int np = nn + (nn & 1);
  bool converged = (nn == 1);
  for (int sweep = 0; sweep < 80 && !converged; ++sweep) {
    if (threadIdx.x == 0) rotations = 0;
    __syncthreads();
    for (int round = 0; round < np - 1; ++round) {
      for (int pr = warp; pr < np / 2; pr += NW) {
        int p = rr_index(pr, round, np), q = rr_index(np - 1 - pr, round, np);
        if (p >= nn || q >= nn) continue;
        if (p > q) { int t = p; p = q; q = t; }
        double* up = U + (size_t)p * mm;
        double* uq = U + (size_t)q * mm;
        double al = 0, be = 0, ga = 0;
        for (int i = lane; i < mm; i += 32) {
          double x = up[i], y = uq[i];
          al += x * x; be += y * y; ga += x * y;
        }
        al = warp_sum(al); be = warp_sum(be); ga = warp_sum(ga);
        if (!(al >= DBL_MIN && be >= DBL_MIN) || ga == 0.0 || !(fabs(ga) > tol * sqrt(al) * sqrt(be))) continue;
        double zeta = (be - al) / (2.0 * ga);
        double t = copysign(1.0, zeta) / (fabs(zeta) + hypot(1.0, zeta));
        double c = 1.0 / sqrt(1.0 + t * t), sn = c * t;
        for (int i = lane; i < mm; i += 32) {
          double x = up[i], y = uq[i];
          up[i] = c * x - sn * y;
          uq[i] = sn * x + c * y;
        }
        double* vp = V + (size_t)p * nn;
        double* vq = V + (size_t)q * nn;
        for (int i = lane; i < nn; i += 32) {
          double x = vp[i], y = vq[i];
          vp[i] = c * x - sn * y;
          vq[i] = sn * x + c * y;
        }
        if (lane == 0) atomicAdd(&rotations, 1);
      }
      __syncthreads();
    }
    converged = (rotations == 0);
    __syncthreads();
  }
  if (!converged && threadIdx.x == 0) *flag = 1;
  __shared__ int deficient[SPS_NOALLOC_MAX_RANK];
  __shared__ int bad;
  if (threadIdx.x == 0) bad = 0;
  __syncthreads();
  for (int c = warp; c < nn; c += NW) {
    double* uc = U + (size_t)c * mm;
    double v = 0;
    for (int i = lane; i < mm; i += 32) v += uc[i] * uc[i];
    v = warp_sum(v);
    const double sc = sqrt(v);
    // a column whose squared norm is below DBL_MIN took part in no rotation
    // test: its direction carries no information and is replaced below
    const bool zero = !(v >= DBL_MIN);
    if (lane == 0) {
      sig[c] = zero ? 0.0 : sc;
      deficient[c] = zero ? 1 : 0;
      if (!isfinite(sc)) bad = 1;
    }
    const double inv = zero ? 0.0 : 1.0 / sc;
    for (int i = lane; i < mm; i += 32) uc[i] *= inv;   // normalised Jacobi columns
  }
  __syncthreads();
  if (bad) {   // overflow in the column norms
    if (threadIdx.x == 0) *flag = 2;
    return;
  }
  // Complete the normalised columns to an orthonormal set where a column is
  // zero: take the unit vector e_j least covered by the columns already
  // orthonormal (sum_c U[j,c]^2 smallest, so its residual has squared norm at
  // least 1/mm), subtract its projection twice (classical Gram-Schmidt with
  // one reorthogonalisation) and normalise.
  __shared__ double red_v[NT];
  __shared__ int red_i[NT];
  __shared__ double coef[SPS_NOALLOC_MAX_RANK];
  for (int c = 0; c < nn; ++c) {
    if (!deficient[c]) continue;
    double best = 2.0;
    int bj = 0;
    for (int j = threadIdx.x; j < mm; j += NT) {
      double cov = 0;
      for (int q = 0; q < nn; ++q)
        if (!deficient[q]) cov += U[j + (size_t)q * mm] * U[j + (size_t)q * mm];
      if (cov < best) { best = cov; bj = j; }
    }
    red_v[threadIdx.x] = best;
    red_i[threadIdx.x] = bj;
    __syncthreads();
    for (int o = NT / 2; o > 0; o >>= 1) {
      if (threadIdx.x < o) {
        const double v2 = red_v[threadIdx.x + o];
        const int i2 = red_i[threadIdx.x + o];
        if (v2 < red_v[threadIdx.x] || (v2 == red_v[threadIdx.x] && i2 < red_i[threadIdx.x])) {
          red_v[threadIdx.x] = v2;
          red_i[threadIdx.x] = i2;
        }
      }
      __syncthreads();
    }
    const int jstar = red_i[0];
    double* x = U + (size_t)c * mm;
    for (int i = threadIdx.x; i < mm; i += NT) x[i] = (i == jstar) ? 1.0 : 0.0;
    __syncthreads();
    for (int pass = 0; pass < 2; ++pass) {
      for (int q = warp; q < nn; q += NW) {
        double d = 0;
        if (!deficient[q]) {
          const double* uq = U + (size_t)q * mm;
          for (int i = lane; i < mm; i += 32) d += uq[i] * x[i];
          d = warp_sum(d);
        }
        if (lane == 0) coef[q] = d;
      }
      __syncthreads();
      for (int i = threadIdx.x; i < mm; i += NT) {
        double v = x[i];
        for (int q = 0; q < nn; ++q)
          if (!deficient[q]) v -= coef[q] * U[i + (size_t)q * mm];
        x[i] = v;
      }
      __syncthreads();
    }
    if (warp == 0) {
      double v = 0;
      for (int i = lane; i < mm; i += 32) v += x[i] * x[i];
      v = warp_sum(v);
      if (lane == 0) coef[0] = v > 0 ? 1.0 / sqrt(v) : 0.0;
    }
    __syncthreads();
    const double inv = coef[0];
    for (int i = threadIdx.x; i < mm; i += NT) x[i] *= inv;
    __syncthreads();
    if (threadIdx.x == 0) deficient[c] = 0;   // now part of the orthonormal set
    __syncthreads();
  }
  for (int c = threadIdx.x; c < nn; c += NT) {
    double sc = sig[c];
    int r = 0;
    for (int j = 0; j < nn; ++j) r += (sig[j] > sc) || (sig[j] == sc && j < c);
    rank[c] = r;
    s[r] = sc;
  }
  __syncthreads();
  // X = Ux S V^T; for a^T the roles of the two factors swap.
  for (int c = warp; c < nn; c += NW) {
    int r = rank[c];
    const double* uc = U + (size_t)c * mm;
    const double* vc = V + (size_t)c * nn;
    if (tall) {
      for (int i = lane; i < m; i += 32) u[i + (size_t)r * m] = uc[i];
      for (int j = lane; j < n; j += 32) vt[r + (size_t)j * nn] = vc[j];
    } else {
      for (int i = lane; i < m; i += 32) u[i + (size_t)r * m] = vc[i];
      for (int j = lane; j < n; j += 32) vt[r + (size_t)j * nn] = uc[j];
    }
  }
}

// Once per device, with that device current: the device address of the array.
int scratch_for(int device, double** out) {
  if (device < 0 || device >= MAXDEV) return SPS_ERR_ARGUMENT;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_ptr[device]) {
    int prev = 0;
    if (cudaGetDevice(&prev) != cudaSuccess) return SPS_ERR_CUDA;
    if (cudaSetDevice(device) != cudaSuccess) return SPS_ERR_CUDA;
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    cudaSetDevice(prev);
    if (e != cudaSuccess || !p) return SPS_ERR_CUDA;
    g_scratch_ptr[device] = (double*)p;
  }
  *out = g_scratch_ptr[device];
  return SPS_OK;
}

}  // namespace

extern "C" int sps_la_svd_noalloc(int32_t device, void* stream, int32_t m, int32_t n, const double* a, double* u,
                                  double* s, double* vt) {
  if (m < 1 || n < 1 || !a || !u || !s || !vt) return SPS_ERR_ARGUMENT;
  if ((m > n ? m : n) > SPS_NOALLOC_MAX_DIM || (m < n ? m : n) > SPS_NOALLOC_MAX_RANK) return SPS_ERR_ARGUMENT;
  double* scratch = nullptr;
  int rc = scratch_for(device, &scratch);
  if (rc != SPS_OK) return rc;
  int prev = 0;
  if (cudaGetDevice(&prev) != cudaSuccess) return SPS_ERR_CUDA;
  if (prev != device && cudaSetDevice(device) != cudaSuccess) return SPS_ERR_CUDA;
  cudaStream_t st = (cudaStream_t)stream;
  svd_noalloc_kernel<<<1, NT, 0, st>>>(a, m, n, u, s, vt, scratch);
  cudaError_t e = cudaGetLastError();
  int flag = 0;
  if (e == cudaSuccess) {
    const double* fw = scratch + (size_t)SPS_NOALLOC_MAX_DIM * SPS_NOALLOC_MAX_RANK +
                       (size_t)SPS_NOALLOC_MAX_RANK * SPS_NOALLOC_MAX_RANK + 2 * SPS_NOALLOC_MAX_RANK;
    e = cudaMemcpyAsync(&flag, fw, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  }
  if (prev != device) cudaSetDevice(prev);
  if (e != cudaSuccess) return SPS_ERR_CUDA;
  if (flag == 2) return SPS_ERR_NUMERIC;
  return flag ? SPS_ERR_CONVERGENCE : SPS_OK;
}
