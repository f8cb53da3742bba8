// Z2 block-tensor engine on one B200: device buffers, strided Z2 tensors and
// the table-driven contraction / factorization primitives the hot path is
// written in.
//
// A tensor is a dense float64 array (arbitrary strides) plus one parity bit
// per basis state of every leg.  Entries whose parities sum to an odd number
// are structural zeros: kernels never read them as operands of a parity
// block and always leave them zero in outputs.  A matrix view of a tensor
// for (row legs | column legs) has two parity blocks; block c lists the
// row-major fused indices of parity c in increasing order (rows and columns
// alike).  Every GEMM, QR, LQ, SVD and eigendecomposition works on those
// blocks, which is what TensorKit does per coupled sector of a Z2 TensorMap.
#pragma once
#include <algorithm>
#include <chrono>
#include <functional>
#include <unordered_map>
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "stopeps_gpu.h"   // status codes shared with the C ABI

namespace sps {

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define SPS_CUDA(x)                                                              \
  do {                                                                           \
    cudaError_t e_ = (x);                                                        \
    if (e_ != cudaSuccess)                                                       \
      throw ::sps::Error(SPS_ERR_CUDA,                                  \
                         std::string(#x) + ": " + cudaGetErrorString(e_));       \
  } while (0)

// ---------------------------------------------------------------------------
// device memory pool (stream-ordered reuse on the engine's single stream)
// ---------------------------------------------------------------------------
// Thread-safe: a buffer allocated by one engine may be released by another
// host thread (batch workers hand states back to the handle).  Reuse stays
// stream-ordered because every batch call orders the handle's stream and the
// workers' streams by events at its start and end.
class Pool {
 public:
  void* get(size_t bytes);
  void put(void* p, size_t bytes);
  void trim();
  ~Pool();
  size_t held() const { return held_; }
 private:
  void trim_locked();
  std::mutex mu_;
  std::multimap<size_t, void*> free_;
  size_t held_ = 0;
};

struct DevBuf {
  Pool* pool = nullptr;
  void* ptr = nullptr;
  size_t bytes = 0;
  ~DevBuf() {
    if (ptr && pool) pool->put(ptr, bytes);
  }
};
using Buf = std::shared_ptr<DevBuf>;

using Par = std::shared_ptr<const std::vector<uint8_t>>;  // parity of each basis state
Par make_par(int n0, int n1);
Par make_par(std::vector<uint8_t> v);
Par fused_par(const std::vector<Par>& parts);
int par_count(const Par& p, int c);

struct Tensor {
  std::vector<Par> legs;
  std::vector<int64_t> dims;
  std::vector<int64_t> strides;   // in elements
  Buf buf;
  int64_t offset = 0;             // element offset into buf

  int rank() const { return (int)legs.size(); }
  int64_t size() const {
    int64_t s = 1;
    for (auto d : dims) s *= d;
    return s;
  }
  double* ptr() const { return buf ? (double*)buf->ptr + offset : nullptr; }
  bool contiguous() const;
};

// Scratch for values the host reads back after a sync.
struct HostScalars {
  double* h = nullptr;     // pinned host
  double* d = nullptr;     // device
  int n = 0;
};

class Engine {
 public:
  explicit Engine(int device);
  ~Engine();
  cudaStream_t stream = nullptr;
  int device = 0;
  int num_sms = 148;
  Pool pool;

  Buf alloc(size_t bytes);
  Tensor empty(const std::vector<Par>& legs);      // row-major, uninitialised
  Tensor zeros(const std::vector<Par>& legs);      // row-major, zero-filled
  Tensor upload(const std::vector<Par>& legs, const double* host);
  std::vector<double> download(const Tensor& t);   // row-major dense copy

  // device tables (int64) uploaded through a pinned staging ring
  int64_t* upload_i64(const std::vector<int64_t>& v, Buf& keep);
  int* upload_i32(const std::vector<int>& v, Buf& keep);

  // Copy small host data to the device through a pinned staging ring, so the
  // copy stays asynchronous (pageable-source copies serialise the stream).
  void stage(const void* src, size_t bytes, void* dst);
  char* ring = nullptr;
  size_t ring_size = 0, ring_pos = 0;

  void sync();
  // device-side error flag written by kernels (nonfinite values, iteration caps)
  int* dflag = nullptr;
  // dflag[1]: largest Jacobi sweep count since the last reset (diagnostic)
  void check_flag(const char* where);
  // throw for a flag value already copied to the host (after a sync)
  void raise_flag(int value, const char* where);

  // pinned scalar scratch
  double* hscal = nullptr;
  double* dscal = nullptr;
  static constexpr int NSCAL = 4096;

  // contraction plans: device-resident index tables of ein, keyed by the
  // spec and the operands' layouts (the same layouts recur in every draw)
  struct EinBlock {
    Buf ra, ca, rb, cb, rc, cc;
    int M = 0, N = 0, K = 0, a_kfast = 0, b_jfast = 0;
  };
  std::unordered_map<std::string, std::vector<EinBlock>> ein_plans;
  size_t ein_plan_bytes = 0;
  // arrival counters of the split-K contractions: zero between launches (the
  // last CTA of an output tile resets its counter)
  Buf gg_counters;
  size_t gg_counter_slots = 0;

  // largest grid of a cooperative launch (0: the whole GPU); engines that run
  // concurrently on one GPU share its SMs
  int ctas_cap = 0;
  int coop_capacity(int per_sm) const {
    const int c = std::max(1, per_sm) * num_sms;
    return ctas_cap > 0 ? std::min(c, ctas_cap) : c;
  }

  // pick launch shapes (split-K slices of the table-driven contraction, tile
  // width of the tcgen05 GEMM) by timing the candidates on first use (tune::)
  bool autotune = false;

  // arithmetic of the large contraction GEMMs: 0 FP64 (tensor-core DMMA and
  // table-driven kernels), 1 TF32, 2 3xTF32 (split), 3 3xBF16 (split), the last
  // three on tcgen05 with FP32 accumulation (tcgemm.cu); factorizations,
  // normalisations and log weights are FP64 in every mode
  int precision = 0;

  // host-side failure injection (tests): sweep cap of the single-CTA Jacobi
  // SVD / eigh kernels (0: their default of 80) and a forced PSD repair of
  // every full-update bond
  int sweep_cap = 0;
  bool force_repair = false;
  bool full_spectrum = false;    // truncated SVDs by the full spectrum (no subspace iteration)
  // eigendecompositions of blocks with at least this many rows in the PSD
  // repair take the multi-CTA route (eigh_unit_shifted); smaller ones the
  // single-CTA Jacobi eigh
  int eigh_multi_min = 1024;

  // starting iteration count of the subspace-iteration SVD (adapted per call)
  int topk_hint = 6;
  int topk_streak = 0;

  // counters
  long long launches = 0;
  double flops = 0;

  // optional per-kernel timing: tic() before a launch, toc() after it; events
  // are resolved by kernel_stats() after a sync.  Off unless `profile` is set.
  int profile = 0;   // 0 off, 1 per-kernel stats, 2 also per-shape contraction stats
  int tic(const char* name);
  void toc(int id, double algorithmic_flops = 0, double algorithmic_bytes = 0);
  void set_work(int id, double algorithmic_flops, double algorithmic_bytes = 0);
  struct KStat { double ms = 0, flops = 0, bytes = 0; long long count = 0; };
  std::map<std::string, KStat> kernel_stats();
  void reset_stats();
  void add_stat(const std::string& name, double ms, long long count = 1);   // host-measured sub-phase
 private:
  struct Pending { std::string name; cudaEvent_t a, b; double flops, bytes; };
  std::vector<Pending> pending_;
  std::vector<cudaEvent_t> event_pool_;
  std::map<std::string, KStat> stats_;
  cudaEvent_t get_event();
};

// ---------------------------------------------------------------------------
// tensor primitives (tensor_ops.cu)
// ---------------------------------------------------------------------------
// einsum with two operands: "abc,cde->abde" style labels (single chars).
Tensor ein(Engine& E, const std::string& spec, const Tensor& A, const Tensor& B, double alpha = 1.0);
// single-operand relabel / permutation (materialised contiguous)
Tensor perm(Engine& E, const Tensor& A, const std::vector<int>& order);
Tensor perm_view(const Tensor& A, const std::vector<int>& order);
Tensor contiguous(Engine& E, const Tensor& A);
Tensor fuse(Engine& E, const Tensor& A, int first, int count);
Tensor split(Engine& E, const Tensor& A, int axis, const std::vector<Par>& parts);
Tensor clone(Engine& E, const Tensor& A);
Tensor slice_leg(Engine& E, const Tensor& A, int axis, int index, Par newpar);

void scale_inplace(Engine& E, Tensor& A, double s);
// A := A / ||A|| computed on device (no host sync); flags nonfinite norms.
void safe_scale_inplace(Engine& E, Tensor& A);
Tensor axpby(Engine& E, double a, const Tensor& X, double b, const Tensor& Y);  // a X + b Y (same legs)
// Reductions into device scalar slot `slot` of E.dscal (read after E.sync()).
void norm2_to(Engine& E, const Tensor& A, int slot);   // sum of squares
void dot_to(Engine& E, const Tensor& A, const Tensor& B, int slot);
double norm(Engine& E, const Tensor& A);   // syncs
double dot(Engine& E, const Tensor& A, const Tensor& B);   // syncs
double sum_all(Engine& E, const Tensor& A);  // syncs
bool all_finite(Engine& E, const Tensor& A);  // syncs

// factorizations on the parity blocks of (rows | cols)
struct QRres { Tensor Q, R; };
QRres qr(Engine& E, const Tensor& A, const std::vector<int>& rows, const std::vector<int>& cols);
struct LQres { Tensor L, Q; };
LQres lq(Engine& E, const Tensor& A, const std::vector<int>& rows, const std::vector<int>& cols);

struct Trunc {
  int chi = -1;             // truncrank (-1: none)
  int space[2] = {-1, -1};  // truncspace per sector (-1: none)
  double atol = -1;         // trunctol (<0: none)
  // acceptance of iteratively computed singular triplets: residual
  // ||M v - s u|| relative to the largest singular value (rounding level by default)
  double rtol = 5e-14;
  // iterate on M M^T (one product per step; the condition number is squared,
  // so only for an rtol far above rounding)
  bool gram = false;
};
struct SVDres {
  Tensor U, V;                    // U (rows..., new), V (new, cols...)
  std::vector<double> S[2];       // kept singular values per sector (descending)
  double err = 0;                 // 2-norm of discarded values
  double entropy = 0;             // pretruncation Schmidt entropy (if asked)
  double norm = 0;                // Frobenius norm of the input
};
SVDres svd(Engine& E, const Tensor& A, const std::vector<int>& rows, const std::vector<int>& cols,
           const Trunc& tr, bool want_entropy = false);
// Truncated SVD returning one orthonormal factor and the product of the other
// with the singular values, computed from the original matrix by one GEMM:
//  left  = true : F = U (rows..., new),  W = S V^T = U^T A  (new, cols...)
//  left  = false: F = V^T (new, cols...), W = U S = A V     (rows..., new)
// Large blocks: QR/LQ preconditioning + U-only Jacobi (multi-CTA).
struct KeptSVD {
  Tensor F, W;
  std::vector<double> S[2];
  double err = 0, entropy = 0, norm = 0;
};
KeptSVD svd_kept(Engine& E, const Tensor& A, const std::vector<int>& rows, const std::vector<int>& cols,
                 const Trunc& tr, bool want_entropy, bool left);
// the kept index sets of a truncation over per-block singular values (each
// block descending): truncrank & truncspace & trunctol, as svd applies them
void truncation_keep(const std::vector<double> s[2], const Trunc& tr, std::vector<char> keep[2]);
// true when the kept-vector path (svd_kept) beats the full SVD for this view
bool svd_prefers_kept(const Tensor& A, const std::vector<int>& rows, const std::vector<int>& cols, const Trunc& tr,
                      bool want_entropy);
// eigendecomposition of a symmetric block matrix (rows | cols must match)
struct EIGres {
  std::vector<double> w[2];   // eigenvalues (ascending) per block
  Tensor V;                   // (rows..., new)
};
EIGres eigh(Engine& E, const Tensor& A, const std::vector<int>& rows, const std::vector<int>& cols);
// eigendecomposition of a symmetric block matrix whose spectral norm is at
// most 1 (e.g. Frobenius-normalised), for blocks too large for the single-CTA
// eigh: the one-sided Jacobi SVD (multi-CTA) of A + I, which is positive
// semidefinite, so its singular pairs are its eigenpairs; w = sigma - 1
// (descending per block), V the singular vectors
EIGres eigh_unit_shifted(Engine& E, const Tensor& A, const std::vector<int>& rows, const std::vector<int>& cols);
// block inverse of a square 2-leg tensor (out,in) -> (in,out)
Tensor block_inverse(Engine& E, const Tensor& R);
// multiply a leg by a per-state diagonal (values in leg order) : A[..k..] *= d[k]
Tensor scale_leg(Engine& E, const Tensor& A, int axis, const std::vector<double>& d);

// host view of parity blocks (for tests / small control decisions)
std::vector<int64_t> block_index(const std::vector<Par>& legs, const std::vector<int64_t>& strides,
                                 int c);

// Householder / Jacobi kernels (linalg.cu)
namespace la {
// column-major m x n blocks, batched over `count` problems given by descriptor arrays
struct MatDesc {
  double* a;       // input (overwritten), column-major, lda
  double* q;       // output Q (column-major, ldq) for QR / U for SVD / V for eig
  double* r;       // output R (column-major, ldr) / V for SVD
  double* s;       // singular / eigen values
  int m, n, lda, ldq, ldr;
};
void qr_batched(Engine& E, const std::vector<MatDesc>& d);
void svd_batched(Engine& E, const std::vector<MatDesc>& d);    // m >= n required
void eigh_batched(Engine& E, const std::vector<MatDesc>& d);   // symmetric n x n
void inv_batched(Engine& E, const std::vector<MatDesc>& d);    // general square
// multi-CTA versions for large blocks (bigla.cu)
void qr_big(Engine& E, double* a, int m, int n, int lda, double* q, int ldq, double* r, int ldr);  // m >= n
void qr_big_opt(Engine& E, double* a, int m, int n, int lda, double* q, int ldq, double* r, int ldr, bool form_q);
// U-only one-sided Jacobi: q = sorted normalized columns of a (left singular vectors), s = values
void jacobi_left(Engine& E, const std::vector<MatDesc>& d);
void transpose_cm(Engine& E, const double* src, int m, int n, int lds, double* dst, int ldd);
void svd_big(Engine& E, const std::vector<MatDesc>& d);        // m >= n, ld = m / n
// symmetric: the product is known to be symmetric (M == N, e.g. A A^T); only
// tiles on or above the diagonal are computed and the rest mirrored
void dgemm_cm(Engine& E, bool ta, int M, int N, int K, double alpha, const double* A, int lda, const double* B,
              int ldb, double beta, double* C, int ldc, bool symmetric = false);
bool qr_is_big(int m, int n);
bool svd_is_big(int m, int n);
// leading k singular triplets of an m x n column-major block (ld m) by block
// subspace iteration with Rayleigh-Ritz extraction (topk.cu)
struct TopkDesc {
  const double* M;
  int m, n, k;
  double* U;                 // m x k (ld m), left vectors, descending values
  double* V;                 // n x k (ld n), right vectors
  bool gram = false;         // iterate on the Gram matrix M M^T (extraction still from M)
  // results
  int b = 0, status = -1, iterations = 0;
  double fro2 = 0, residual = 0;   // ||M||_F^2; largest residual / acceptance threshold
  std::vector<double> s;     // b Ritz values, descending (the first k are the wanted values)
};
int topk_block_size(int k, int m, int n);   // 0 when the block is too small for the method
bool topk_fits(int k, int m, int n, int nprob, Engine& E);
void svd_topk(Engine& E, std::vector<TopkDesc>& ds, double tol);
}  // namespace la

// host time of a scope, recorded as a statistic in profile mode
struct HostTimer {
  Engine& E;
  const char* name;
  std::chrono::steady_clock::time_point t0;
  HostTimer(Engine& e, const char* n);
  ~HostTimer();
};

// Per-device kernel attributes.  The opt-in dynamic shared-memory limit is a
// property of the (device, kernel) pair, so it is set once per pair for the
// current device; occupancy (CTAs per SM) is cached per (device, kernel, smem).
void set_max_dynamic_smem(const void* kernel, int bytes);
int occupancy_per_sm(const void* kernel, int threads, size_t smem);

// autotuner (autotune.cu): a process-wide table of launch-shape choices
namespace tune {
std::string key(Engine& E, const char* op, std::initializer_list<long long> shape);
bool lookup(const std::string& key, int* choice);
// the tuned choice for `key`: on a miss, times run(candidate) for each
// candidate on the engine's stream (synchronising) and stores the fastest
int pick(Engine& E, const std::string& key, const std::vector<int>& candidates, const std::function<void(int)>& run);
std::string report_json();
void clear();
}  // namespace tune

// tcgen05 contraction GEMM of one parity block (tcgemm.cu):
// C[rc[i] + cc[j]] = alpha sum_k A[ra[i] + ca[k]] B[rb[k] + cb[j]] in the
// low-precision mode `mode` (1 TF32, 2 3xTF32, 3 3xBF16) with FP32 accumulation
namespace tc {
void gemm_block(Engine& E, int mode, const double* A, const int64_t* ra, const int64_t* ca, int a_kfast,
                const double* B, const int64_t* rb, const int64_t* cb, int b_jfast, double* C, const int64_t* rc,
                const int64_t* cc, int M, int N, int K, double alpha);
// a block worth the pack + tensor-core route
inline bool worth(int M, int N, int K) {
  return M >= 64 && N >= 32 && K >= 32 && 2.0 * M * N * (double)K >= 3.2e7;
}
}  // namespace tc

// gather/scatter between tensors and dense column-major block matrices
void gather_block(Engine& E, const Tensor& A, const int64_t* rt, const int64_t* ct, int M, int N,
                  double* dst, int ld, bool transpose);
void scatter_block(Engine& E, Tensor& A, const int64_t* rt, const int64_t* ct, int M, int N,
                   const double* src, int ld, bool transpose);

}  // namespace sps
