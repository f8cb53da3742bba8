// Engine plumbing and the Z2 tensor primitives: table-driven block GEMM
// (the contraction of every @tensor/ncon in the reference), strided
// permutes, reductions, and the block gather/scatter around the
// factorization kernels of linalg.cu.
#include "engine.h"
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <mutex>
#include <numeric>
#include <tuple>

namespace sps {

// ---------------------------------------------------------------------------
// pool
// ---------------------------------------------------------------------------
static size_t round_bytes(size_t b) {
  if (b < 256) return 256;
  if (b < (1u << 20)) {
    size_t r = 256;
    while (r < b) r <<= 1;
    return r;
  }
  size_t mb = (size_t)1 << 20;
  return ((b + mb - 1) / mb) * mb;
}

void* Pool::get(size_t bytes) {
  std::lock_guard<std::mutex> g(mu_);
  auto it = free_.lower_bound(bytes);
  if (it != free_.end() && it->first <= bytes + bytes / 4 + 4096) {
    void* p = it->second;
    held_ -= it->first;
    free_.erase(it);
    return p;
  }
  void* p = nullptr;
  cudaError_t e = cudaMalloc(&p, bytes);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    trim_locked();
    SPS_CUDA(cudaMalloc(&p, bytes));
  }
  return p;
}

void Pool::put(void* p, size_t bytes) {
  std::lock_guard<std::mutex> g(mu_);
  free_.emplace(bytes, p);
  held_ += bytes;
}

void Pool::trim() {
  std::lock_guard<std::mutex> g(mu_);
  trim_locked();
}

void Pool::trim_locked() {
  cudaDeviceSynchronize();
  for (auto& kv : free_) cudaFree(kv.second);
  free_.clear();
  held_ = 0;
}

Pool::~Pool() {
  for (auto& kv : free_) cudaFree(kv.second);
}

// ---------------------------------------------------------------------------
// parities
// ---------------------------------------------------------------------------
Par make_par(int n0, int n1) {
  std::vector<uint8_t> v(n0 + n1, 0);
  for (int i = n0; i < n0 + n1; ++i) v[i] = 1;
  return std::make_shared<const std::vector<uint8_t>>(std::move(v));
}
Par make_par(std::vector<uint8_t> v) { return std::make_shared<const std::vector<uint8_t>>(std::move(v)); }
Par fused_par(const std::vector<Par>& parts) {
  std::vector<uint8_t> out(1, 0);
  for (auto& p : parts) {
    std::vector<uint8_t> nx;
    nx.reserve(out.size() * p->size());
    for (auto a : out)
      for (auto b : *p) nx.push_back(a ^ b);
    out.swap(nx);
  }
  return make_par(std::move(out));
}
int par_count(const Par& p, int c) {
  int n = 0;
  for (auto x : *p) n += (x == c);
  return n;
}

bool Tensor::contiguous() const {
  int64_t s = 1;
  for (int k = rank() - 1; k >= 0; --k) {
    if (dims[k] != 1 && strides[k] != s) return false;
    s *= dims[k];
  }
  return true;
}

static std::vector<int64_t> rowmajor_strides(const std::vector<int64_t>& dims) {
  std::vector<int64_t> s(dims.size());
  int64_t acc = 1;
  for (int k = (int)dims.size() - 1; k >= 0; --k) {
    s[k] = acc;
    acc *= dims[k];
  }
  return s;
}

// ---------------------------------------------------------------------------
// engine
// ---------------------------------------------------------------------------
Engine::Engine(int dev) : device(dev) {
  SPS_CUDA(cudaSetDevice(dev));
  SPS_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
  cudaDeviceProp prop;
  SPS_CUDA(cudaGetDeviceProperties(&prop, dev));
  num_sms = prop.multiProcessorCount;
  SPS_CUDA(cudaMalloc(&dflag, sizeof(int) * 4));
  SPS_CUDA(cudaMemset(dflag, 0, sizeof(int) * 4));
  SPS_CUDA(cudaMallocHost(&hscal, sizeof(double) * NSCAL));
  ring_size = (size_t)64 << 20;
  SPS_CUDA(cudaMallocHost(&ring, ring_size));
  SPS_CUDA(cudaMalloc(&dscal, sizeof(double) * NSCAL));
}

Engine::~Engine() {
  cudaStreamSynchronize(stream);
  cudaFree(dflag);
  cudaFree(dscal);
  cudaFreeHost(hscal);
  cudaFreeHost(ring);
  cudaStreamDestroy(stream);
}

Buf Engine::alloc(size_t bytes) {
  auto b = std::make_shared<DevBuf>();
  b->pool = &pool;
  b->bytes = round_bytes(std::max<size_t>(bytes, 1));
  b->ptr = pool.get(b->bytes);
  return b;
}

Tensor Engine::empty(const std::vector<Par>& legs) {
  Tensor t;
  t.legs = legs;
  for (auto& p : legs) t.dims.push_back((int64_t)p->size());
  t.strides = rowmajor_strides(t.dims);
  t.buf = alloc(std::max<int64_t>(t.size(), 1) * sizeof(double));
  return t;
}

Tensor Engine::zeros(const std::vector<Par>& legs) {
  Tensor t = empty(legs);
  SPS_CUDA(cudaMemsetAsync(t.ptr(), 0, std::max<int64_t>(t.size(), 1) * sizeof(double), stream));
  return t;
}

Tensor Engine::upload(const std::vector<Par>& legs, const double* host) {
  Tensor t = empty(legs);
  stage(host, t.size() * sizeof(double), t.ptr());
  return t;
}

std::vector<double> Engine::download(const Tensor& t0) {
  Tensor t = contiguous(*this, t0);
  std::vector<double> h(t.size());
  SPS_CUDA(cudaMemcpyAsync(h.data(), t.ptr(), t.size() * sizeof(double), cudaMemcpyDeviceToHost,
                           stream));
  sync();
  return h;
}

void Engine::stage(const void* src, size_t bytes, void* dst) {
  if (bytes == 0) return;
  size_t need = (bytes + 255) & ~(size_t)255;
  if (need > ring_size) {   // too large for the ring: synchronous copy
    SPS_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream));
    return;
  }
  if (ring_pos + need > ring_size) sync();   // every earlier staged copy has completed
  std::memcpy(ring + ring_pos, src, bytes);
  SPS_CUDA(cudaMemcpyAsync(dst, ring + ring_pos, bytes, cudaMemcpyHostToDevice, stream));
  ring_pos += need;
}

int64_t* Engine::upload_i64(const std::vector<int64_t>& v, Buf& keep) {
  keep = alloc(std::max<size_t>(v.size(), 1) * sizeof(int64_t));
  stage(v.data(), v.size() * sizeof(int64_t), keep->ptr);
  return (int64_t*)keep->ptr;
}

int* Engine::upload_i32(const std::vector<int>& v, Buf& keep) {
  keep = alloc(std::max<size_t>(v.size(), 1) * sizeof(int));
  stage(v.data(), v.size() * sizeof(int), keep->ptr);
  return (int*)keep->ptr;
}

cudaEvent_t Engine::get_event() {
  if (!event_pool_.empty()) {
    cudaEvent_t e = event_pool_.back();
    event_pool_.pop_back();
    return e;
  }
  cudaEvent_t e;
  SPS_CUDA(cudaEventCreate(&e));
  return e;
}

int Engine::tic(const char* name) {
  if (!profile) return -1;
  Pending p;
  p.name = name;
  p.a = get_event();
  p.b = get_event();
  p.flops = p.bytes = 0;
  SPS_CUDA(cudaEventRecord(p.a, stream));
  pending_.push_back(p);
  return (int)pending_.size() - 1;
}

void Engine::toc(int id, double fl, double by) {
  if (id < 0 || id >= (int)pending_.size()) return;
  pending_[id].flops = fl;
  pending_[id].bytes = by;
  SPS_CUDA(cudaEventRecord(pending_[id].b, stream));
}

void Engine::set_work(int id, double fl, double by) {
  if (id < 0 || id >= (int)pending_.size()) return;
  pending_[id].flops = fl;
  pending_[id].bytes = by;
}

HostTimer::HostTimer(Engine& e, const char* n) : E(e), name(n) {
  if (E.profile) t0 = std::chrono::steady_clock::now();
}
HostTimer::~HostTimer() {
  if (E.profile)
    E.add_stat(name, std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count());
}

void Engine::add_stat(const std::string& name, double ms, long long count) {
  auto& k = stats_[name];
  k.ms += ms;
  k.count += count;
}

std::map<std::string, Engine::KStat> Engine::kernel_stats() {
  SPS_CUDA(cudaStreamSynchronize(stream));
  for (auto& p : pending_) {
    float ms = 0;
    SPS_CUDA(cudaEventElapsedTime(&ms, p.a, p.b));
    auto& k = stats_[p.name];
    k.ms += ms;
    k.flops += p.flops;
    k.bytes += p.bytes;
    k.count++;
    event_pool_.push_back(p.a);
    event_pool_.push_back(p.b);
  }
  pending_.clear();
  return stats_;
}

void Engine::reset_stats() {
  kernel_stats();
  stats_.clear();
}

void Engine::sync() {
  HostTimer ht(*this, "host.sync");
  SPS_CUDA(cudaStreamSynchronize(stream));
  ring_pos = 0;
}

void Engine::check_flag(const char* where) {
  int h = 0;
  SPS_CUDA(cudaMemcpyAsync(&h, dflag, sizeof(int), cudaMemcpyDeviceToHost, stream));
  sync();
  raise_flag(h, where);
}

void Engine::raise_flag(int h, const char* where) {
  if (h) {
    SPS_CUDA(cudaMemsetAsync(dflag, 0, sizeof(int), stream));
    if (h & 2) throw Error(SPS_ERR_CONVERGENCE, std::string(where) + ": device iteration cap reached");
    if (h & 4) throw Error(SPS_ERR_NUMERIC, std::string(where) + ": a grid barrier wait reached its cap");
    if (h & 8) throw Error(SPS_ERR_NUMERIC, std::string(where) + ": a bulk-copy wait reached its cap");
    throw Error(SPS_ERR_NUMERIC, std::string(where) + ": nonfinite or singular value on device");
  }
}

// ---------------------------------------------------------------------------
// per-device kernel attributes
// ---------------------------------------------------------------------------
void set_max_dynamic_smem(const void* kernel, int bytes) {
  static std::mutex mu;
  static std::map<std::pair<int, const void*>, int> done;
  int dev = 0;
  SPS_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> g(mu);
  auto key = std::make_pair(dev, kernel);
  auto it = done.find(key);
  if (it != done.end() && it->second >= bytes) return;
  SPS_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  done[key] = bytes;
}

int occupancy_per_sm(const void* kernel, int threads, size_t smem) {
  static std::mutex mu;
  static std::map<std::tuple<int, const void*, int, size_t>, int> cache;
  int dev = 0;
  SPS_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> g(mu);
  auto key = std::make_tuple(dev, kernel, threads, smem);
  auto it = cache.find(key);
  if (it != cache.end()) return it->second;
  int per_sm = 0;
  SPS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem));
  cache[key] = per_sm;
  return per_sm;
}

// ---------------------------------------------------------------------------
// index tables: offsets of the parity-c fused indices (row-major order)
// ---------------------------------------------------------------------------
std::vector<int64_t> block_index(const std::vector<Par>& legs, const std::vector<int64_t>& strides,
                                 int c) {
  std::vector<int64_t> out;
  const int r = (int)legs.size();
  if (r == 0) {
    if (c == 0) out.push_back(0);
    return out;
  }
  int64_t total = 1;
  for (auto& p : legs) total *= (int64_t)p->size();
  if (total == 0) return out;
  out.reserve(total / 2 + 1);
  std::vector<int> idx(r, 0);
  int par = 0;
  int64_t off = 0;
  for (int k = 0; k < r; ++k) par ^= (*legs[k])[0];
  while (true) {
    if (par == c) out.push_back(off);
    int k = r - 1;
    while (k >= 0) {
      const auto& p = *legs[k];
      par ^= p[idx[k]];
      off -= (int64_t)idx[k] * strides[k];
      idx[k]++;
      if (idx[k] < (int)p.size()) {
        par ^= p[idx[k]];
        off += (int64_t)idx[k] * strides[k];
        break;
      }
      idx[k] = 0;
      par ^= p[0];
      --k;
    }
    if (k < 0) break;
  }
  return out;
}

// ---------------------------------------------------------------------------
// kernels: gather GEMM, permute, elementwise, reductions
// ---------------------------------------------------------------------------
struct GemmProb {
  const double* A;
  const double* B;
  double* C;
  const int64_t *ra, *ca, *rb, *cb, *rc, *cc;
  int M, N, K;
  int a_kfast, b_jfast;
  double* ws;   // split-K partial sums, S x M x N (row-major M x N per slice)
  int* cnt;     // split-K arrival counters, one per output tile
};

static constexpr int TM = 64, TN = 64, TK = 16, GT = 256;
static constexpr int GALD = TM + 8, GBLD = TN + 8;   // k-major tiles: a fragment load is 2 wavefronts

__device__ __forceinline__ void dmma_f64(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// C_c[i, j] = alpha sum_k A[ra[i] + ca[k]] B[rb[k] + cb[j]] for the parity
// block c = blockIdx.z / S, written through C's tables.  The gathered operands
// are staged global -> registers -> shared memory (double-buffered, so the
// indirect loads of the next k tile overlap the products of this one) and
// multiplied on the FP64 tensor cores (mma.m8n8k4.f64): 8 warps as 2 (M) x
// 4 (N), warp tile 32 x 16.  With S > 1 the contraction is split into S
// slices (blockIdx.z % S): every slice stores its partial tile, and the last
// CTA of a tile to arrive adds the S partials in slice order (deterministic)
// and resets the tile's counter.
__global__ void __launch_bounds__(GT) gemm_gather_kernel(const GemmProb* probs, double alpha, int S) {
  const GemmProb P = probs[blockIdx.z / S];
  const int kz = blockIdx.z % S;
  const int i0 = blockIdx.y * TM, j0 = blockIdx.x * TN;
  if (i0 >= P.M || j0 >= P.N) return;
  const int kchunk = (((P.K + S - 1) / S + TK - 1) / TK) * TK;
  const int kb = min(P.K, kz * kchunk), ke = min(P.K, kb + kchunk);
  __shared__ __align__(16) double As[2][TK * GALD];
  __shared__ __align__(16) double Bs[2][TK * GBLD];
  __shared__ int64_t rA[TM], cB[TN];
  const int t = threadIdx.x;
  if (t < TM) rA[t] = (i0 + t < P.M) ? P.ra[i0 + t] : 0;
  else if (t < TM + TN) cB[t - TM] = (j0 + t - TM < P.N) ? P.cb[j0 + t - TM] : 0;
  __syncthreads();
  double ra[4], rb[4];
  auto load = [&](int k0) {
    if (P.a_kfast) {
      const int kk = t % 16;
      const int64_t ck = (k0 + kk < ke) ? P.ca[k0 + kk] : -1;
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const int ii = t / 16 + 16 * r;
        ra[r] = (ck >= 0 && i0 + ii < P.M) ? P.A[rA[ii] + ck] : 0.0;
      }
    } else {
      const int ii = t % 64;
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const int kk = t / 64 + 4 * r;
        ra[r] = (k0 + kk < ke && i0 + ii < P.M) ? P.A[rA[ii] + P.ca[k0 + kk]] : 0.0;
      }
    }
    if (P.b_jfast) {
      const int jj = t % 64;
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const int kk = t / 64 + 4 * r;
        rb[r] = (k0 + kk < ke && j0 + jj < P.N) ? P.B[P.rb[k0 + kk] + cB[jj]] : 0.0;
      }
    } else {
      const int kk = t % 16;
      const int64_t rk = (k0 + kk < ke) ? P.rb[k0 + kk] : -1;
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const int jj = t / 16 + 16 * r;
        rb[r] = (rk >= 0 && j0 + jj < P.N) ? P.B[rk + cB[jj]] : 0.0;
      }
    }
  };
  auto store = [&](double* as, double* bs) {
    if (P.a_kfast) {
      const int kk = t % 16;
#pragma unroll
      for (int r = 0; r < 4; ++r) as[kk * GALD + t / 16 + 16 * r] = ra[r];
    } else {
      const int ii = t % 64;
#pragma unroll
      for (int r = 0; r < 4; ++r) as[(t / 64 + 4 * r) * GALD + ii] = ra[r];
    }
    if (P.b_jfast) {
      const int jj = t % 64;
#pragma unroll
      for (int r = 0; r < 4; ++r) bs[(t / 64 + 4 * r) * GBLD + jj] = rb[r];
    } else {
      const int kk = t % 16;
#pragma unroll
      for (int r = 0; r < 4; ++r) bs[kk * GBLD + t / 16 + 16 * r] = rb[r];
    }
  };
  const int warp = t >> 5, lane = t & 31, fr = lane >> 2, fc = lane & 3;
  const int wm = (warp & 1) * 32, wn = (warp >> 1) * 16;
  double acc[4][2][2];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;
  int buf = 0;
  load(kb);
  store(As[0], Bs[0]);
  __syncthreads();
  for (int k0 = kb; k0 < ke; k0 += TK) {
    const bool more = k0 + TK < ke;
    if (more) load(k0 + TK);
    const double* as = As[buf];
    const double* bs = Bs[buf];
#pragma unroll
    for (int ks = 0; ks < TK; ks += 4) {
      double fa[4], fb[2];
#pragma unroll
      for (int a = 0; a < 4; ++a) fa[a] = as[(ks + fc) * GALD + wm + a * 8 + fr];
#pragma unroll
      for (int b = 0; b < 2; ++b) fb[b] = bs[(ks + fc) * GBLD + wn + b * 8 + fr];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b) dmma_f64(acc[a][b][0], acc[a][b][1], fa[a], fb[b]);
    }
    if (more) {
      store(As[buf ^ 1], Bs[buf ^ 1]);
      buf ^= 1;
    }
    __syncthreads();
  }
  // accumulator fragment: row fr, columns 2 fc + {0, 1} of each 8 x 8 tile
  if (S == 1) {
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      const int i = i0 + wm + a * 8 + fr;
      if (i >= P.M) continue;
      const int64_t ro = P.rc[i];
#pragma unroll
      for (int b = 0; b < 2; ++b)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int j = j0 + wn + b * 8 + 2 * fc + e;
          if (j < P.N) P.C[ro + P.cc[j]] = alpha * acc[a][b][e];
        }
    }
    return;
  }
  double* part = P.ws + (size_t)kz * P.M * P.N;
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const int i = i0 + wm + a * 8 + fr;
    if (i >= P.M) continue;
#pragma unroll
    for (int b = 0; b < 2; ++b)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int j = j0 + wn + b * 8 + 2 * fc + e;
        if (j < P.N) part[(size_t)i * P.N + j] = acc[a][b][e];
      }
  }
  __threadfence();
  __syncthreads();
  __shared__ int last;
  int* cnt = P.cnt + blockIdx.y * gridDim.x + blockIdx.x;
  if (t == 0) last = (atomicAdd(cnt, 1) == S - 1);
  __syncthreads();
  if (!last) return;
  __threadfence();
  const int mi = min(TM, P.M - i0), nj = min(TN, P.N - j0);
  for (int e = t; e < mi * nj; e += GT) {
    const int i = i0 + e / nj, j = j0 + e % nj;
    double v = 0.0;
    for (int z = 0; z < S; ++z) v += __ldcg(&P.ws[(size_t)z * P.M * P.N + (size_t)i * P.N + j]);
    P.C[P.rc[i] + P.cc[j]] = alpha * v;
  }
  if (t == 0) *cnt = 0;
}

struct PermDesc {
  int rank;
  int64_t dims[16];
  int64_t istr[16];
};

__global__ void permute_kernel(const double* __restrict__ in, double* __restrict__ out, PermDesc d,
                               int64_t total) {
  for (int64_t o = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; o < total;
       o += (int64_t)gridDim.x * blockDim.x) {
    int64_t rem = o, off = 0;
    for (int k = d.rank - 1; k >= 0; --k) {
      int64_t q = rem / d.dims[k];
      off += (rem - q * d.dims[k]) * d.istr[k];
      rem = q;
    }
    out[o] = in[off];
  }
}

__global__ void scale_kernel(double* a, int64_t n, double s) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    a[i] *= s;
}

__global__ void axpby_kernel(const double* x, const double* y, double* z, int64_t n, double a,
                             double b) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    z[i] = a * x[i] + b * y[i];
}

static constexpr int RED_BLOCKS = 256;

// per-block partial sums of x*y (y == nullptr: x*x), then a final pass.
__global__ void dot_partial_kernel(const double* x, const double* y, int64_t n, double* partial) {
  __shared__ double red[32];
  double v = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    v += x[i] * (y ? y[i] : x[i]);
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
    partial[blockIdx.x] = s;
  }
}

__global__ void final_sum_kernel(const double* partial, int nb, double* out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double s = 0;
    for (int i = 0; i < nb; ++i) s += partial[i];
    *out = s;
  }
}

__global__ void sum_partial_kernel(const double* x, int64_t n, double* partial) {
  __shared__ double red[9];
  double v = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    v += x[i];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
    partial[blockIdx.x] = s;
  }
}

__global__ void finite_partial_kernel(const double* x, int64_t n, double* partial) {
  __shared__ int bad;
  if (threadIdx.x == 0) bad = 0;
  __syncthreads();
  int b = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    b |= !isfinite(x[i]);
  if (b) bad = 1;
  __syncthreads();
  if (threadIdx.x == 0) partial[blockIdx.x] = bad;
}

// A /= sqrt(*nrm2) when finite and nonzero; flags nonfinite.
__global__ void safe_scale_kernel(double* a, int64_t n, const double* nrm2, int* flag) {
  double s2 = *nrm2;
  double s = sqrt(s2);
  if (!isfinite(s)) {
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(flag, 1);
    return;
  }
  if (s == 0.0) return;
  double inv = 1.0 / s;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    a[i] *= inv;
}

__global__ void gather_kernel(const double* __restrict__ A, const int64_t* rt, const int64_t* ct,
                              int M, int N, double* dst, int ld, int transpose) {
  int64_t total = (int64_t)M * N;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    int i, j;
    if (transpose) { j = (int)(e % N); i = (int)(e / N); }
    else { i = (int)(e % M); j = (int)(e / M); }
    double v = A[rt[i] + ct[j]];
    if (transpose) dst[j + (int64_t)i * ld] = v;
    else dst[i + (int64_t)j * ld] = v;
  }
}

__global__ void scatter_kernel(double* __restrict__ A, const int64_t* rt, const int64_t* ct, int M,
                               int N, const double* src, int ld, int transpose) {
  int64_t total = (int64_t)M * N;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    int i, j;
    if (transpose) { j = (int)(e % N); i = (int)(e / N); }
    else { i = (int)(e % M); j = (int)(e / M); }
    A[rt[i] + ct[j]] = transpose ? src[j + (int64_t)i * ld] : src[i + (int64_t)j * ld];
  }
}

__global__ void scale_leg_kernel(const double* in, double* out, const double* d, int64_t total,
                                 int64_t stride, int64_t dim) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x)
    out[i] = in[i] * d[(i / stride) % dim];
}

static int grid_for(int64_t n, int threads = 256) {
  int64_t g = (n + threads - 1) / threads;
  return (int)std::max<int64_t>(1, std::min<int64_t>(g, 148 * 16));
}

// ---------------------------------------------------------------------------
// views / permutes
// ---------------------------------------------------------------------------
Tensor perm_view(const Tensor& A, const std::vector<int>& order) {
  Tensor t;
  t.buf = A.buf;
  t.offset = A.offset;
  for (int k : order) {
    t.legs.push_back(A.legs[k]);
    t.dims.push_back(A.dims[k]);
    t.strides.push_back(A.strides[k]);
  }
  return t;
}

Tensor contiguous(Engine& E, const Tensor& A) {
  if (A.contiguous()) return A;
  Tensor out = E.empty(A.legs);
  int64_t n = out.size();
  if (n == 0) return out;
  PermDesc d;
  d.rank = A.rank();
  if (d.rank > 16) throw Error(SPS_ERR_ARGUMENT, "rank > 16");
  for (int k = 0; k < d.rank; ++k) {
    d.dims[k] = A.dims[k];
    d.istr[k] = A.strides[k];
  }
  int tk = E.tic("permute");
  permute_kernel<<<grid_for(n), 256, 0, E.stream>>>(A.ptr(), out.ptr(), d, n);
  E.toc(tk, 0, 16.0 * n);
  SPS_CUDA(cudaGetLastError());
  E.launches++;
  return out;
}

Tensor perm(Engine& E, const Tensor& A, const std::vector<int>& order) {
  return contiguous(E, perm_view(A, order));
}

Tensor clone(Engine& E, const Tensor& A) {
  Tensor c = contiguous(E, A);
  if (c.buf != A.buf) return c;
  Tensor out = E.empty(A.legs);
  if (out.size())
    SPS_CUDA(cudaMemcpyAsync(out.ptr(), c.ptr(), out.size() * sizeof(double),
                             cudaMemcpyDeviceToDevice, E.stream));
  return out;
}

Tensor fuse(Engine& E, const Tensor& A0, int first, int count) {
  if (count == 1) return A0;
  bool ok = true;
  for (int k = first; k < first + count - 1; ++k)
    if (A0.strides[k] != A0.strides[k + 1] * A0.dims[k + 1]) ok = false;
  Tensor A = ok ? A0 : contiguous(E, A0);
  Tensor t;
  t.buf = A.buf;
  t.offset = A.offset;
  std::vector<Par> parts(A.legs.begin() + first, A.legs.begin() + first + count);
  int64_t d = 1;
  for (int k = first; k < first + count; ++k) d *= A.dims[k];
  for (int k = 0; k < A.rank(); ++k) {
    if (k == first) {
      t.legs.push_back(fused_par(parts));
      t.dims.push_back(d);
      t.strides.push_back(A.strides[first + count - 1]);
      k = first + count - 1;
      continue;
    }
    t.legs.push_back(A.legs[k]);
    t.dims.push_back(A.dims[k]);
    t.strides.push_back(A.strides[k]);
  }
  return t;
}

Tensor split(Engine& E, const Tensor& A, int axis, const std::vector<Par>& parts) {
  (void)E;
  Tensor t;
  t.buf = A.buf;
  t.offset = A.offset;
  for (int k = 0; k < A.rank(); ++k) {
    if (k == axis) {
      int64_t s = A.strides[k];
      std::vector<int64_t> ps(parts.size());
      for (int q = (int)parts.size() - 1; q >= 0; --q) {
        ps[q] = s;
        s *= (int64_t)parts[q]->size();
      }
      for (size_t q = 0; q < parts.size(); ++q) {
        t.legs.push_back(parts[q]);
        t.dims.push_back((int64_t)parts[q]->size());
        t.strides.push_back(ps[q]);
      }
      continue;
    }
    t.legs.push_back(A.legs[k]);
    t.dims.push_back(A.dims[k]);
    t.strides.push_back(A.strides[k]);
  }
  return t;
}

Tensor slice_leg(Engine& E, const Tensor& A, int axis, int index, Par newpar) {
  Tensor t = A;
  t.offset += (int64_t)index * A.strides[axis];
  t.dims[axis] = 1;
  t.legs[axis] = newpar;
  return contiguous(E, t);
}

// ---------------------------------------------------------------------------
// elementwise and reductions
// ---------------------------------------------------------------------------
void scale_inplace(Engine& E, Tensor& A, double s) {
  A = contiguous(E, A);
  int64_t n = A.size();
  if (!n) return;
  scale_kernel<<<grid_for(n), 256, 0, E.stream>>>(A.ptr(), n, s);
  SPS_CUDA(cudaGetLastError());
  E.launches++;
}

static void reduce_dot(Engine& E, const double* x, const double* y, int64_t n, double* out) {
  Buf part = E.alloc(RED_BLOCKS * sizeof(double));
  int nb = (int)std::max<int64_t>(1, std::min<int64_t>(RED_BLOCKS, (n + 255) / 256));
  dot_partial_kernel<<<nb, 256, 0, E.stream>>>(x, y, n, (double*)part->ptr);
  final_sum_kernel<<<1, 32, 0, E.stream>>>((double*)part->ptr, nb, out);
  SPS_CUDA(cudaGetLastError());
  E.launches += 2;
}

void norm2_to(Engine& E, const Tensor& A0, int slot) {
  Tensor A = contiguous(E, A0);
  reduce_dot(E, A.ptr(), nullptr, A.size(), E.dscal + slot);
}

void dot_to(Engine& E, const Tensor& A0, const Tensor& B0, int slot) {
  Tensor A = contiguous(E, A0), B = contiguous(E, B0);
  if (A.size() != B.size()) throw Error(SPS_ERR_ARGUMENT, "dot: size mismatch");
  reduce_dot(E, A.ptr(), B.ptr(), A.size(), E.dscal + slot);
}

static double read_slot(Engine& E, int slot) {
  SPS_CUDA(cudaMemcpyAsync(E.hscal + slot, E.dscal + slot, sizeof(double), cudaMemcpyDeviceToHost,
                           E.stream));
  E.sync();
  return E.hscal[slot];
}

double norm(Engine& E, const Tensor& A) {
  norm2_to(E, A, 0);
  return std::sqrt(read_slot(E, 0));
}

double dot(Engine& E, const Tensor& A, const Tensor& B) {
  dot_to(E, A, B, 0);
  return read_slot(E, 0);
}

double sum_all(Engine& E, const Tensor& A0) {
  Tensor A = contiguous(E, A0);
  Buf part = E.alloc(RED_BLOCKS * sizeof(double));
  int64_t n = A.size();
  int nb = (int)std::max<int64_t>(1, std::min<int64_t>(RED_BLOCKS, (n + 255) / 256));
  sum_partial_kernel<<<nb, 256, 0, E.stream>>>(A.ptr(), n, (double*)part->ptr);
  final_sum_kernel<<<1, 32, 0, E.stream>>>((double*)part->ptr, nb, E.dscal);
  E.launches += 2;
  return read_slot(E, 0);
}

bool all_finite(Engine& E, const Tensor& A0) {
  Tensor A = contiguous(E, A0);
  Buf part = E.alloc(RED_BLOCKS * sizeof(double));
  int64_t n = A.size();
  int nb = (int)std::max<int64_t>(1, std::min<int64_t>(RED_BLOCKS, (n + 255) / 256));
  finite_partial_kernel<<<nb, 256, 0, E.stream>>>(A.ptr(), n, (double*)part->ptr);
  sum_partial_kernel<<<1, 256, 0, E.stream>>>((double*)part->ptr, nb, E.dscal + 1);
  E.launches += 2;
  return read_slot(E, 1) == 0.0;
}

void safe_scale_inplace(Engine& E, Tensor& A) {
  A = contiguous(E, A);
  norm2_to(E, A, 2);
  int64_t n = A.size();
  safe_scale_kernel<<<grid_for(n), 256, 0, E.stream>>>(A.ptr(), n, E.dscal + 2, E.dflag);
  SPS_CUDA(cudaGetLastError());
  E.launches++;
}

Tensor axpby(Engine& E, double a, const Tensor& X0, double b, const Tensor& Y0) {
  Tensor X = contiguous(E, X0), Y = contiguous(E, Y0);
  if (X.size() != Y.size()) throw Error(SPS_ERR_ARGUMENT, "axpby: size mismatch");
  Tensor Z = E.empty(X.legs);
  int64_t n = Z.size();
  if (n) {
    axpby_kernel<<<grid_for(n), 256, 0, E.stream>>>(X.ptr(), Y.ptr(), Z.ptr(), n, a, b);
    SPS_CUDA(cudaGetLastError());
    E.launches++;
  }
  return Z;
}

Tensor scale_leg(Engine& E, const Tensor& A0, int axis, const std::vector<double>& d) {
  Tensor A = contiguous(E, A0);
  Tensor out = E.empty(A.legs);
  Buf kd = E.alloc(std::max<size_t>(d.size(), 1) * sizeof(double));
  E.stage(d.data(), d.size() * sizeof(double), kd->ptr);
  int64_t n = A.size();
  if (n) {
    scale_leg_kernel<<<grid_for(n), 256, 0, E.stream>>>(A.ptr(), out.ptr(), (double*)kd->ptr, n,
                                                         A.strides[axis], A.dims[axis]);
    SPS_CUDA(cudaGetLastError());
    E.launches++;
  }
  return out;
}

void gather_block(Engine& E, const Tensor& A, const int64_t* rt, const int64_t* ct, int M, int N,
                  double* dst, int ld, bool transpose) {
  int64_t n = (int64_t)M * N;
  if (!n) return;
  int tk = E.tic("block_gather");
  gather_kernel<<<grid_for(n), 256, 0, E.stream>>>(A.ptr(), rt, ct, M, N, dst, ld, transpose);
  E.toc(tk, 0, 16.0 * n);
  SPS_CUDA(cudaGetLastError());
  E.launches++;
}

void scatter_block(Engine& E, Tensor& A, const int64_t* rt, const int64_t* ct, int M, int N,
                   const double* src, int ld, bool transpose) {
  int64_t n = (int64_t)M * N;
  if (!n) return;
  int tk = E.tic("block_scatter");
  scatter_kernel<<<grid_for(n), 256, 0, E.stream>>>(A.ptr(), rt, ct, M, N, src, ld, transpose);
  E.toc(tk, 0, 16.0 * n);
  SPS_CUDA(cudaGetLastError());
  E.launches++;
}

// ---------------------------------------------------------------------------
// einsum (two operands)
// ---------------------------------------------------------------------------
static bool same_par(const Par& a, const Par& b) { return a == b || *a == *b; }

Tensor ein(Engine& E, const std::string& spec, const Tensor& A, const Tensor& B, double alpha) {
  HostTimer ht(E, "host.ein");
  auto arrow = spec.find("->");
  auto comma = spec.find(',');
  if (arrow == std::string::npos || comma == std::string::npos || comma > arrow)
    throw Error(SPS_ERR_ARGUMENT, "ein: bad spec " + spec);
  std::string la = spec.substr(0, comma), lb = spec.substr(comma + 1, arrow - comma - 1),
              lo = spec.substr(arrow + 2);
  if ((int)la.size() != A.rank() || (int)lb.size() != B.rank())
    throw Error(SPS_ERR_ARGUMENT, "ein: rank mismatch in " + spec);
  std::vector<int> fa, fb, ka, kb;   // free A, free B, contracted (A idx, B idx)
  for (int i = 0; i < (int)la.size(); ++i) {
    char ch = la[i];
    auto pb = lb.find(ch);
    auto po = lo.find(ch);
    if (pb != std::string::npos && po == std::string::npos) {
      ka.push_back(i);
      kb.push_back((int)pb);
      if (A.dims[i] != B.dims[pb] || !same_par(A.legs[i], B.legs[pb]))
        throw Error(SPS_ERR_ARGUMENT, std::string("ein: leg mismatch on '") + ch + "' in " + spec);
    } else if (po != std::string::npos && pb == std::string::npos) {
      fa.push_back(i);
    } else {
      throw Error(SPS_ERR_ARGUMENT, "ein: unsupported label use in " + spec);
    }
  }
  for (int j = 0; j < (int)lb.size(); ++j) {
    char ch = lb[j];
    if (la.find(ch) != std::string::npos) continue;
    if (lo.find(ch) == std::string::npos) throw Error(SPS_ERR_ARGUMENT, "ein: trace in " + spec);
    fb.push_back(j);
  }
  if (fa.size() + fb.size() != lo.size()) throw Error(SPS_ERR_ARGUMENT, "ein: output mismatch " + spec);
  std::vector<Par> olegs;
  for (char ch : lo) {
    auto p = la.find(ch);
    if (p != std::string::npos) olegs.push_back(A.legs[p]);
    else olegs.push_back(B.legs[lb.find(ch)]);
  }
  Tensor C = E.zeros(olegs);
  if (C.size() == 0 || A.size() == 0 || B.size() == 0) return C;
  auto pick = [](const Tensor& T, const std::vector<int>& ix, std::vector<Par>& L,
                 std::vector<int64_t>& S) {
    for (int k : ix) {
      L.push_back(T.legs[k]);
      S.push_back(T.strides[k]);
    }
  };
  std::vector<Par> LfA, LfB, Lk;
  std::vector<int64_t> SfA, SfB, SkA, SkB, ScA, ScB;
  pick(A, fa, LfA, SfA);
  pick(B, fb, LfB, SfB);
  {
    std::vector<Par> dummy;
    pick(A, ka, Lk, SkA);
    pick(B, kb, dummy, SkB);
  }
  for (int k : fa) ScA.push_back(C.strides[lo.find(la[k])]);
  for (int k : fb) ScB.push_back(C.strides[lo.find(lb[k])]);
  // plan: the index tables of both parity blocks, cached per layout
  std::string key = spec;
  auto add_layout = [&key](const Tensor& T) {   // binary: rank, then (dim, stride, parity hash) per leg
    auto put = [&key](uint64_t v) { key.append(reinterpret_cast<const char*>(&v), sizeof v); };
    put((uint64_t)T.rank());
    for (int k = 0; k < T.rank(); ++k) {
      put((uint64_t)T.dims[k]);
      put((uint64_t)T.strides[k]);
      uint64_t h = 1469598103934665603ull;   // FNV-1a of the leg's parities
      for (uint8_t v : *T.legs[k]) h = (h ^ v) * 1099511628211ull;
      put(h);
    }
  };
  add_layout(A);
  add_layout(B);
  auto it = E.ein_plans.find(key);
  if (it == E.ein_plans.end()) {
    std::vector<Engine::EinBlock> blocks;
    size_t bytes = 0;
    for (int c = 0; c < 2; ++c) {
      auto ra = block_index(LfA, SfA, c), rc = block_index(LfA, ScA, c);
      auto ca = block_index(Lk, SkA, c), rb = block_index(Lk, SkB, c);
      auto cb = block_index(LfB, SfB, c), cc = block_index(LfB, ScB, c);
      if (ra.empty() || cb.empty() || ca.empty()) continue;
      Engine::EinBlock bl;
      E.upload_i64(ra, bl.ra);
      E.upload_i64(ca, bl.ca);
      E.upload_i64(rb, bl.rb);
      E.upload_i64(cb, bl.cb);
      E.upload_i64(rc, bl.rc);
      E.upload_i64(cc, bl.cc);
      bl.M = (int)ra.size();
      bl.N = (int)cb.size();
      bl.K = (int)ca.size();
      bl.a_kfast = (ca.size() > 1 && ca[1] - ca[0] == 1) ? 1 : 0;
      bl.b_jfast = (cb.size() > 1 && cb[1] - cb[0] == 1) ? 1 : (rb.size() > 1 && rb[1] - rb[0] == 1 ? 0 : 1);
      bytes += 8 * (ra.size() + ca.size() + rb.size() + cb.size() + rc.size() + cc.size());
      blocks.push_back(std::move(bl));
    }
    if (E.ein_plan_bytes + bytes > ((size_t)256 << 20)) {   // bounded: start over when full
      E.ein_plans.clear();
      E.ein_plan_bytes = 0;
    }
    E.ein_plan_bytes += bytes;
    it = E.ein_plans.emplace(key, std::move(blocks)).first;
  }
  std::vector<GemmProb> probs;
  int maxM = 0, maxN = 0;
  for (const auto& bl : it->second) {
    GemmProb P;
    P.ws = nullptr;
    P.cnt = nullptr;
    P.A = A.ptr();
    P.B = B.ptr();
    P.C = C.ptr();
    P.ra = (const int64_t*)bl.ra->ptr;
    P.ca = (const int64_t*)bl.ca->ptr;
    P.rb = (const int64_t*)bl.rb->ptr;
    P.cb = (const int64_t*)bl.cb->ptr;
    P.rc = (const int64_t*)bl.rc->ptr;
    P.cc = (const int64_t*)bl.cc->ptr;
    P.M = bl.M;
    P.N = bl.N;
    P.K = bl.K;
    P.a_kfast = bl.a_kfast;
    P.b_jfast = bl.b_jfast;
    maxM = std::max(maxM, P.M);
    maxN = std::max(maxN, P.N);
    E.flops += 2.0 * P.M * P.N * P.K;
    probs.push_back(P);
  }
  if (probs.empty()) return C;
  if (E.precision > 0) {
    // low-precision mode: large blocks on the tcgen05 GEMM, the rest stays FP64
    std::vector<GemmProb> small;
    for (auto& P : probs) {
      if (tc::worth(P.M, P.N, P.K)) {
        tc::gemm_block(E, E.precision, P.A, P.ra, P.ca, P.a_kfast, P.B, P.rb, P.cb, P.b_jfast, P.C, P.rc, P.cc, P.M,
                       P.N, P.K, alpha);
        E.flops -= 2.0 * P.M * P.N * P.K;   // counted once, by gemm_block
      } else {
        small.push_back(P);
      }
    }
    if (small.empty()) return C;
    if (small.size() != probs.size()) {
      probs = small;
      maxM = maxN = 0;
      for (auto& P : probs) {
        maxM = std::max(maxM, P.M);
        maxN = std::max(maxN, P.N);
      }
    }
  }
  // split the contraction when the output tiles alone leave most SMs idle
  // and every slice keeps at least 4 k-steps
  const int tiles = ((maxN + TN - 1) / TN) * ((maxM + TM - 1) / TM);
  const int nprob = (int)probs.size();
  int maxK = 0;
  for (auto& P : probs) maxK = std::max(maxK, P.K);
  int S = 1;
  if (maxK >= 8 * TK && tiles * nprob < E.num_sms)
    S = std::min((maxK + 4 * TK - 1) / (4 * TK), (E.num_sms + tiles * nprob - 1) / (tiles * nprob));
  // candidate slice counts for the autotuner: the heuristic's, half and double
  // it, and no split; every slice keeps at least two k-steps
  std::vector<int> cands;
  int Smax = S;
  if (E.autotune && maxK >= 4 * TK) {
    const int cap = std::max(1, maxK / (2 * TK));
    for (int c : {1, std::max(1, S / 2), S, 2 * S})
      if (c <= cap && std::find(cands.begin(), cands.end(), c) == cands.end()) cands.push_back(c);
    for (int c : cands) Smax = std::max(Smax, c);
  }
  Buf ws;
  if (Smax > 1) {
    size_t wsz = 0;
    for (auto& P : probs) wsz += (size_t)Smax * P.M * P.N;
    ws = E.alloc(wsz * sizeof(double));
    const size_t slots = (size_t)tiles * nprob;
    if (slots > E.gg_counter_slots) {   // zeroed once; the kernels leave them zero
      E.gg_counter_slots = std::max<size_t>(slots, 4096);
      E.gg_counters = E.alloc(E.gg_counter_slots * sizeof(int));
      SPS_CUDA(cudaMemsetAsync(E.gg_counters->ptr, 0, E.gg_counter_slots * sizeof(int), E.stream));
    }
    size_t off = 0;
    for (int p = 0; p < nprob; ++p) {
      probs[p].ws = (double*)ws->ptr + off;
      off += (size_t)Smax * probs[p].M * probs[p].N;
      probs[p].cnt = (int*)E.gg_counters->ptr + (size_t)p * tiles;
    }
  }
  Buf kp = E.alloc(probs.size() * sizeof(GemmProb));
  E.stage(probs.data(), probs.size() * sizeof(GemmProb), kp->ptr);
  if (cands.size() > 1) {
    const std::string key = tune::key(E, "gemm_gather.split", {maxM, maxN, maxK, nprob});
    S = tune::pick(E, key, cands, [&](int c) {
      dim3 g((maxN + TN - 1) / TN, (maxM + TM - 1) / TM, (unsigned)(probs.size() * c));
      gemm_gather_kernel<<<g, GT, 0, E.stream>>>((const GemmProb*)kp->ptr, alpha, c);
      SPS_CUDA(cudaGetLastError());
    });
  }
  dim3 grid((maxN + TN - 1) / TN, (maxM + TM - 1) / TM, (unsigned)(probs.size() * S));
  double fl = 0, by = 0;
  for (auto& P : probs) {
    fl += 2.0 * P.M * P.N * (double)P.K;
    by += 8.0 * ((double)P.M * P.K + (double)P.K * P.N + (double)P.M * P.N);
  }
  int tk = E.tic("gemm_gather");
  int tshape = -1;
  if (E.profile > 1) {
    std::string nm = "gemm_gather " + std::to_string(maxM) + "x" + std::to_string(maxN) + "x" +
                     std::to_string(probs[0].K) + " p" + std::to_string(nprob) + " s" + std::to_string(S) + " g" +
                     std::to_string(grid.x * grid.y * grid.z);
    tshape = E.tic(nm.c_str());
  }
  gemm_gather_kernel<<<grid, GT, 0, E.stream>>>((const GemmProb*)kp->ptr, alpha, S);
  E.toc(tk, fl, by);
  E.toc(tshape, fl, by);
  SPS_CUDA(cudaGetLastError());
  E.launches++;
  return C;
}

// ---------------------------------------------------------------------------
// factorizations
// ---------------------------------------------------------------------------
namespace {
struct BlockTables {
  std::vector<Par> rp, cp;
  std::vector<int64_t> rs, cs;
  std::vector<int64_t> rt[2], ct[2];
};

BlockTables tables_of(const Tensor& A, const std::vector<int>& rows, const std::vector<int>& cols) {
  BlockTables t;
  for (int k : rows) {
    t.rp.push_back(A.legs[k]);
    t.rs.push_back(A.strides[k]);
  }
  for (int k : cols) {
    t.cp.push_back(A.legs[k]);
    t.cs.push_back(A.strides[k]);
  }
  for (int c = 0; c < 2; ++c) {
    t.rt[c] = block_index(t.rp, t.rs, c);
    t.ct[c] = block_index(t.cp, t.cs, c);
  }
  return t;
}

std::vector<int64_t> leg_offsets(int c, int k0, int k1, int64_t stride) {
  std::vector<int64_t> v;
  int base = c == 0 ? 0 : k0;
  int k = c == 0 ? k0 : k1;
  for (int i = 0; i < k; ++i) v.push_back((int64_t)(base + i) * stride);
  return v;
}

std::vector<int64_t> tensor_rows(const Tensor& T, int first, int count, int c) {
  std::vector<Par> L(T.legs.begin() + first, T.legs.begin() + first + count);
  std::vector<int64_t> S(T.strides.begin() + first, T.strides.begin() + first + count);
  return block_index(L, S, c);
}
}  // namespace

namespace la {
bool qr_is_big(int m, int n) { return m >= n && (double)m * n * n >= 4.0e6; }
bool svd_is_big(int m, int n) { return m >= n && n >= 160; }
}  // namespace la

// small blocks share one batched single-CTA launch; large ones use the multi-CTA path
static void run_qr(Engine& E, const std::vector<la::MatDesc>& ds) {
  std::vector<la::MatDesc> small;
  for (auto& d : ds) {
    if (la::qr_is_big(d.m, d.n)) la::qr_big(E, d.a, d.m, d.n, d.lda, d.q, d.ldq, d.r, d.ldr);
    else small.push_back(d);
  }
  la::qr_batched(E, small);
}

static void run_svd(Engine& E, const std::vector<la::MatDesc>& ds) {
  std::vector<la::MatDesc> small, big;
  for (auto& d : ds) (la::svd_is_big(d.m, d.n) ? big : small).push_back(d);
  la::svd_batched(E, small);
  la::svd_big(E, big);
}

QRres qr(Engine& E, const Tensor& A, const std::vector<int>& rows, const std::vector<int>& cols) {
  BlockTables bt = tables_of(A, rows, cols);
  int m[2], n[2], k[2];
  for (int c = 0; c < 2; ++c) {
    m[c] = (int)bt.rt[c].size();
    n[c] = (int)bt.ct[c].size();
    k[c] = std::min(m[c], n[c]);
  }
  Par nl = make_par(k[0], k[1]);
  std::vector<Par> ql = bt.rp;
  ql.push_back(nl);
  std::vector<Par> rl{nl};
  rl.insert(rl.end(), bt.cp.begin(), bt.cp.end());
  QRres res{E.zeros(ql), E.zeros(rl)};
  std::vector<la::MatDesc> ds;
  std::vector<Buf> keep;
  for (int c = 0; c < 2; ++c) {
    if (k[c] == 0) continue;
    Buf ba = E.alloc(sizeof(double) * ((size_t)m[c] * n[c] + (size_t)m[c] * k[c] + (size_t)k[c] * n[c] + k[c]));
    double* a = (double*)ba->ptr;
    double* q = a + (size_t)m[c] * n[c];
    double* r = q + (size_t)m[c] * k[c];
    double* s = r + (size_t)k[c] * n[c];
    Buf t1, t2;
    int64_t* rt = E.upload_i64(bt.rt[c], t1);
    int64_t* ct = E.upload_i64(bt.ct[c], t2);
    gather_block(E, A, rt, ct, m[c], n[c], a, m[c], false);
    ds.push_back({a, q, r, s, m[c], n[c], m[c], m[c], k[c]});
    keep.insert(keep.end(), {ba, t1, t2});
  }
  run_qr(E, ds);
  int di = 0;
  for (int c = 0; c < 2; ++c) {
    if (k[c] == 0) continue;
    auto& d = ds[di++];
    Buf t1, t2, t3, t4;
    int nr = (int)rows.size();
    auto qrow = tensor_rows(res.Q, 0, nr, c);
    auto qcol = leg_offsets(c, k[0], k[1], res.Q.strides[nr]);
    scatter_block(E, res.Q, E.upload_i64(qrow, t1), E.upload_i64(qcol, t2), m[c], k[c], d.q, m[c], false);
    auto rrow = leg_offsets(c, k[0], k[1], res.R.strides[0]);
    auto rcol = tensor_rows(res.R, 1, (int)cols.size(), c);
    scatter_block(E, res.R, E.upload_i64(rrow, t3), E.upload_i64(rcol, t4), k[c], n[c], d.r, k[c], false);
    keep.insert(keep.end(), {t1, t2, t3, t4});
  }
  return res;
}

LQres lq(Engine& E, const Tensor& A, const std::vector<int>& rows, const std::vector<int>& cols) {
  BlockTables bt = tables_of(A, rows, cols);
  int m[2], n[2], k[2];
  for (int c = 0; c < 2; ++c) {
    m[c] = (int)bt.rt[c].size();
    n[c] = (int)bt.ct[c].size();
    k[c] = std::min(m[c], n[c]);
  }
  Par nl = make_par(k[0], k[1]);
  std::vector<Par> ll = bt.rp;
  ll.push_back(nl);
  std::vector<Par> qlg{nl};
  qlg.insert(qlg.end(), bt.cp.begin(), bt.cp.end());
  LQres res{E.zeros(ll), E.zeros(qlg)};
  std::vector<la::MatDesc> ds;
  std::vector<Buf> keep;
  for (int c = 0; c < 2; ++c) {
    if (k[c] == 0) continue;
    // QR of the transpose: a = M^T (n x m)
    Buf ba = E.alloc(sizeof(double) * ((size_t)m[c] * n[c] + (size_t)n[c] * k[c] + (size_t)k[c] * m[c] + k[c]));
    double* a = (double*)ba->ptr;
    double* q = a + (size_t)m[c] * n[c];
    double* r = q + (size_t)n[c] * k[c];
    double* s = r + (size_t)k[c] * m[c];
    Buf t1, t2;
    gather_block(E, A, E.upload_i64(bt.rt[c], t1), E.upload_i64(bt.ct[c], t2), m[c], n[c], a, n[c], true);
    ds.push_back({a, q, r, s, n[c], m[c], n[c], n[c], k[c]});
    keep.insert(keep.end(), {ba, t1, t2});
  }
  run_qr(E, ds);
  int di = 0;
  for (int c = 0; c < 2; ++c) {
    if (k[c] == 0) continue;
    auto& d = ds[di++];
    Buf t1, t2, t3, t4;
    int nr = (int)rows.size();
    // L (m x k) = R'^T, R' is k x m col-major (ld k)
    auto lrow = tensor_rows(res.L, 0, nr, c);
    auto lcol = leg_offsets(c, k[0], k[1], res.L.strides[nr]);
    scatter_block(E, res.L, E.upload_i64(lrow, t1), E.upload_i64(lcol, t2), m[c], k[c], d.r, k[c], true);
    // Q (k x n) = Q'^T, Q' is n x k col-major (ld n)
    auto qrow = leg_offsets(c, k[0], k[1], res.Q.strides[0]);
    auto qcol = tensor_rows(res.Q, 1, (int)cols.size(), c);
    scatter_block(E, res.Q, E.upload_i64(qrow, t3), E.upload_i64(qcol, t4), k[c], n[c], d.q, n[c], true);
    keep.insert(keep.end(), {t1, t2, t3, t4});
  }
  return res;
}

static std::vector<char> select_truncation(const std::vector<double> s[2], const Trunc& tr,
                                           std::vector<char> keep[2]) {
  for (int c = 0; c < 2; ++c) keep[c].assign(s[c].size(), 1);
  if (tr.chi >= 0) {
    struct E3 { double v; int c, i; };
    std::vector<E3> all;
    for (int c = 0; c < 2; ++c)
      for (int i = 0; i < (int)s[c].size(); ++i) all.push_back({s[c][i], c, i});
    std::stable_sort(all.begin(), all.end(), [](const E3& a, const E3& b) {
      if (a.v != b.v) return a.v > b.v;
      if (a.c != b.c) return a.c < b.c;
      return a.i < b.i;
    });
    std::vector<char> sel[2];
    for (int c = 0; c < 2; ++c) sel[c].assign(s[c].size(), 0);
    for (int q = 0; q < (int)all.size() && q < tr.chi; ++q) sel[all[q].c][all[q].i] = 1;
    for (int c = 0; c < 2; ++c)
      for (size_t i = 0; i < s[c].size(); ++i) keep[c][i] &= sel[c][i];
  }
  for (int c = 0; c < 2; ++c) {
    if (tr.space[0] >= 0)
      for (size_t i = 0; i < s[c].size(); ++i)
        if ((int)i >= tr.space[c]) keep[c][i] = 0;
    if (tr.atol >= 0)
      for (size_t i = 0; i < s[c].size(); ++i)
        if (!(s[c][i] > tr.atol)) keep[c][i] = 0;
  }
  return {};
}

void truncation_keep(const std::vector<double> s[2], const Trunc& tr, std::vector<char> keep[2]) {
  select_truncation(s, tr, keep);
}

// Device value arrays to the host after one synchronisation: through the
// pinned scalar scratch when they fit, else by plain copies after the sync.
// The device flag is checked (and raised as an error) on the way.
static std::vector<std::vector<double>> read_values(Engine& E, const std::vector<std::pair<const double*, int>>& src,
                                                    const char* where) {
  size_t total = 0;
  for (auto& x : src) total += (size_t)x.second;
  std::vector<std::vector<double>> out(src.size());
  if (total <= (size_t)Engine::NSCAL) {
    size_t off = 0;
    for (auto& x : src) {
      if (x.second > 0)
        SPS_CUDA(cudaMemcpyAsync(E.hscal + off, x.first, sizeof(double) * x.second, cudaMemcpyDeviceToHost,
                                 E.stream));
      off += x.second;
    }
    E.sync();
    E.check_flag(where);
    off = 0;
    for (size_t i = 0; i < src.size(); ++i) {
      out[i].assign(E.hscal + off, E.hscal + off + src[i].second);
      off += src[i].second;
    }
  } else {
    E.sync();
    E.check_flag(where);
    for (size_t i = 0; i < src.size(); ++i) {
      out[i].resize(src[i].second);
      if (src[i].second > 0)
        SPS_CUDA(cudaMemcpy(out[i].data(), src[i].first, sizeof(double) * src[i].second, cudaMemcpyDeviceToHost));
    }
  }
  return out;
}

SVDres svd(Engine& E, const Tensor& A, const std::vector<int>& rows, const std::vector<int>& cols,
           const Trunc& tr, bool want_entropy) {
  BlockTables bt = tables_of(A, rows, cols);
  int m[2], n[2], k[2];
  bool tall[2];
  for (int c = 0; c < 2; ++c) {
    m[c] = (int)bt.rt[c].size();
    n[c] = (int)bt.ct[c].size();
    k[c] = std::min(m[c], n[c]);
    tall[c] = m[c] >= n[c];
  }
  std::vector<la::MatDesc> ds;
  std::vector<Buf> keep;
  int dmap[2] = {-1, -1};
  for (int c = 0; c < 2; ++c) {
    if (k[c] == 0) continue;
    int mm = tall[c] ? m[c] : n[c], nn = tall[c] ? n[c] : m[c];
    Buf ba = E.alloc(sizeof(double) * ((size_t)mm * nn * 2 + (size_t)nn * nn + nn));
    double* a = (double*)ba->ptr;
    double* q = a + (size_t)mm * nn;
    double* r = q + (size_t)mm * nn;
    double* s = r + (size_t)nn * nn;
    Buf t1, t2;
    gather_block(E, A, E.upload_i64(bt.rt[c], t1), E.upload_i64(bt.ct[c], t2), m[c], n[c], a,
                 tall[c] ? m[c] : n[c], !tall[c]);
    dmap[c] = (int)ds.size();
    ds.push_back({a, q, r, s, mm, nn, mm, mm, nn});
    keep.insert(keep.end(), {ba, t1, t2});
  }
  run_svd(E, ds);
  SVDres res;
  std::vector<double> sv[2];
  // copy singular values back
  {
    std::vector<std::pair<const double*, int>> src;
    for (int c = 0; c < 2; ++c) src.push_back({dmap[c] < 0 ? nullptr : ds[dmap[c]].s, dmap[c] < 0 ? 0 : k[c]});
    auto v = read_values(E, src, "svd");
    for (int c = 0; c < 2; ++c) sv[c] = std::move(v[c]);
  }
  double tot2 = 0;
  for (int c = 0; c < 2; ++c)
    for (double x : sv[c]) tot2 += x * x;
  res.norm = std::sqrt(tot2);
  if (want_entropy) {
    double scale = res.norm;
    if (scale == 0) res.entropy = NAN;
    else {
      double ent = 0;
      for (int c = 0; c < 2; ++c)
        for (double x : sv[c]) {
          double p = (x / scale) * (x / scale);
          if (p != 0) ent -= p * std::log(p);
        }
      res.entropy = std::max(0.0, ent);
    }
  }
  std::vector<char> kp[2];
  select_truncation(sv, tr, kp);
  int kk[2] = {0, 0};
  double disc = 0;
  for (int c = 0; c < 2; ++c) {
    for (size_t i = 0; i < sv[c].size(); ++i) {
      if (kp[c][i]) {
        if ((int)i != kk[c]) throw Error(SPS_ERR_NUMERIC, "svd: non-prefix truncation");
        kk[c]++;
        res.S[c].push_back(sv[c][i]);
      } else {
        disc += sv[c][i] * sv[c][i];
      }
    }
  }
  res.err = std::sqrt(disc);
  Par nl = make_par(kk[0], kk[1]);
  std::vector<Par> ul = bt.rp;
  ul.push_back(nl);
  std::vector<Par> vl{nl};
  vl.insert(vl.end(), bt.cp.begin(), bt.cp.end());
  res.U = E.zeros(ul);
  res.V = E.zeros(vl);
  int nr = (int)rows.size();
  for (int c = 0; c < 2; ++c) {
    if (dmap[c] < 0 || kk[c] == 0) continue;
    auto& d = ds[dmap[c]];
    Buf t1, t2, t3, t4;
    auto urow = tensor_rows(res.U, 0, nr, c);
    auto ucol = leg_offsets(c, kk[0], kk[1], res.U.strides[nr]);
    auto vrow = leg_offsets(c, kk[0], kk[1], res.V.strides[0]);
    auto vcol = tensor_rows(res.V, 1, (int)cols.size(), c);
    int64_t* urd = E.upload_i64(urow, t1);
    int64_t* ucd = E.upload_i64(ucol, t2);
    int64_t* vrd = E.upload_i64(vrow, t3);
    int64_t* vcd = E.upload_i64(vcol, t4);
    if (tall[c]) {
      // U = q (m x n, ld m), V rows = columns of r (n x n, ld n)
      scatter_block(E, res.U, urd, ucd, m[c], kk[c], d.q, m[c], false);
      scatter_block(E, res.V, vrd, vcd, kk[c], n[c], d.r, n[c], true);
    } else {
      // M^T = U' S V'^T: U = V' (r, m x m, ld m); V rows = columns of U' (q, n x m, ld n)
      scatter_block(E, res.U, urd, ucd, m[c], kk[c], d.r, m[c], false);
      scatter_block(E, res.V, vrd, vcd, kk[c], n[c], d.q, n[c], true);
    }
    keep.insert(keep.end(), {t1, t2, t3, t4});
  }
  return res;
}

bool svd_prefers_kept(const Tensor& A, const std::vector<int>& rows, const std::vector<int>& cols, const Trunc& tr,
                      bool want_entropy) {
  BlockTables bt = tables_of(A, rows, cols);
  for (int c = 0; c < 2; ++c)
    if (std::min(bt.rt[c].size(), bt.ct[c].size()) >= 160) return true;
  if (want_entropy) return false;
  // blocks that suit the subspace iteration (a few kept vectors of a larger block)
  bool any = false;
  for (int c = 0; c < 2; ++c) {
    const int m = (int)bt.rt[c].size(), n = (int)bt.ct[c].size();
    if (std::min(m, n) == 0) continue;
    int k = std::min(m, n);
    if (tr.chi >= 0) k = std::min(k, tr.chi);
    if (tr.space[0] >= 0) k = std::min(k, tr.space[c]);
    if (k < 1 || std::max(m, n) < 96 || la::topk_block_size(k, m, n) == 0) return false;
    any = true;
  }
  return any;
}

// Output tensors of a kept-vector truncated SVD.  Block c has the gathered
// matrix Mb[c] (m x n, ld m) and its wanted vectors Fv[c] (left: m x kk, ld m;
// right: n x kk, ld n, as columns); F holds those vectors, W the other factor
// from one GEMM with the matrix (left: W = U_k^T M; right: W = M V_k).
static void kept_assemble(Engine& E, const BlockTables& bt, int nr, int nc, bool left, const int m[2],
                          const int n[2], const int kk[2], double* const Mb[2], double* const Fv[2], KeptSVD& res) {
  std::vector<Buf> keep;
  Par nl = make_par(kk[0], kk[1]);
  if (left) {
    std::vector<Par> fl = bt.rp;
    fl.push_back(nl);
    std::vector<Par> wl{nl};
    wl.insert(wl.end(), bt.cp.begin(), bt.cp.end());
    res.F = E.zeros(fl);
    res.W = E.zeros(wl);
  } else {
    std::vector<Par> fl{nl};
    fl.insert(fl.end(), bt.cp.begin(), bt.cp.end());
    std::vector<Par> wl = bt.rp;
    wl.push_back(nl);
    res.F = E.zeros(fl);
    res.W = E.zeros(wl);
  }
  for (int c = 0; c < 2; ++c) {
    if (kk[c] == 0) continue;
    Buf wb = E.alloc(sizeof(double) * (size_t)std::max(m[c], n[c]) * kk[c]);
    double* Wm = (double*)wb->ptr;
    Buf t1, t2, t3, t4;
    if (left) {
      la::dgemm_cm(E, true, kk[c], n[c], m[c], 1.0, Fv[c], m[c], Mb[c], m[c], 0.0, Wm, kk[c]);
      auto frow = tensor_rows(res.F, 0, nr, c);
      auto fcol = leg_offsets(c, kk[0], kk[1], res.F.strides[nr]);
      scatter_block(E, res.F, E.upload_i64(frow, t1), E.upload_i64(fcol, t2), m[c], kk[c], Fv[c], m[c], false);
      auto wrow = leg_offsets(c, kk[0], kk[1], res.W.strides[0]);
      auto wcol = tensor_rows(res.W, 1, nc, c);
      scatter_block(E, res.W, E.upload_i64(wrow, t3), E.upload_i64(wcol, t4), kk[c], n[c], Wm, kk[c], false);
    } else {
      la::dgemm_cm(E, false, m[c], kk[c], n[c], 1.0, Mb[c], m[c], Fv[c], n[c], 0.0, Wm, m[c]);
      auto frow = leg_offsets(c, kk[0], kk[1], res.F.strides[0]);
      auto fcol = tensor_rows(res.F, 1, nc, c);
      scatter_block(E, res.F, E.upload_i64(frow, t1), E.upload_i64(fcol, t2), kk[c], n[c], Fv[c], n[c], true);
      auto wrow = tensor_rows(res.W, 0, nr, c);
      auto wcol = leg_offsets(c, kk[0], kk[1], res.W.strides[nr]);
      scatter_block(E, res.W, E.upload_i64(wrow, t3), E.upload_i64(wcol, t4), m[c], kk[c], Wm, m[c], false);
    }
    keep.insert(keep.end(), {wb, t1, t2, t3, t4});
  }
}

// Kept sets of a truncation from per-block leading values; every kept set must
// be a prefix of its block.
static void kept_counts(const std::vector<double> sv[2], const Trunc& tr, const char* who, int kk[2], KeptSVD& res,
                        double& kept2, double& disc2) {
  std::vector<char> kp[2];
  select_truncation(sv, tr, kp);
  kk[0] = kk[1] = 0;
  kept2 = disc2 = 0;
  for (int c = 0; c < 2; ++c)
    for (size_t i = 0; i < sv[c].size(); ++i) {
      if (kp[c][i]) {
        if ((int)i != kk[c]) throw Error(SPS_ERR_NUMERIC, std::string(who) + ": non-prefix truncation");
        kk[c]++;
        res.S[c].push_back(sv[c][i]);
        kept2 += sv[c][i] * sv[c][i];
      } else {
        disc2 += sv[c][i] * sv[c][i];
      }
    }
}

// Leading vectors by subspace iteration (la::svd_topk): only the values that
// the truncation can keep are computed; the discarded weight is ||M||_F^2 minus
// the kept weight.  Returns false when a block does not suit the method or the
// iteration did not converge; the caller then uses the full spectrum.
static bool svd_kept_topk(Engine& E, const BlockTables& bt, const Tensor& A, int nr, int nc, const Trunc& tr,
                          bool left, KeptSVD& res) {
  HostTimer ht(E, "host.svd_kept");
  int m[2], n[2], kmax[2];
  std::vector<la::TopkDesc> ds;
  int dmap[2] = {-1, -1};
  int nprob = 0;
  for (int c = 0; c < 2; ++c) {
    m[c] = (int)bt.rt[c].size();
    n[c] = (int)bt.ct[c].size();
    kmax[c] = std::min(m[c], n[c]);
    if (tr.chi >= 0) kmax[c] = std::min(kmax[c], tr.chi);
    if (tr.space[0] >= 0) kmax[c] = std::min(kmax[c], tr.space[c]);
    if (std::min(m[c], n[c]) == 0) continue;
    if (kmax[c] < 1 || la::topk_block_size(kmax[c], m[c], n[c]) == 0) return false;
    nprob++;
  }
  for (int c = 0; c < 2; ++c)
    if (std::min(m[c], n[c]) > 0 && !la::topk_fits(kmax[c], m[c], n[c], nprob, E)) return false;
  if (nprob == 0) return false;
  std::vector<Buf> keep;
  double* Mb[2] = {nullptr, nullptr};
  double* Fv[2] = {nullptr, nullptr};
  for (int c = 0; c < 2; ++c) {
    if (std::min(m[c], n[c]) == 0) continue;
    Buf t1, t2;
    int64_t* rt = E.upload_i64(bt.rt[c], t1);
    int64_t* ct = E.upload_i64(bt.ct[c], t2);
    Buf mb = E.alloc(sizeof(double) * ((size_t)m[c] * n[c] + (size_t)(m[c] + n[c]) * kmax[c]));
    keep.insert(keep.end(), {t1, t2, mb});
    Mb[c] = (double*)mb->ptr;
    gather_block(E, A, rt, ct, m[c], n[c], Mb[c], m[c], false);
    la::TopkDesc d;
    d.M = Mb[c];
    d.m = m[c];
    d.n = n[c];
    d.k = kmax[c];
    d.U = Mb[c] + (size_t)m[c] * n[c];
    d.V = d.U + (size_t)m[c] * kmax[c];
    d.gram = tr.gram;
    Fv[c] = left ? d.U : d.V;
    dmap[c] = (int)ds.size();
    ds.push_back(d);
  }
  la::svd_topk(E, ds, tr.rtol);
  // A Gram-mode problem whose iterate lost wanted directions (a spectrum that
  // decays faster than the rounding level of M M^T resolves: status 4) runs
  // again on M itself.
  constexpr int TOPK_ZERO = 4;
  std::vector<la::TopkDesc> again;
  std::vector<int> where;
  for (size_t i = 0; i < ds.size(); ++i)
    if (ds[i].status == TOPK_ZERO && ds[i].gram) {
      again.push_back(ds[i]);
      again.back().gram = false;
      where.push_back((int)i);
    }
  if (!again.empty()) {
    if (E.profile) E.add_stat("svd_topk.gram_retry", 0.0, (long long)again.size());
    la::svd_topk(E, again, tr.rtol);
    for (size_t i = 0; i < again.size(); ++i) ds[where[i]] = again[i];
  }
  for (auto& d : ds)
    if (d.status != 0 && !(d.status == TOPK_ZERO && !d.gram)) return false;
  std::vector<double> sv[2];
  double fro2 = 0;
  for (int c = 0; c < 2; ++c) {
    if (dmap[c] < 0) continue;
    la::TopkDesc& d = ds[dmap[c]];
    fro2 += d.fro2;
    sv[c].assign(d.s.begin(), d.s.begin() + kmax[c]);
    if (d.status == 0) continue;
    // Converged on M with r < k nonzero values (fewer than k singular values
    // above the rounding level): the wanted vectors r..k-1 carry zero values,
    // so any orthonormal completion gives the same contractions.  Seeded
    // Gaussian columns after the first r, a Householder QR of the len x k set,
    // and Q's columns r..k-1 (orthogonal to the first r) into place; the first
    // r columns are kept as they are.
    int r = 0;
    while (r < kmax[c] && sv[c][r] > 0.0) ++r;
    for (int i = r; i < kmax[c]; ++i) sv[c][i] = 0.0;
    const int len = left ? d.m : d.n, kk = kmax[c];
    if (r == kk) continue;
    std::vector<double> rnd((size_t)len * (kk - r));
    uint64_t st = 0x9E3779B97F4A7C15ull ^ ((uint64_t)len << 20) ^ (uint64_t)kk;
    auto next = [&st]() {   // splitmix64
      uint64_t z = (st += 0x9E3779B97F4A7C15ull);
      z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
      z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
      return (double)((z ^ (z >> 31)) >> 11) * (1.0 / 9007199254740992.0);
    };
    for (auto& v : rnd) {   // two uniforms -> Box-Muller
      const double u1 = std::max(next(), 1e-300), u2 = next();
      v = std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    }
    double* F = Fv[c];
    Buf qb = E.alloc(sizeof(double) * ((size_t)len * kk * 2 + (size_t)kk * kk + kk));
    double* T = (double*)qb->ptr;
    double* Q = T + (size_t)len * kk;
    double* R = Q + (size_t)len * kk;
    SPS_CUDA(cudaMemcpyAsync(T, F, sizeof(double) * (size_t)len * r, cudaMemcpyDeviceToDevice, E.stream));
    E.stage(rnd.data(), sizeof(double) * rnd.size(), T + (size_t)len * r);
    la::qr_batched(E, {la::MatDesc{T, Q, R, R + (size_t)kk * kk, len, kk, len, len, kk}});
    SPS_CUDA(cudaMemcpyAsync(F + (size_t)len * r, Q + (size_t)len * r, sizeof(double) * (size_t)len * (kk - r),
                             cudaMemcpyDeviceToDevice, E.stream));
    keep.push_back(qb);
    if (E.profile) E.add_stat("svd_topk.completed", 0.0, (long long)(kk - r));
  }
  int kk[2];
  double kept2, disc2;
  kept_counts(sv, tr, "svd_kept", kk, res, kept2, disc2);
  res.norm = std::sqrt(fro2);
  res.err = std::sqrt(std::max(0.0, fro2 - kept2));
  kept_assemble(E, bt, nr, nc, left, m, n, kk, Mb, Fv, res);
  return true;
}

KeptSVD svd_kept(Engine& E, const Tensor& A, const std::vector<int>& rows, const std::vector<int>& cols,
                 const Trunc& tr, bool want_entropy, bool left) {
  BlockTables bt = tables_of(A, rows, cols);
  const int nr = (int)rows.size(), nc = (int)cols.size();
  if (!want_entropy && !E.full_spectrum) {
    KeptSVD res;
    if (svd_kept_topk(E, bt, A, nr, nc, tr, left, res)) return res;
  }
  int m[2], n[2], k[2];
  struct Work { Buf mb, xb, qb, rb, sb, ub; double *M, *X, *U, *s; int mx, nx; bool direct; };
  Work w[2] = {};
  std::vector<la::MatDesc> jac;
  int jmap[2] = {-1, -1};
  std::vector<Buf> keep;
  for (int c = 0; c < 2; ++c) {
    m[c] = (int)bt.rt[c].size();
    n[c] = (int)bt.ct[c].size();
    k[c] = std::min(m[c], n[c]);
    if (k[c] == 0) continue;
    Work& W = w[c];
    Buf t1, t2;
    int64_t* rt = E.upload_i64(bt.rt[c], t1);
    int64_t* ct = E.upload_i64(bt.ct[c], t2);
    keep.insert(keep.end(), {t1, t2});
    W.mb = E.alloc(sizeof(double) * (size_t)m[c] * n[c]);
    W.M = (double*)W.mb->ptr;
    gather_block(E, A, rt, ct, m[c], n[c], W.M, m[c], false);
    // vectors wanted: left -> of M (length m), right -> of M^T (length n)
    int a = left ? m[c] : n[c];   // length of the wanted vectors
    int b = left ? n[c] : m[c];   // other dimension
    if (a <= b) {
      // X = L from the LQ of the (a x b) matrix: QR of its transpose (b x a), X = R^T (a x a)
      W.mx = a;
      W.nx = a;
      W.direct = false;
      Buf tb = E.alloc(sizeof(double) * (size_t)b * a);
      double* T = (double*)tb->ptr;
      if (left) la::transpose_cm(E, W.M, m[c], n[c], m[c], T, n[c]);                       // M^T (n x m)
      else SPS_CUDA(cudaMemcpyAsync(T, W.M, sizeof(double) * (size_t)m[c] * n[c], cudaMemcpyDeviceToDevice, E.stream));
      W.rb = E.alloc(sizeof(double) * (size_t)a * a);
      double* R = (double*)W.rb->ptr;
      if (la::qr_is_big(b, a)) {
        la::qr_big_opt(E, T, b, a, b, nullptr, b, R, a, false);
      } else {
        Buf qb = E.alloc(sizeof(double) * (size_t)b * a + a);
        la::qr_batched(E, {la::MatDesc{T, (double*)qb->ptr, R, (double*)qb->ptr + (size_t)b * a, b, a, b, b, a}});
        keep.push_back(qb);
      }
      keep.push_back(tb);
      W.xb = E.alloc(sizeof(double) * (size_t)a * a);
      W.X = (double*)W.xb->ptr;
      la::transpose_cm(E, R, a, a, a, W.X, a);
    } else {
      // a > b: Jacobi directly on the (a x b) matrix whose columns span the wanted space
      W.mx = a;
      W.nx = b;
      W.direct = true;
      W.xb = E.alloc(sizeof(double) * (size_t)a * b);
      W.X = (double*)W.xb->ptr;
      if (left) SPS_CUDA(cudaMemcpyAsync(W.X, W.M, sizeof(double) * (size_t)m[c] * n[c], cudaMemcpyDeviceToDevice, E.stream));
      else la::transpose_cm(E, W.M, m[c], n[c], m[c], W.X, n[c]);
    }
    W.ub = E.alloc(sizeof(double) * (size_t)W.mx * W.nx);
    W.sb = E.alloc(sizeof(double) * W.nx);
    W.U = (double*)W.ub->ptr;
    W.s = (double*)W.sb->ptr;
    jmap[c] = (int)jac.size();
    jac.push_back({W.X, W.U, nullptr, W.s, W.mx, W.nx, W.mx, W.mx, 0});
  }
  la::jacobi_left(E, jac);
  // singular values to the host
  std::vector<double> sv[2];
  {
    std::vector<std::pair<const double*, int>> src;
    for (int c = 0; c < 2; ++c) src.push_back({jmap[c] < 0 ? nullptr : w[c].s, jmap[c] < 0 ? 0 : k[c]});
    auto v = read_values(E, src, "svd_kept");
    for (int c = 0; c < 2; ++c) sv[c] = std::move(v[c]);
  }
  KeptSVD res;
  double tot2 = 0;
  for (int c = 0; c < 2; ++c)
    for (double x : sv[c]) tot2 += x * x;
  res.norm = std::sqrt(tot2);
  if (want_entropy) {
    if (res.norm == 0) res.entropy = NAN;
    else {
      double ent = 0;
      for (int c = 0; c < 2; ++c)
        for (double x : sv[c]) {
          double p = (x / res.norm) * (x / res.norm);
          if (p != 0) ent -= p * std::log(p);
        }
      res.entropy = std::max(0.0, ent);
    }
  }
  int kk[2];
  double kept2, disc2;
  kept_counts(sv, tr, "svd_kept", kk, res, kept2, disc2);
  res.err = std::sqrt(disc2);
  double* Mb[2] = {w[0].M, w[1].M};
  double* Fv[2] = {w[0].U, w[1].U};
  kept_assemble(E, bt, nr, nc, left, m, n, kk, Mb, Fv, res);
  return res;
}

EIGres eigh(Engine& E, const Tensor& A, const std::vector<int>& rows, const std::vector<int>& cols) {
  BlockTables bt = tables_of(A, rows, cols);
  int n[2];
  for (int c = 0; c < 2; ++c) {
    n[c] = (int)bt.rt[c].size();
    if ((int)bt.ct[c].size() != n[c]) throw Error(SPS_ERR_ARGUMENT, "eigh: non-square block");
  }
  std::vector<la::MatDesc> ds;
  std::vector<Buf> keep;
  int dmap[2] = {-1, -1};
  for (int c = 0; c < 2; ++c) {
    if (n[c] == 0) continue;
    Buf ba = E.alloc(sizeof(double) * ((size_t)n[c] * n[c] * 2 + n[c]));
    double* a = (double*)ba->ptr;
    double* q = a + (size_t)n[c] * n[c];
    double* s = q + (size_t)n[c] * n[c];
    Buf t1, t2;
    gather_block(E, A, E.upload_i64(bt.rt[c], t1), E.upload_i64(bt.ct[c], t2), n[c], n[c], a, n[c], false);
    dmap[c] = (int)ds.size();
    ds.push_back({a, q, nullptr, s, n[c], n[c], n[c], n[c], 0});
    keep.insert(keep.end(), {ba, t1, t2});
  }
  la::eigh_batched(E, ds);
  EIGres res;
  {
    std::vector<std::pair<const double*, int>> src;
    for (int c = 0; c < 2; ++c) src.push_back({dmap[c] < 0 ? nullptr : ds[dmap[c]].s, dmap[c] < 0 ? 0 : n[c]});
    auto v = read_values(E, src, "eigh");
    for (int c = 0; c < 2; ++c) res.w[c] = std::move(v[c]);
  }
  Par nl = make_par(n[0], n[1]);
  std::vector<Par> vl = bt.rp;
  vl.push_back(nl);
  res.V = E.zeros(vl);
  int nr = (int)rows.size();
  for (int c = 0; c < 2; ++c) {
    if (dmap[c] < 0) continue;
    Buf t1, t2;
    auto vr = tensor_rows(res.V, 0, nr, c);
    auto vc = leg_offsets(c, n[0], n[1], res.V.strides[nr]);
    scatter_block(E, res.V, E.upload_i64(vr, t1), E.upload_i64(vc, t2), n[c], n[c], ds[dmap[c]].q, n[c],
                  false);
    keep.insert(keep.end(), {t1, t2});
  }
  return res;
}

__global__ void add_diag_kernel(double* a, int n, int lda, double v) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) a[i + (size_t)i * lda] += v;
}

EIGres eigh_unit_shifted(Engine& E, const Tensor& A, const std::vector<int>& rows, const std::vector<int>& cols) {
  BlockTables bt = tables_of(A, rows, cols);
  int n[2];
  for (int c = 0; c < 2; ++c) {
    n[c] = (int)bt.rt[c].size();
    if ((int)bt.ct[c].size() != n[c]) throw Error(SPS_ERR_ARGUMENT, "eigh_unit_shifted: non-square block");
  }
  // blocks below SMALL rows go to the single-CTA two-sided Jacobi (the block
  // one-sided Jacobi pairs column blocks of four and needs several of them)
  constexpr int SMALL = 32;
  std::vector<la::MatDesc> big, small;
  std::vector<Buf> keep;
  la::MatDesc dd[2];
  bool shifted[2] = {false, false};
  for (int c = 0; c < 2; ++c) {
    if (n[c] == 0) continue;
    Buf ba = E.alloc(sizeof(double) * ((size_t)n[c] * n[c] * 2 + n[c]));
    double* a = (double*)ba->ptr;
    double* q = a + (size_t)n[c] * n[c];
    double* s = q + (size_t)n[c] * n[c];
    Buf t1, t2;
    gather_block(E, A, E.upload_i64(bt.rt[c], t1), E.upload_i64(bt.ct[c], t2), n[c], n[c], a, n[c], false);
    dd[c] = {a, q, nullptr, s, n[c], n[c], n[c], n[c], 0};
    if (n[c] >= SMALL) {
      add_diag_kernel<<<std::min(1024, (n[c] + 255) / 256), 256, 0, E.stream>>>(a, n[c], n[c], 1.0);
      SPS_CUDA(cudaGetLastError());
      shifted[c] = true;
      big.push_back(dd[c]);
    } else {
      small.push_back(dd[c]);
    }
    keep.insert(keep.end(), {ba, t1, t2});
  }
  if (!big.empty()) la::jacobi_left(E, big);
  if (!small.empty()) la::eigh_batched(E, small);
  EIGres res;
  {
    std::vector<std::pair<const double*, int>> src;
    for (int c = 0; c < 2; ++c) src.push_back({n[c] == 0 ? nullptr : dd[c].s, n[c]});
    auto v = read_values(E, src, "eigh_unit_shifted");
    for (int c = 0; c < 2; ++c) {
      res.w[c] = std::move(v[c]);
      if (shifted[c])
        for (double& x : res.w[c]) x -= 1.0;
    }
  }
  Par nl = make_par(n[0], n[1]);
  std::vector<Par> vl = bt.rp;
  vl.push_back(nl);
  res.V = E.zeros(vl);
  int nr = (int)rows.size();
  for (int c = 0; c < 2; ++c) {
    if (n[c] == 0) continue;
    Buf t1, t2;
    auto vr = tensor_rows(res.V, 0, nr, c);
    auto vc = leg_offsets(c, n[0], n[1], res.V.strides[nr]);
    scatter_block(E, res.V, E.upload_i64(vr, t1), E.upload_i64(vc, t2), n[c], n[c], dd[c].q, n[c], false);
    keep.insert(keep.end(), {t1, t2});
  }
  return res;
}

Tensor block_inverse(Engine& E, const Tensor& R) {
  BlockTables bt = tables_of(R, {0}, {1});
  Tensor out = E.zeros({R.legs[1], R.legs[0]});
  std::vector<la::MatDesc> ds;
  std::vector<Buf> keep;
  int dmap[2] = {-1, -1};
  for (int c = 0; c < 2; ++c) {
    int m = (int)bt.rt[c].size(), n = (int)bt.ct[c].size();
    if (m != n) throw Error(SPS_ERR_ARGUMENT, "block_inverse: non-square block");
    if (n == 0) continue;
    Buf ba = E.alloc(sizeof(double) * (size_t)n * n * 2);
    double* a = (double*)ba->ptr;
    double* q = a + (size_t)n * n;
    Buf t1, t2;
    gather_block(E, R, E.upload_i64(bt.rt[c], t1), E.upload_i64(bt.ct[c], t2), n, n, a, n, false);
    dmap[c] = (int)ds.size();
    ds.push_back({a, q, nullptr, nullptr, n, n, n, n, 0});
    keep.insert(keep.end(), {ba, t1, t2});
  }
  la::inv_batched(E, ds);
  for (int c = 0; c < 2; ++c) {
    if (dmap[c] < 0) continue;
    int n = ds[dmap[c]].n;
    Buf t1, t2;
    auto rr = tensor_rows(out, 0, 1, c);
    auto cc = tensor_rows(out, 1, 1, c);
    scatter_block(E, out, E.upload_i64(rr, t1), E.upload_i64(cc, t2), n, n, ds[dmap[c]].q, n, false);
    keep.insert(keep.end(), {t1, t2});
  }
  return out;
}

}  // namespace sps
