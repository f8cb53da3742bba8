// Mixed-precision contraction GEMM on the 5th-generation tensor cores
// (tcgen05): the low-precision path of the contraction GEMMs (row
// absorptions, row steps, reduced metrics).  Factorizations, normalisations,
// log weights and Born probabilities stay FP64 elsewhere.
//
// C_c[i, j] = alpha sum_k A[ra[i] + ca[k]] B[rb[k] + cb[j]] for one parity
// block of a table-addressed contraction (the operands and the output are
// Z2 tensors addressed through int64 offset tables, as in the FP64 path):
//
//   1. pack: the A block (M x K) and the transposed B block (N x K) are
//      gathered from FP64, rounded and written K-contiguous, zero-padded to
//      the tile grid -- TF32 (fp32 bits rounded to 10 mantissa bits), or a
//      split x = hi + lo into two TF32 or two BF16 parts;
//   2. GEMM: one 128 x BN output tile per CTA (BN = 64, 128 or 256).  Warp 0
//      streams 128-byte wide K slices of A and B into shared memory with TMA
//      (128-byte swizzle, mbarrier stages); one thread of warp 1 issues
//      tcgen05.mma with the accumulator in tensor memory (FP32, 128 lanes x BN
//      columns): one product per K step, or three for a split (lo*hi + hi*lo +
//      hi*hi, the lo*lo term dropped); warps 2-5 read the accumulator back with
//      tcgen05.ld and write alpha * acc as FP64 through C's offset tables.
//
// Precision per product: TF32 ~ 2^-11 relative, 3xTF32 ~ 2^-21, 3xBF16 ~ 2^-16,
// with FP32 accumulation over K.
#include "engine.h"
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <mutex>

namespace sps {
namespace tc {

namespace {

constexpr int BM = 128;             // tile rows = tensor-memory lanes
constexpr int SLICE = 128;          // bytes of K per operand row and stage (one swizzle atom row)
constexpr int NT = 192;             // warp 0 TMA, warp 1 TMEM + MMA, warps 2-5 epilogue
constexpr int TILE_A = BM * SLICE;  // 16 KB
constexpr int SMEM_TILES = 196608;  // stage budget (192 KB)
constexpr long long WAIT_CAP = 1ll << 26;
constexpr int FLAG_COPY_WAIT = 8;   // the engine's "bulk-copy wait reached its cap"

__device__ __forceinline__ unsigned saddr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ bool mbar_try(unsigned bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// bounded wait: false (and the flag raised) when the cap is reached
__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned parity, int* flag) {
  long long spins = 0;
  while (!mbar_try(bar, parity))
    if (++spins > WAIT_CAP) {
      atomicOr(flag, FLAG_COPY_WAIT);
      return false;
    }
  return true;
}

__device__ __forceinline__ void tma_load_2d(unsigned dst, const CUtensorMap* map, int x, int y, unsigned bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
          "r"(dst),
      "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(bar)
      : "memory");
}

// shared-memory matrix descriptor of a K-major operand tile in the canonical
// 128-byte-swizzle layout: rows of 128 bytes, 8-row atoms 1024 bytes apart
__device__ __forceinline__ unsigned long long smem_desc(unsigned addr) {
  unsigned long long d = 0;
  d |= (unsigned long long)((addr >> 4) & 0x3FFFu);        // start address
  d |= (unsigned long long)1 << 16;                         // leading byte offset (unused when swizzled)
  d |= (unsigned long long)(1024 >> 4) << 32;               // stride byte offset: one 8-row atom
  d |= (unsigned long long)1 << 46;                         // descriptor version of tcgen05
  d |= (unsigned long long)2 << 61;                         // 128-byte swizzle
  return d;
}

template <int KIND>   // 0: kind::tf32, 1: kind::f16 (bf16 operands)
__device__ __forceinline__ void mma(unsigned tmem, unsigned long long a, unsigned long long b, unsigned idesc,
                                    unsigned accumulate) {
  if (KIND == 0)
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}" ::
            "r"(tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
        : "memory");
  else
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}" ::
            "r"(tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void mma_commit(unsigned bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

struct OutDesc {
  double* C;
  const int64_t* rc;
  const int64_t* cc;
  int M, N;
  double alpha;
  int* flag;
};

// One 128 x BN tile of C over KT K slices (BN = 64, 128 or 256 accumulator
// columns).  SPLIT: A and B come as hi and lo parts (three products per K step).
template <int KIND, bool SPLIT, int BN>
__global__ void __launch_bounds__(NT, 1) tc_gemm_kernel(const __grid_constant__ CUtensorMap tAh,
                                                         const __grid_constant__ CUtensorMap tAl,
                                                         const __grid_constant__ CUtensorMap tBh,
                                                         const __grid_constant__ CUtensorMap tBl, OutDesc out,
                                                         int KT) {
  constexpr int PARTS = SPLIT ? 2 : 1;
  constexpr int TILE_B = BN * SLICE;
  constexpr int STAGE_BYTES = PARTS * (TILE_A + TILE_B);
  constexpr int S = SMEM_TILES / STAGE_BYTES;   // 2 .. 8 stages
  static_assert(S >= 2 && (BN == 64 || BN == 128 || BN == 256), "tile");
  extern __shared__ unsigned char smem_raw[];
  // tiles start at a 1024-byte boundary (the swizzle atom)
  unsigned char* smem = (unsigned char*)(((unsigned long long)smem_raw + 1023) & ~1023ull);
  __shared__ __align__(8) unsigned long long full[S], empty[S], accbar;
  __shared__ unsigned tmem_slot;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;

  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(saddr(&full[s])) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(saddr(&empty[s])) : "memory");
    }
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(saddr(&accbar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {   // the whole warp allocates BN accumulator columns
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(&tmem_slot)),
                 "r"(BN)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const unsigned tmem = tmem_slot;

  auto tileA = [&](int s, int part) { return smem + s * STAGE_BYTES + part * TILE_A; };
  auto tileB = [&](int s, int part) { return smem + s * STAGE_BYTES + PARTS * TILE_A + part * TILE_B; };
  constexpr int KEL = KIND == 0 ? SLICE / 4 : SLICE / 2;   // elements of K per slice

  if (warp == 0) {
    if (lane == 0) {   // TMA producer
      for (int kt = 0; kt < KT; ++kt) {
        const int s = kt % S, use = kt / S;
        if (use > 0 && !mbar_wait(saddr(&empty[s]), (use - 1) & 1, out.flag)) break;
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(saddr(&full[s])),
                     "r"(STAGE_BYTES)
                     : "memory");
        tma_load_2d(saddr(tileA(s, 0)), &tAh, kt * KEL, m0, saddr(&full[s]));
        tma_load_2d(saddr(tileB(s, 0)), &tBh, kt * KEL, n0, saddr(&full[s]));
        if (SPLIT) {
          tma_load_2d(saddr(tileA(s, 1)), &tAl, kt * KEL, m0, saddr(&full[s]));
          tma_load_2d(saddr(tileB(s, 1)), &tBl, kt * KEL, n0, saddr(&full[s]));
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {   // MMA issuer
      // D f32; A, B: tf32 (2) or bf16 (1), K-major; N >> 3; M >> 4
      constexpr unsigned fmt = KIND == 0 ? 2u : 1u;
      constexpr unsigned idesc = (1u << 4) | (fmt << 7) | (fmt << 10) | ((unsigned)(BN >> 3) << 17) |
                                 ((unsigned)(BM >> 4) << 24);
      for (int kt = 0; kt < KT; ++kt) {
        const int s = kt % S, use = kt / S;
        if (!mbar_wait(saddr(&full[s]), use & 1, out.flag)) break;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const unsigned ah = saddr(tileA(s, 0)), bh = saddr(tileB(s, 0));
#pragma unroll
        for (int kk = 0; kk < SLICE / 32; ++kk) {   // 32 bytes of K per instruction
          const unsigned first = (kt | kk) != 0;
          if (SPLIT) {
            const unsigned al = saddr(tileA(s, 1)), bl = saddr(tileB(s, 1));
            mma<KIND>(tmem, smem_desc(al + 32 * kk), smem_desc(bh + 32 * kk), idesc, first);
            mma<KIND>(tmem, smem_desc(ah + 32 * kk), smem_desc(bl + 32 * kk), idesc, 1u);
            mma<KIND>(tmem, smem_desc(ah + 32 * kk), smem_desc(bh + 32 * kk), idesc, 1u);
          } else {
            mma<KIND>(tmem, smem_desc(ah + 32 * kk), smem_desc(bh + 32 * kk), idesc, first);
          }
        }
        mma_commit(saddr(&empty[s]));   // the stage is free once these products have read it
      }
      mma_commit(saddr(&accbar));       // arrives when every product issued above has completed
    }
  } else {
    // epilogue: warp w reads tensor-memory lanes 32 (w % 4) .. + 31, one output row per thread
    const int q = warp & 3;
    const int row = m0 + 32 * q + lane;
    const bool ready = __all_sync(0xffffffffu, mbar_wait(saddr(&accbar), 0, out.flag));
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (ready) {
      const bool live = row < out.M;
      const int64_t rbase = live ? out.rc[row] : 0;
#pragma unroll 1
      for (int c0 = 0; c0 < BN; c0 += 16) {
        unsigned v[16];
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
              "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
            : "r"(tmem + ((unsigned)(32 * q) << 16) + (unsigned)c0)
            : "memory");
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (live) {
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            const int col = n0 + c0 + j;
            if (col < out.N) out.C[rbase + out.cc[col]] = out.alpha * (double)__uint_as_float(v[j]);
          }
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 1) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(BN) : "memory");
  }
}

// ---------------------------------------------------------------------------
// pack: FP64 block (through offset tables) -> K-contiguous low-precision parts
// ---------------------------------------------------------------------------
__device__ __forceinline__ float tf32_round(float x) {
  unsigned r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

// dst[r * Kp + k], r < Rp, k < Kp: element (r, k) = S[rt[r] + ct[k]] inside
// R x K, zero outside.  kfast: the source is contiguous along k (else along r),
// and a 32 x 32 tile is transposed through shared memory so that both the
// reads and the writes are coalesced.
template <int MODE>   // 1 TF32, 2 split TF32, 3 split BF16
__global__ void __launch_bounds__(256) pack_kernel(const double* __restrict__ S, const int64_t* __restrict__ rt,
                                                   const int64_t* __restrict__ ct, int R, int K, int Kp, void* hi,
                                                   void* lo, int kfast) {
  __shared__ double tile[32][33];
  const int r0 = blockIdx.y * 32, k0 = blockIdx.x * 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  if (kfast) {
    for (int rr = ty; rr < 32; rr += 8) {
      const int r = r0 + rr, k = k0 + tx;
      tile[rr][tx] = (r < R && k < K) ? S[rt[r] + ct[k]] : 0.0;
    }
  } else {
    for (int kk = ty; kk < 32; kk += 8) {
      const int r = r0 + tx, k = k0 + kk;
      tile[tx][kk] = (r < R && k < K) ? S[rt[r] + ct[k]] : 0.0;
    }
  }
  __syncthreads();
  for (int rr = ty; rr < 32; rr += 8) {
    const int r = r0 + rr, k = k0 + tx;
    const double x = tile[rr][tx];
    const size_t o = (size_t)r * Kp + k;
    if (MODE == 3) {
      const __nv_bfloat16 h = __double2bfloat16(x);
      ((__nv_bfloat16*)hi)[o] = h;
      ((__nv_bfloat16*)lo)[o] = __double2bfloat16(x - (double)__bfloat162float(h));
    } else {
      const float h = tf32_round((float)x);
      ((float*)hi)[o] = h;
      if (MODE == 2) ((float*)lo)[o] = tf32_round((float)(x - (double)h));
    }
  }
}

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

// rows x Kp operand (K contiguous), boxes of one 128-byte slice x box_rows rows
void encode(CUtensorMap* map, const void* base, bool bf16, int Kp, int rows, int box_rows) {
  const int es = bf16 ? 2 : 4;
  const cuuint64_t dims[2] = {(cuuint64_t)Kp, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)Kp * es};
  const cuuint32_t box[2] = {(cuuint32_t)(SLICE / es), (cuuint32_t)box_rows};
  const cuuint32_t estr[2] = {1u, 1u};
  const CUresult r = encode_fn()(map, bf16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2,
                                 const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                 CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                 CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) throw Error(SPS_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
}

template <int KIND, bool SPLIT, int BN>
void launch_bn(Engine& E, const CUtensorMap* m, const OutDesc& o, int KT, dim3 grid) {
  const size_t smem = SMEM_TILES + 1024;
  set_max_dynamic_smem((const void*)tc_gemm_kernel<KIND, SPLIT, BN>, (int)smem);
  tc_gemm_kernel<KIND, SPLIT, BN><<<grid, NT, smem, E.stream>>>(m[0], m[1], m[2], m[3], o, KT);
}

template <int KIND, bool SPLIT>
void launch_gemm(Engine& E, const CUtensorMap* m, const OutDesc& o, int KT, dim3 grid, int bn) {
  if (bn == 64) launch_bn<KIND, SPLIT, 64>(E, m, o, KT, grid);
  else if (bn == 256) launch_bn<KIND, SPLIT, 256>(E, m, o, KT, grid);
  else launch_bn<KIND, SPLIT, 128>(E, m, o, KT, grid);
}

}  // namespace

// One parity block: C[rc[i] + cc[j]] = alpha sum_k A[ra[i] + ca[k]] B[rb[k] + cb[j]]
// (i < M, j < N, k < K); tables are device pointers.  C's entries of the block
// are overwritten.
void gemm_block(Engine& E, int mode, const double* A, const int64_t* ra, const int64_t* ca, int a_kfast,
                const double* B, const int64_t* rb, const int64_t* cb, int b_jfast, double* C, const int64_t* rc,
                const int64_t* cc, int M, int N, int K, double alpha) {
  if (mode < 1 || mode > 3) throw Error(SPS_ERR_ARGUMENT, "tc::gemm_block: unknown precision mode");
  if (M <= 0 || N <= 0 || K <= 0) return;
  const bool bf16 = mode == 3;
  const int es = bf16 ? 2 : 4;
  const int kel = SLICE / es;
  const int Kp = (K + kel - 1) / kel * kel;
  const int Mp = (M + BM - 1) / BM * BM;
  // tile width: 64 for narrow outputs, else 128; the autotuner times 64 / 128 / 256
  std::vector<int> cands;
  for (int c : {64, 128, 256})
    if (c == 64 || N > c / 2) cands.push_back(c);
  int bn = N <= 64 ? 64 : 128;
  std::string key;
  bool tuned = false;
  if (E.autotune && cands.size() > 1) {
    key = tune::key(E, "tc_gemm.bn", {mode, M, N, K});
    tuned = tune::lookup(key, &bn);
  }
  const bool tuning = E.autotune && cands.size() > 1 && !tuned;
  const int padn = tuning ? 256 : bn;
  const int Np = (N + padn - 1) / padn * padn;
  const int parts = mode == 1 ? 1 : 2;
  const size_t abytes = (size_t)Mp * Kp * es, bbytes = (size_t)Np * Kp * es;
  Buf ws = E.alloc(parts * (abytes + bbytes) + 256);
  char* base = (char*)ws->ptr;
  void* Ah = base;
  void* Al = parts == 2 ? base + abytes : nullptr;
  void* Bh = base + parts * abytes;
  void* Bl = parts == 2 ? base + parts * abytes + bbytes : nullptr;
  const int tk = E.tic("tc_pack");
  {
    dim3 ga(Kp / 32, Mp / 32), gb(Kp / 32, Np / 32);
    // A block: rows i (table ra), k (table ca); B^T block: rows j (table cb), k (table rb)
    if (mode == 1) {
      pack_kernel<1><<<ga, 256, 0, E.stream>>>(A, ra, ca, M, K, Kp, Ah, nullptr, a_kfast);
      pack_kernel<1><<<gb, 256, 0, E.stream>>>(B, cb, rb, N, K, Kp, Bh, nullptr, b_jfast ? 0 : 1);
    } else if (mode == 2) {
      pack_kernel<2><<<ga, 256, 0, E.stream>>>(A, ra, ca, M, K, Kp, Ah, Al, a_kfast);
      pack_kernel<2><<<gb, 256, 0, E.stream>>>(B, cb, rb, N, K, Kp, Bh, Bl, b_jfast ? 0 : 1);
    } else {
      pack_kernel<3><<<ga, 256, 0, E.stream>>>(A, ra, ca, M, K, Kp, Ah, Al, a_kfast);
      pack_kernel<3><<<gb, 256, 0, E.stream>>>(B, cb, rb, N, K, Kp, Bh, Bl, b_jfast ? 0 : 1);
    }
  }
  E.toc(tk, 0, 8.0 * ((double)M * K + (double)K * N) + (double)parts * es * ((double)Mp * Kp + (double)Np * Kp));
  SPS_CUDA(cudaGetLastError());
  OutDesc o{C, rc, cc, M, N, alpha, E.dflag};
  const int KT = Kp / kel;
  auto run = [&](int w) {
    CUtensorMap maps[4];
    encode(&maps[0], Ah, bf16, Kp, Mp, BM);
    encode(&maps[1], parts == 2 ? Al : Ah, bf16, Kp, Mp, BM);
    encode(&maps[2], Bh, bf16, Kp, Np, w);
    encode(&maps[3], parts == 2 ? Bl : Bh, bf16, Kp, Np, w);
    const dim3 grid((N + w - 1) / w, Mp / BM);
    if (mode == 1) launch_gemm<0, false>(E, maps, o, KT, grid, w);
    else if (mode == 2) launch_gemm<0, true>(E, maps, o, KT, grid, w);
    else launch_gemm<1, true>(E, maps, o, KT, grid, w);
    SPS_CUDA(cudaGetLastError());
  };
  if (tuning) bn = tune::pick(E, key, cands, run);
  const int tg = E.tic(mode == 1 ? "tc_gemm_tf32" : mode == 2 ? "tc_gemm_3xtf32" : "tc_gemm_3xbf16");
  run(bn);
  E.toc(tg, 2.0 * M * N * (double)K, 0);
  E.launches += 3;
  E.flops += 2.0 * M * N * (double)K;
}

}  // namespace tc
}  // namespace sps
