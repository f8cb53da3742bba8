// Device helpers shared by the cooperative (grid-synchronising) kernels.
#pragma once
#include <cuda_runtime.h>

namespace sps {
namespace la {

static constexpr int FLAG_CONV = 2;
static constexpr int FLAG_BARRIER = 4;
static constexpr int FLAG_COPY = 8;   // a bulk-copy completion wait reached its cap

__device__ __forceinline__ double wsum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Software barrier over `count` CTAs of a cooperative launch (all co-resident).
// bar[0] = arrival count, bar[1] = generation.  Acquire/release ordering at gpu
// scope; the spin is bounded and reports FLAG_BARRIER through `flag` when the
// cap is reached (only possible after a fault elsewhere).
__device__ __forceinline__ void group_barrier(unsigned* bar, unsigned count, int* flag) {
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned g;
    asm volatile("ld.acquire.gpu.u32 %0, [%1];" : "=r"(g) : "l"(bar + 1) : "memory");
    unsigned arrived;
    asm volatile("atom.add.acq_rel.gpu.u32 %0, [%1], 1;" : "=r"(arrived) : "l"(bar) : "memory");
    if (arrived == count - 1) {
      asm volatile("st.relaxed.gpu.u32 [%0], 0;" ::"l"(bar) : "memory");
      asm volatile("red.release.gpu.add.u32 [%0], 1;" ::"l"(bar + 1) : "memory");
    } else {
      long long spins = 0;
      unsigned cur;
      do {
        asm volatile("ld.acquire.gpu.u32 %0, [%1];" : "=r"(cur) : "l"(bar + 1) : "memory");
        if (++spins > (1ll << 27)) {
          atomicOr(flag, FLAG_BARRIER);
          break;
        }
      } while (cur == g);
    }
  }
  __syncthreads();
}

}  // namespace la
}  // namespace sps
