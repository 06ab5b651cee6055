// gcl_device.cuh -- device helpers shared by the canonical-labeling kernels.
#pragma once
#include <cstdint>

#define GCL_FULL 0xffffffffu

namespace gcl {

// Invariant hash of the reference (partition_refinement.h:9-19, nauty's
// MASH/CLEANUP).  The reference keeps the running value in a uint64_t but
// masks every step to 15 bits, so 32-bit arithmetic gives identical codes.
__device__ __forceinline__ uint32_t mash(uint32_t l, uint32_t i) {
  return ((l ^ 065435u) + i) & 077777u;
}
__device__ __forceinline__ int cleanup(uint32_t l) { return (int)(l % 077777u); }
constexpr int kSentinel = 077777;  // code appended at a leaf (sequential.cpp:268)

// 64-bit mask helpers that are defined for shift counts 0..64.
__device__ __forceinline__ uint64_t low_mask(uint32_t k) {  // bits < k
  return k >= 64 ? ~0ull : ((1ull << k) - 1ull);
}
__device__ __forceinline__ uint64_t ge_mask(uint32_t k) {  // bits >= k
  return k >= 64 ? 0ull : (~0ull << k);
}
__device__ __forceinline__ uint32_t ctz64(uint64_t x) { return (uint32_t)(__ffsll((long long)x) - 1); }
__device__ __forceinline__ uint32_t msb64(uint64_t x) { return 63u - (uint32_t)__clzll((long long)x); }
__device__ __forceinline__ uint32_t popc64(uint64_t x) { return (uint32_t)__popcll(x); }

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

// mash folded over the items of the lanes in `mask`, in lane order (lane k
// holds v_k; other lanes are ignored), mask != 0: the 15 bits of the result
// computed one
// bit position at a time over all items at once.  With y_k = x_k ^ 065435,
// x_{k+1} = y_k + v_k; bit j of x flips at item k by 065435_j ^ v_kj ^
// carry_kj, so bit j before item k is bit j of x_0 xor the parity of the
// flips of the items before it (a ballot), and that gives the carries into
// bit j+1.  Bits above 14 of x_0 and v_k never reach bits 0..14.  Warp-wide;
// returns the same value on every lane.
__device__ __forceinline__ uint32_t mash_fold_mask(uint32_t lc, uint32_t v, uint32_t mask) {
  uint32_t lt;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(lt));
  const bool valid = (mask >> (threadIdx.x & 31u)) & 1u;
  uint32_t carry = 0, out = 0;
#pragma unroll
  for (int j = 0; j < 15; ++j) {
    const uint32_t cj = (065435u >> j) & 1u;
    const uint32_t vj = (v >> j) & 1u;
    const uint32_t x0 = (lc >> j) & 1u;
    const uint32_t flip = valid ? (cj ^ vj ^ carry) : 0u;
    const uint32_t B = __ballot_sync(GCL_FULL, flip != 0);
    const uint32_t y = x0 ^ ((uint32_t)__popc(B & lt) & 1u) ^ cj;
    carry = (y & vj) | (y & carry) | (vj & carry);
    out |= (x0 ^ ((uint32_t)__popc(B) & 1u)) << j;
  }
  return out;
}
// ... over lanes 0 .. m-1, 1 <= m <= 32
__device__ __forceinline__ uint32_t mash_fold32(uint32_t lc, uint32_t v, uint32_t m) {
  return mash_fold_mask(lc, v, m >= 32 ? 0xffffffffu : ((1u << m) - 1u));
}

__device__ __forceinline__ uint64_t warp_or64(uint64_t x) {
  uint32_t lo = __reduce_or_sync(GCL_FULL, (uint32_t)x);
  uint32_t hi = __reduce_or_sync(GCL_FULL, (uint32_t)(x >> 32));
  return ((uint64_t)hi << 32) | lo;
}
__device__ __forceinline__ uint64_t bcast64(uint64_t x, int src) {
  uint32_t lo = __shfl_sync(GCL_FULL, (uint32_t)x, src);
  uint32_t hi = __shfl_sync(GCL_FULL, (uint32_t)(x >> 32), src);
  return ((uint64_t)hi << 32) | lo;
}

}  // namespace gcl
