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
