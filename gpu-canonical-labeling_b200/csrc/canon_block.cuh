// canon_block.cuh -- graphs with n > 64 (one thread block per graph).
#pragma once
#include <cuda_runtime.h>

#include "canon_warp64.cuh"

struct gcl_context;

namespace gcl {

struct Deferred;

// Blocks of the large-graph kernel that fit on the device at once.
inline cudaError_t block_occupancy(int* grid, int sms) {
  *grid = sms;
  return cudaSuccess;
}

// Enqueue the large-graph pass over the graphs the warp pass deferred.
// Until the block kernel lands these graphs keep status kTooLarge.
inline int block_pass_async(gcl_context*, const BatchArgs&, Deferred*, int*, int, uint32_t) {
  return 0;
}

}  // namespace gcl
