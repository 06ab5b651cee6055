// gcl_format.cu -- the reference's canonical adjacency-list text written on
// the device from bit-packed canonical rows (print_canonical_adjacency_list,
// main.cpp:33-70; the row format is gcl_format.h's).
//
// Three kernels on the context's stream: the text length of every graph
// (a block per graph, its threads over the rows), an exclusive scan of the
// lengths into byte offsets (one block), and the text itself (a block per
// graph: each chunk of rows is scanned in shared memory for the rows' byte
// offsets, then each thread writes its row).
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/gcl.h"
#include "gcl_format.h"
#include "gcl_guard.h"

namespace gcl {

int context_device(const gcl_context* c);  // gcl_capi.cu

namespace {

constexpr int kFmtThreads = 256;
constexpr int kScanThreads = 1024;

// exclusive prefix sum over the block (blockDim.x a multiple of 32, at most
// 1024); returns the thread's prefix and the block total in *total
__device__ uint64_t block_exclusive_scan(uint64_t v, uint64_t* total) {
  __shared__ uint64_t warp_sums[32];
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint32_t nwarps = blockDim.x >> 5;
  uint64_t x = v;
  for (uint32_t d = 1; d < 32; d <<= 1) {
    const uint64_t y = __shfl_up_sync(0xffffffffu, x, d);
    if (lane >= d) x += y;
  }
  if (lane == 31) warp_sums[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint64_t s = lane < nwarps ? warp_sums[lane] : 0;
    for (uint32_t d = 1; d < 32; d <<= 1) {
      const uint64_t y = __shfl_up_sync(0xffffffffu, s, d);
      if (lane >= d) s += y;
    }
    if (lane < nwarps) warp_sums[lane] = s;  // inclusive over warps
  }
  __syncthreads();
  const uint64_t before = warp == 0 ? 0 : warp_sums[warp - 1];
  *total = warp_sums[nwarps - 1];
  __syncthreads();  // warp_sums is reused by the next call
  return before + x - v;
}

__global__ void __launch_bounds__(kFmtThreads)
format_len_kernel(int count, const int64_t* voff, const uint64_t* rows, const int64_t* roff,
                  int64_t* toff) {
  __shared__ uint64_t part[kFmtThreads / 32];
  for (int g = blockIdx.x; g < count; g += gridDim.x) {
    const uint32_t n = (uint32_t)(voff[g + 1] - voff[g]);
    const uint32_t words = (n + 63) / 64;
    const uint64_t* R = rows + roff[g];
    uint64_t sum = 0;
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x)
      sum += format_row(R + (uint64_t)i * words, n, i, nullptr);
    for (uint32_t d = 16; d > 0; d >>= 1) sum += __shfl_down_sync(0xffffffffu, sum, d);
    if ((threadIdx.x & 31u) == 0) part[threadIdx.x >> 5] = sum;
    __syncthreads();
    if (threadIdx.x == 0) {
      uint64_t t = 0;
      for (uint32_t w = 0; w < blockDim.x / 32; ++w) t += part[w];
      toff[g + 1] = (int64_t)t;
    }
    __syncthreads();
  }
}

// toff[1..count] lengths -> toff[0..count] byte offsets (toff[0] = 0)
__global__ void __launch_bounds__(kScanThreads) format_scan_kernel(int count, int64_t* toff) {
  const uint64_t per = ((uint64_t)count + blockDim.x - 1) / blockDim.x;
  const uint64_t lo = min((uint64_t)count, per * threadIdx.x);
  const uint64_t hi = min((uint64_t)count, lo + per);
  uint64_t s = 0;
  for (uint64_t k = lo; k < hi; ++k) s += (uint64_t)toff[k + 1];
  uint64_t total = 0;
  uint64_t run = block_exclusive_scan(s, &total);
  for (uint64_t k = lo; k < hi; ++k) {
    const uint64_t len = (uint64_t)toff[k + 1];
    run += len;
    toff[k + 1] = (int64_t)run;
  }
  if (threadIdx.x == 0) toff[0] = 0;
}

__global__ void __launch_bounds__(kFmtThreads)
format_text_kernel(int count, const int64_t* voff, const uint64_t* rows, const int64_t* roff,
                   const int64_t* toff, char* text) {
  for (int g = blockIdx.x; g < count; g += gridDim.x) {
    const uint32_t n = (uint32_t)(voff[g + 1] - voff[g]);
    const uint32_t words = (n + 63) / 64;
    const uint64_t* R = rows + roff[g];
    char* out = text + toff[g];
    uint64_t base = 0;
    for (uint32_t i0 = 0; i0 < n; i0 += blockDim.x) {
      const uint32_t i = i0 + threadIdx.x;
      const uint64_t len = i < n ? format_row(R + (uint64_t)i * words, n, i, nullptr) : 0;
      uint64_t total = 0;
      const uint64_t at = block_exclusive_scan(len, &total);
      if (i < n) format_row(R + (uint64_t)i * words, n, i, out + base + at);
      base += total;
    }
  }
}

}  // namespace
}  // namespace gcl

extern "C" int gcl_format_adjacency_device_async(gcl_context* c, int count, const int64_t* d_voff,
                                                 const uint64_t* d_rows, const int64_t* d_roff,
                                                 int64_t* d_toff, char* d_text) try {
  using namespace gcl;
  if (!c || count < 0 || (count > 0 && (!d_voff || !d_rows || !d_roff || !d_toff)))
    return GCL_ERR_ARG;
  if (cudaSetDevice(context_device(c)) != cudaSuccess) return GCL_ERR_CUDA;
  cudaStream_t s = (cudaStream_t)gcl_stream(c);
  if (count == 0) {
    if (d_text) return GCL_OK;
    return cudaMemsetAsync(d_toff, 0, sizeof(int64_t), s) == cudaSuccess ? GCL_OK : GCL_ERR_CUDA;
  }
  const int grid = count < 4096 ? count : 4096;  // grid-stride over the graphs
  if (!d_text) {
    format_len_kernel<<<grid, kFmtThreads, 0, s>>>(count, d_voff, d_rows, d_roff, d_toff);
    if (cudaGetLastError() != cudaSuccess) return GCL_ERR_CUDA;
    format_scan_kernel<<<1, kScanThreads, 0, s>>>(count, d_toff);
  } else {
    format_text_kernel<<<grid, kFmtThreads, 0, s>>>(count, d_voff, d_rows, d_roff, d_toff,
                                                    d_text);
  }
  return cudaGetLastError() == cudaSuccess ? GCL_OK : GCL_ERR_CUDA;
} GCL_CATCH_ALL
