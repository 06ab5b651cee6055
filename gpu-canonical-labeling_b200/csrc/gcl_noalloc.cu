// gcl_noalloc.cu -- batched canonization of graphs with n <= 64 that
// allocates nothing.
//
// Some callers cannot call cudaMalloc at the point where they want canonical
// forms: a host framework that owns every byte of device memory through its
// own caching allocator (a raw cudaMalloc there either fails because the pool
// has reserved the device, or escapes the framework's accounting), a plugin
// loaded into a process whose policy forbids device allocations after
// start-up, or a latency-critical request path where a cudaMalloc/cudaFree
// pair would synchronize the whole device.  gcl_canon_batch_noalloc serves
// them: the caller passes device buffers it already owns for every input and
// output, and the per-warp scratch the warp kernel needs (orbit
// representatives per search level and the automorphism ring) comes from one
// fixed-size device array that the library reserves statically on every GPU
// it is loaded on, held until the process exits.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <mutex>

#include "../../include/gcl.h"
#include "canon_warp64.cuh"

namespace gcl {

constexpr uint32_t kNoAllocRing = 128;  // automorphism ring entries per warp slot
constexpr int kNoAllocSlots = 512;      // warp slots = 128 blocks of 4 warps
constexpr uint64_t kNoAllocSlotBytes = w64_slot_bytes(kNoAllocRing);
constexpr uint64_t kNoAllocHeader = 256;  // the work counter
constexpr uint64_t kNoAllocBytes = kNoAllocHeader + (uint64_t)kNoAllocSlots * kNoAllocSlotBytes;

// The statically reserved scratch (about 6.6 MiB per GPU).  Host code must
// not pass this name to a kernel: on the host it only stands for the symbol;
// the device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) uint8_t g_noalloc_scratch[kNoAllocBytes];

__global__ void __launch_bounds__(kW64Threads, 8)
    w64_noalloc_kernel(BatchArgs A, uint8_t* scratch) {
  const int warp = (int)(threadIdx.x >> 5);
  const uint32_t lane = lane_id();
  int* next = reinterpret_cast<int*>(scratch);
  uint8_t* slot = scratch + kNoAllocHeader +
                  ((uint64_t)blockIdx.x * kW64Warps + (uint64_t)warp) * kNoAllocSlotBytes;
  while (true) {
    int i = 0;
    if (lane == 0) i = atomicAdd(next, 1);
    i = __shfl_sync(GCL_FULL, i, 0);
    if (i >= A.count) break;
    const int n = (int)(A.voff[i + 1] - A.voff[i]);
    if (n > kW64MaxN) {
      if (lane == 0) A.status[i] = kTooLarge;
      continue;
    }
    w64_canon_one(A, i, slot);
  }
}

}  // namespace gcl

using namespace gcl;

namespace {

struct NoAllocDevice {
  bool ready = false;
  uint8_t* scratch = nullptr;  // device address of g_noalloc_scratch
  int grid = 0;
};
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
NoAllocDevice g_noalloc_dev[kMaxDevices];

// A failed runtime call of the set-up: its error is returned as a status and
// not left behind as the thread's last error, where a later launch check of
// the caller's own work would find it.
int noalloc_fail() {
  (void)cudaGetLastError();
  return GCL_ERR_CUDA;
}

// Once per device, with that device current: resolve the scratch's device
// address and the launch shape.  The result is kept for the life of the
// process; a cudaDeviceReset of the device discards the module that holds the
// array, so the entry point must not be called on a device after a reset.
int noalloc_setup(int dev, NoAllocDevice** out) {
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  NoAllocDevice& d = g_noalloc_dev[dev];
  if (!d.ready) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return noalloc_fail();
    int sms = 0, per_sm = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
      return noalloc_fail();
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, w64_noalloc_kernel, kW64Threads,
                                                      0) != cudaSuccess)
      return noalloc_fail();
    d.scratch = static_cast<uint8_t*>(p);
    d.grid = std::min(kNoAllocSlots / kW64Warps, std::max(1, sms * std::max(per_sm, 1)));
    d.ready = true;
  }
  *out = &d;
  return GCL_OK;
}

}  // namespace

extern "C" int gcl_canon_batch_noalloc(void* stream, int count, const int64_t* d_voff,
                                       const int64_t* d_eoff, const int32_t* d_rowptr,
                                       const int32_t* d_col, const int32_t* d_color,
                                       int max_aut, int max_n, uint8_t* d_out_dense,
                                       const int64_t* d_ooff, int32_t* d_out_label,
                                       int64_t* d_out_stats, int32_t* d_out_status) {
  if (count < 0 || max_aut <= 0 || max_n < 0 || !d_voff || !d_eoff || !d_rowptr ||
      !d_out_status || (d_out_dense && !d_ooff))
    return GCL_ERR_ARG;
  if (max_n > kW64MaxN) return GCL_ERR_TOO_LARGE;  // this entry point: n <= 64 only
  if (count == 0) return GCL_OK;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return noalloc_fail();
  if (dev < 0 || dev >= kMaxDevices) return GCL_ERR_ARG;
  NoAllocDevice* d = nullptr;
  const int rc = noalloc_setup(dev, &d);
  if (rc != GCL_OK) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // A non-sticky error left by the caller's earlier work would otherwise be
  // reported by the launch check below as this call's failure.
  (void)cudaGetLastError();
  // The scratch keeps the previous call's contents; only the work counter
  // must start at zero (representatives and ring entries are written before
  // they are read within each graph's search).
  if (cudaMemsetAsync(d->scratch, 0, kNoAllocHeader, s) != cudaSuccess) return noalloc_fail();

  BatchArgs A;
  A.count = count;
  A.voff = d_voff;
  A.eoff = d_eoff;
  A.rowptr = d_rowptr;
  A.col = d_col;
  A.color = d_color;
  A.order = nullptr;
  A.max_aut = (uint32_t)max_aut;
  A.aut_cap = std::min<uint32_t>((uint32_t)max_aut, kNoAllocRing);
  A.out_dense = d_out_dense;
  A.ooff = d_ooff;
  A.out_rows = nullptr;
  A.roff = nullptr;
  A.out_label = d_out_label;
  A.out_stats = d_out_stats;
  A.status = d_out_status;
  A.work = d->scratch + kNoAllocHeader;
  A.slot_bytes = kNoAllocSlotBytes;
  const char* b = std::getenv("GCL_GRAPH_BUDGET_S");
  const double budget_s = b ? std::atof(b) : 600.0;
  A.budget_ns = budget_s > 0 ? (uint64_t)(budget_s * 1e9) : 0;
  const int grid = (int)std::min<int64_t>(d->grid, ((int64_t)count + kW64Warps - 1) / kW64Warps);
  w64_noalloc_kernel<<<grid, kW64Threads, 0, s>>>(A, d->scratch);
  return cudaGetLastError() == cudaSuccess ? GCL_OK : noalloc_fail();
}
