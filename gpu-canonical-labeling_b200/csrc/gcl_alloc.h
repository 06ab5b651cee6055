// gcl_alloc.h -- every device and pinned host allocation of the library.
//
// A failed allocation is returned to the caller and leaves nothing behind:
// the runtime also records the failure as the thread's last error, which a
// later launch check (cudaGetLastError) would report against a kernel that
// ran fine -- after a wide search that found no workspace falls back to the
// sequential search, for one.  So the record is cleared here.
//
// GCL_FAULT_ALLOC_AT=k in the environment (k >= 1) makes the k-th allocation
// of the process (device and pinned host counted together) fail as out of
// memory, once, without calling the allocator, and says so on stderr
// ("gcl: injected allocation failure k").  It is a test hook for the
// callers' error paths: the call that needed the memory returns
// GCL_ERR_NOMEM (or falls back, where it has a fallback) and the context
// stays usable.  Unset, or not a positive integer: no effect.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <mutex>

namespace gcl {

inline int64_t alloc_fault_target() {
  static const int64_t k = [] {
    const char* s = std::getenv("GCL_FAULT_ALLOC_AT");
    if (!s || !*s) return (int64_t)0;
    char* end = nullptr;
    const long long v = std::strtoll(s, &end, 10);
    return (*end == '\0' && v > 0) ? (int64_t)v : (int64_t)0;
  }();
  return k;
}

// true for the one allocation that is to fail
inline bool alloc_fault_hit() {
  const int64_t k = alloc_fault_target();
  if (k == 0) return false;
  static std::atomic<int64_t> seen{0};
  if (seen.fetch_add(1, std::memory_order_relaxed) + 1 != k) return false;
  std::fprintf(stderr, "gcl: injected allocation failure %lld\n", (long long)k);
  return true;
}

// The library's own stream-ordered memory pool on the current device,
// created on first use, or null (then the device's default pool serves).
// It keeps up to kPoolKeepBytes of freed memory mapped instead of returning
// it to the driver at every synchronization (the default pool's release
// threshold is 0): workspaces that are freed and grown again, as the serving
// lanes' are when a larger graph arrives, then reuse memory instead of
// mapping new memory while other streams are busy.
constexpr uint64_t kPoolKeepBytes = 16ull << 30;
inline cudaMemPool_t library_pool() {
  constexpr int kMaxDev = 64;
  static std::mutex mu;
  static cudaMemPool_t pools[kMaxDev] = {};
  static bool tried[kMaxDev] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDev) {
    (void)cudaGetLastError();
    return nullptr;
  }
  std::lock_guard<std::mutex> lk(mu);
  if (!tried[dev]) {
    tried[dev] = true;
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool = nullptr;
    if (cudaMemPoolCreate(&pool, &props) == cudaSuccess) {
      uint64_t keep = kPoolKeepBytes;
      if (cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep) != cudaSuccess)
        (void)cudaGetLastError();
      pools[dev] = pool;
    } else {
      (void)cudaGetLastError();
    }
  }
  return pools[dev];
}

// stream-ordered device allocation (cudaMallocAsync, from the library's
// pool); *p is null on failure
inline cudaError_t device_alloc(void** p, size_t bytes, cudaStream_t s) {
  *p = nullptr;
  if (alloc_fault_hit()) return cudaErrorMemoryAllocation;
  cudaMemPool_t pool = library_pool();
  const cudaError_t e = pool ? cudaMallocFromPoolAsync(p, bytes, pool, s)
                             : cudaMallocAsync(p, bytes, s);
  if (e != cudaSuccess) {
    *p = nullptr;
    (void)cudaGetLastError();
  }
  return e;
}

// pinned host allocation (cudaHostAlloc); *p is null on failure
inline cudaError_t pinned_alloc(void** p, size_t bytes) {
  *p = nullptr;
  if (alloc_fault_hit()) return cudaErrorMemoryAllocation;
  const cudaError_t e = cudaHostAlloc(p, bytes, cudaHostAllocDefault);
  if (e != cudaSuccess) {
    *p = nullptr;
    (void)cudaGetLastError();
  }
  return e;
}

// pinned host allocation mapped into the device's address space
// (gcl_host_alloc): kernels read and write it in place over the bus; *p and
// *dev are null on failure
inline cudaError_t mapped_alloc(void** p, void** dev, size_t bytes) {
  *p = nullptr;
  *dev = nullptr;
  if (alloc_fault_hit()) return cudaErrorMemoryAllocation;
  cudaError_t e = cudaHostAlloc(p, bytes, cudaHostAllocMapped | cudaHostAllocPortable);
  if (e == cudaSuccess) {
    e = cudaHostGetDevicePointer(dev, *p, 0);
    if (e != cudaSuccess) {
      cudaFreeHost(*p);
      *dev = nullptr;
    }
  }
  if (e != cudaSuccess) {
    *p = nullptr;
    (void)cudaGetLastError();
  }
  return e;
}

}  // namespace gcl
