// gcl_capi.cu -- the C ABI (include/gcl.h) and its host-side context.
//
// Dispatch: every batch first runs the warp-per-graph kernel for n <= 64
// (canon_warp64.cuh).  Graphs it cannot finish are appended to device-side
// lists and picked up by later launches on the same stream, so the batched
// device path never synchronizes with the host:
//   * an automorphism ring that outgrew its per-slot capacity -> rerun with a
//     workspace holding the full max_aut ring;
//   * n > 64 -> the sparse warp-per-graph kernel (canon_sparse.cuh), first
//     with a small pool of per-level orbit arrays and a short ring, then a
//     rerun of the graphs that outgrew them with both at full size.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/gcl.h"
#include "canon_sparse.cuh"
#include "canon_warp64.cuh"
#include "canon_wide.cuh"
#include "gcl_alloc.h"
#include "gcl_batch_check.h"
#include "gcl_group.h"
#include "gcl_guard.h"

namespace gcl {

constexpr uint32_t kW64AutCap = 256;  // ring slots per warp in the fast pass

// Size buckets of the sparse kernel (n > 64): each bucket is one launch whose
// warps stage their per-step arrays in shared memory sized for the bucket's
// largest graph (the last bucket uses device memory only).
constexpr int kSpBuckets = 4;
constexpr uint32_t kSpBucketHi[kSpBuckets] = {256, 1024, 4096, 0xffffffffu};
__host__ __device__ inline int sp_bucket(int64_t n) {
  return n <= 256 ? 0 : n <= 1024 ? 1 : n <= 4096 ? 2 : 3;
}

// Device-side lists of deferred graphs.
struct Deferred {
  int overflow_count;  // n <= 64 graphs that outgrew the ring
  int next_overflow;
  int next;            // work counter of the first pass
  int sp_fail_count;   // n > 64 graphs that outgrew pool or ring
  int next_sp_fail;
  int sp_fail2_count;  // ... and the middle rerun's pool or ring
  int next_sp_fail2;
  int large_count[kSpBuckets];  // n > 64 graphs per size bucket
  int next_large[kSpBuckets];
  int search_count;    // root slots handed to the search queue
  int next_search;     // tickets of the search queue
  int roots_done;      // graphs whose root step is over
};

// Largest graphs first: a counting sort of the graph ids by descending n
// (n > 64 first, they only pass through the warp kernel), so the persistent
// warps do not finish on a few large graphs (longest-processing-time order).
constexpr int kOrderThreads = 1024;
__global__ void __launch_bounds__(kOrderThreads)
    order_by_size_kernel(int count, const int64_t* voff, int* order) {
  constexpr int kBins = kW64MaxN + 2;  // n = 0..64, and every n > 64 in the last bin
  constexpr int kPer = 8;              // graphs per thread and chunk, loaded before use
  __shared__ int hist[kBins];
  __shared__ int start[kBins];
  for (int b = threadIdx.x; b < kBins; b += blockDim.x) hist[b] = 0;
  __syncthreads();
  const int chunk = (int)blockDim.x * kPer;
  // a thread's graphs of a chunk: every size is read before the first is
  // counted, so the reads overlap instead of waiting on each other
  auto bins = [&](int base, int (&bn)[kPer]) {
    int64_t a[kPer], b[kPer];
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
      const int g = base + k * (int)blockDim.x + (int)threadIdx.x;
      a[k] = g < count ? voff[g] : 0;
      b[k] = g < count ? voff[g + 1] : -1;
    }
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
      const int64_t n = b[k] - a[k];
      bn[k] = n < 0 ? -1 : (n > kW64MaxN ? kW64MaxN + 1 : (int)n);
    }
  };
  for (int base = 0; base < count; base += chunk) {
    int bn[kPer];
    bins(base, bn);
#pragma unroll
    for (int k = 0; k < kPer; ++k)
      if (bn[k] >= 0) atomicAdd(&hist[bn[k]], 1);
  }
  __syncthreads();
  if (threadIdx.x == 0) {  // starts, largest bin first
    int run = 0;
    for (int b = kBins - 1; b >= 0; --b) {
      start[b] = run;
      run += hist[b];
    }
  }
  __syncthreads();
  for (int base = 0; base < count; base += chunk) {
    int bn[kPer];
    bins(base, bn);
#pragma unroll
    for (int k = 0; k < kPer; ++k)
      if (bn[k] >= 0) order[atomicAdd(&start[bn[k]], 1)] = base + k * (int)blockDim.x + (int)threadIdx.x;
  }
}

constexpr int kSpSmemPerBlock = 200 * 1024;  // dynamic shared memory cap of one sparse block
constexpr uint32_t kWidePool = 64;  // per-level orbit arrays of a wide-search warp
constexpr uint64_t kWideStoreBytes = 1ull << 30;  // automorphism store of a wide search
constexpr uint64_t kWideStoreEntries = 1ull << 22;  // ... and at most this many entries
constexpr uint32_t kWideFixCap = 4096;  // entries whose fix state a wide-search warp keeps
constexpr uint64_t kGroupWorkCap = 40000000000ull;  // Schreier-Sims operations (~25 s)
// the check of a search's group order: Schreier-Sims operations for each of
// the general and the known-base completion (~0.3 s and ~0.6 s)
constexpr uint64_t kGroupCheckCap = 400000000ull;

// entries of a wide search's automorphism store: max_aut, within kWideStoreBytes
static uint32_t wide_store_cap(uint32_t n, int max_aut) {
  const uint64_t per_aut = 2ull * ((uint64_t)n + 2);
  return (uint32_t)std::max<uint64_t>(
      1, std::min<uint64_t>(std::min<uint64_t>((uint64_t)max_aut, kWideStoreBytes / per_aut),
                            kWideStoreEntries));
}
// Per-level orbit arrays and automorphism-ring entries of the sparse passes:
// the first pass (n <= 4096 / larger), then a middle rerun of the graphs
// that outgrew them, then a rerun with a full-size pool and ring.  Each
// tier's slots are smaller than the next one's, so more warps fit in the
// workspace budget.
constexpr uint32_t kSpPool = 32, kSpPoolHuge = 8;
constexpr uint32_t kSpAutCap = 256, kSpAutCapHuge = 64;
constexpr uint32_t kSpPoolMid = 256, kSpAutCapMid = 2048;

__global__ void __launch_bounds__(kSpThreads, 5)
    sp_batch_kernel(BatchArgs A, const int* list, const int* count, int* next, int* fail_list,
                    int* fail_count, uint32_t n_max, uint64_t m2_max, uint32_t pool, uint32_t cap,
                    uint64_t slot_bytes, uint64_t smem_per_warp) {
  extern __shared__ __align__(16) uint8_t sp_dyn[];
  const int warp = (int)(threadIdx.x >> 5);
  const uint32_t lane = lane_id();
  uint8_t* slot = A.work + ((uint64_t)blockIdx.x * kSpWarps + (uint64_t)warp) * slot_bytes;
  uint8_t* smem = smem_per_warp ? sp_dyn + (uint64_t)warp * smem_per_warp : nullptr;
  const SpLayout Lo = sp_layout(n_max, m2_max, pool, cap);
  const int total = *(volatile const int*)count;
  while (true) {
    int i = 0;
    if (lane == 0) i = atomicAdd(next, 1);
    i = __shfl_sync(GCL_FULL, i, 0);
    if (i >= total) break;
    const int g = list[i];
    const int64_t n = A.voff[g + 1] - A.voff[g];
    const int64_t m2 = A.eoff[g + 1] - A.eoff[g];
    if (n > (int64_t)n_max || m2 > (int64_t)m2_max) {
      if (lane == 0) A.status[g] = kTooLarge;
      continue;
    }
    const SpResult r = sp_search(A, g, slot, Lo, pool, cap, smem, smem_per_warp);
    if (lane == 0) {
      A.status[g] = r.status;
      if (A.out_stats) {
        A.out_stats[2 * (int64_t)g] = r.num_aut;
        A.out_stats[2 * (int64_t)g + 1] = r.nodes;
      }
      if (r.status == kAutOverflow && fail_list) fail_list[atomicAdd(fail_count, 1)] = g;
    }
    if (r.status == kOk) sp_write_outputs(A, g);
    __syncwarp();
  }
}

__global__ void __launch_bounds__(kW64Threads, 8)
    w64_batch_kernel(BatchArgs A, Deferred* D, int* overflow_list, int* large_list, int pass) {
  const int warp = (int)(threadIdx.x >> 5);
  const uint32_t lane = lane_id();
  uint8_t* slot = A.work + ((uint64_t)blockIdx.x * kW64Warps + (uint64_t)warp) * A.slot_bytes;
  int* ctr = pass == 0 ? &D->next : &D->next_overflow;
  const int total = pass == 0 ? A.count : *(volatile int*)&D->overflow_count;
  while (true) {
    int i = 0;
    if (lane == 0) i = atomicAdd(ctr, 1);
    i = __shfl_sync(GCL_FULL, i, 0);
    if (i >= total) break;
    const int g = pass == 0 ? (A.order ? A.order[i] : i) : overflow_list[i];
    const int n = (int)(A.voff[g + 1] - A.voff[g]);
    if (n > kW64MaxN) {
      if (lane == 0) {
        A.status[g] = kTooLarge;
        const int bk = sp_bucket(n);
        large_list[(int64_t)bk * A.count + atomicAdd(&D->large_count[bk], 1)] = g;
      }
      continue;
    }
    w64_canon_one(A, g, slot);
    if (pass == 0 && lane == 0 && *(volatile int32_t*)&A.status[g] == kAutOverflow)
      overflow_list[atomicAdd(&D->overflow_count, 1)] = g;
    __syncwarp();
  }
}

// A searched graph's results: status, counters, a ring that outgrew the
// first pass's store goes to the full-ring rerun, and the outputs.
__device__ __forceinline__ void w64_finish_search(const BatchArgs& A, Deferred* D,
                                                  int* overflow_list, int g, int n, int64_t vo,
                                                  const W64Result& r) {
  if (lane_id() == 0) {
    A.status[g] = r.status;
    if (A.out_stats) {
      A.out_stats[2 * (int64_t)g] = r.num_aut;
      A.out_stats[2 * (int64_t)g + 1] = r.nodes;
    }
    if (r.status == kAutOverflow) overflow_list[atomicAdd(&D->overflow_count, 1)] = g;
  }
  if (r.status == kOk) w64_write_outputs(A, g, n, vo);
  __syncwarp();
}

// Bounded waits of the search queue (iterations of a sleep of at most 1 us):
// every wait is for a root refinement that a running warp has claimed and
// finishes without waiting itself.
constexpr int kW64QueueWait = 1 << 22;

// The batch's graphs of up to 64 vertices in one pipelined launch.
//
// Roots: every warp takes graphs in the order given (largest first), loads
// each and refines its root partition -- the largest share of the work on
// small sparse graphs.  A graph whose root partition is discrete is finished
// there (its canonical form is the root's).  A graph of search-cost class
// kW64InlineClass or more is searched at once by the same warp, so the
// longest searches of the batch start in its first microseconds; any other
// graph leaves its root partition in a slot of `roots` and flags it ready.
// Searches: a warp that finds no root left takes a ticket, waits until the
// ticket's slot is flagged (or every root is done and the ticket is past the
// last slot) and searches below it.  A warp never waits on a search, only on
// a root refinement a running warp has claimed, so the launch needs no
// co-residency.  Results equal w64_batch_kernel's.
// Six resident blocks per SM (up to 80 registers per thread): measured on the
// batched small-graph workload against 8 (64 registers, spills across the
// inlined phases), 7, 5 and 4 blocks, six gave the shortest launch (0.327
// against 0.372 ms at eight): its warps run the long searches faster.
__global__ void __launch_bounds__(kW64Threads, 6)
    w64_pipe_kernel(BatchArgs A, Deferred* D, int* large_list, int* overflow_list,
                    uint8_t* roots, int* ready) {
  const int warp = (int)(threadIdx.x >> 5);
  const uint32_t lane = lane_id();
  uint8_t* slot = A.work + ((uint64_t)blockIdx.x * kW64Warps + (uint64_t)warp) * A.slot_bytes;
  while (true) {
    int i = 0;
    if (lane == 0) i = atomicAdd(&D->next, 1);
    i = __shfl_sync(GCL_FULL, i, 0);
    if (i >= A.count) break;
    const int g = A.order ? A.order[i] : i;
    const int64_t vo = A.voff[g];
    const int n = (int)(A.voff[g + 1] - vo);
    if (n > kW64MaxN) {
      if (lane == 0) {
        A.status[g] = kTooLarge;
        const int bk = sp_bucket(n);
        large_list[(int64_t)bk * A.count + atomicAdd(&D->large_count[bk], 1)] = g;
        __threadfence();
        atomicAdd(&D->roots_done, 1);
      }
      continue;
    }
    W64Root root{0ull, 0, kOk};
    bool search = false;
    if (n > 0) {
      const int64_t eo = A.eoff[g];
      root = w64_root(A, n, vo, eo, A.eoff[g + 1] - eo, A.rowptr + vo + g);
      search = root.status == kOk && root.starts != low_mask((uint32_t)n);
    }
    if (search && w64_cost_class(n, root.starts) >= kW64InlineClass) {
      if (lane == 0) {
        __threadfence();
        atomicAdd(&D->roots_done, 1);
      }
      const W64Result r = w64_search_tree(A, n, root.starts, root.code, slot, w64_deadline(A));
      w64_finish_search(A, D, overflow_list, g, n, vo, r);
      continue;
    }
    if (search) {
      int j = 0;
      if (lane == 0) j = atomicAdd(&D->search_count, 1);
      j = __shfl_sync(GCL_FULL, j, 0);
      w64_save_root(roots + (uint64_t)j * w64_root_slot_bytes(), g, n, root.starts, root.code);
      if (lane == 0) A.status[g] = kInternal;  // until its search ends
      __threadfence();
      __syncwarp();
      if (lane == 0) atomicExch(&ready[j], 1);
    } else {
      // finished at the root: the discrete root is the first and best leaf
      // (first_terminal, sequential.cpp:259-303), one node, no automorphism
      if (root.status == kOk && n > 0) {
        W64Smem& S = w64_smem();
        const Rows2 R = w64_leaf_rows(n);
        w64_store_leaf(n, R, S.best_cert, S.bpos);
      }
      if (lane == 0) {
        A.status[g] = root.status;
        if (A.out_stats) {
          A.out_stats[2 * (int64_t)g] = 0;
          A.out_stats[2 * (int64_t)g + 1] = 1;
        }
      }
      if (root.status == kOk) w64_write_outputs(A, g, n, vo);
      __syncwarp();
    }
    if (lane == 0) {
      __threadfence();
      atomicAdd(&D->roots_done, 1);
    }
  }
  while (true) {
    int t = 0;
    if (lane == 0) t = atomicAdd(&D->next_search, 1);
    t = __shfl_sync(GCL_FULL, t, 0);
    int ok = 0;
    if (lane == 0) {
      uint32_t nap = 32;
      int it = 0;
      for (; it < kW64QueueWait; ++it) {
        if (*(volatile int*)&D->search_count > t) {
          ok = 1;
          break;
        }
        if (*(volatile int*)&D->roots_done >= A.count) {
          __threadfence();  // every slot taken before the last root is seen
          ok = *(volatile int*)&D->search_count > t ? 1 : 0;
          break;
        }
        __nanosleep(nap);
        if (nap < 1024) nap <<= 1;
      }
      if (ok) {
        int k = 0;
        while (!*(volatile int*)&ready[t] && k < kW64QueueWait) {
          __nanosleep(64);
          ++k;
        }
        if (k == kW64QueueWait) ok = 0;  // the slot's graph keeps its internal-error status
        __threadfence();
      }
    }
    ok = __shfl_sync(GCL_FULL, ok, 0);
    if (!ok) break;
    const uint8_t* root = roots + (uint64_t)t * w64_root_slot_bytes();
    const int g = w64_root_graph(root);
    const int64_t vo = A.voff[g];
    const int n = (int)(A.voff[g + 1] - vo);
    int code = 0;
    const uint64_t starts = w64_restore_root(root, n, &code);
    const W64Result r = w64_search_tree(A, n, starts, code, slot, w64_deadline(A));
    w64_finish_search(A, D, overflow_list, g, n, vo, r);
  }
}

}  // namespace gcl

using namespace gcl;

namespace {

// Device buffer allocated in stream order on its context's stream: growing
// or freeing it never waits for the rest of the device (a cudaFree would,
// stalling every other context's work -- the serving loop runs several).
struct DevBuf {
  void* p = nullptr;
  size_t cap = 0;
  cudaStream_t stream = nullptr;
  cudaError_t ensure(size_t bytes) {
    if (bytes <= cap && p) return cudaSuccess;
    // grow by half again at least, so that a growing buffer is replaced
    // only a logarithmic number of times
    const size_t want = std::max<size_t>(std::max<size_t>(bytes, 256), cap + cap / 2);
    if (p) cudaFreeAsync(p, stream);
    p = nullptr;
    cap = 0;
    cudaError_t e = device_alloc(&p, want, stream);
    if (e == cudaSuccess) cap = want;
    return e;
  }
  void release() {
    if (p) cudaFreeAsync(p, stream);
    p = nullptr;
    cap = 0;
  }
};

// A host-pointer entry point that returns early (an error, or an exception)
// may leave copies from or to the caller's buffers queued on its stream, and
// the caller may reuse or free those buffers once the call has returned: the
// stream is drained first.  A call that completed has synchronized already
// and sets `done`.
struct DrainOnExit {
  cudaStream_t s;
  bool done = false;
  explicit DrainOnExit(cudaStream_t st) : s(st) {}
  ~DrainOnExit() {
    if (!done) cudaStreamSynchronize(s);
  }
};

}  // namespace

struct gcl_context {
  int device = 0;
  int sms = 0;
  cudaStream_t stream = nullptr;
  int w64_grid = 0;
  // fast-pass workspace
  DevBuf work;
  // rerun workspace (full max_aut ring), sized on demand
  DevBuf work_big;
  uint32_t work_big_aut = 0;
  int big_slots = 0;
  DevBuf sp_work[kSpBuckets], sp_work_mid, sp_work_big;
  // wide search of one graph: shared region and per-warp slots
  DevBuf wide_sh, wide_slots;
  template <typename F>
  void each_buf(F f) {
    for (DevBuf& b : sp_work) f(b);
    DevBuf* bufs[] = {&work, &work_big, &sp_work_mid, &sp_work_big, &deferred, &wide_sh,
                      &wide_slots,
                      &overflow_list, &large_list, &sp_fail_list, &sp_fail_list2, &order,
                      &roots, &ready,
                      &voff, &eoff,
                      &rowptr, &col, &color, &ooff, &dense, &roff, &rows, &label, &stats,
                      &status};
    for (DevBuf* b : bufs) f(*b);
  }
  int64_t wide_min_n = kW64MaxN + 1;
  uint64_t workspace_bytes = 0;  // per-pass workspace cap, 0 = GCL_WORKSPACE_GB
  int64_t wide_max_warps = 0;    // 0 = as many as fit
  bool smem_stage = true;        // sparse and wide kernels stage per-step arrays in shared memory
  int wide_gate = 1;             // wide search's level gate: 1 on, 0 off, 2 automatic
  bool wide_share = false;       // wide search: busy warps hand subtrees to idle ones
  bool wide_count = false;       // wide search: the items kernel's counters (GCL_OPT_COUNTERS)
  uint32_t wide_pool = kWidePool;  // wide search: per-level orbit arrays of a warp
  bool wide_probe = true;          // wide search: a level's first item runs before the rest
  uint64_t handoff_ns = 0;         // gcl_canon_batch: batch-warp budget before the wide search
  bool batch_split = false;        // gcl_canon_batch: large small-graph batches in two halves
  gcl_context* peer = nullptr;     // the second half's context (own stream and workspace)
  cudaEvent_t split_ev = nullptr;  // orders the companion stream after this one
  uint64_t budget_override_ns = 0; // per-graph budget of the next batched launch (0 = default)
  // mapped host buffers (gcl_host_alloc): host address, size, device address
  struct Mapped {
    uint8_t* p;
    size_t bytes;
    uint8_t* dev;
  };
  std::vector<Mapped> mapped;
  bool counted = false;          // the last wide search was counted
  // launch shape per size bucket (gcl_autotune / gcl_set_tuning): 0 / -1 = default
  int w64_per_sm = 0;            // resident blocks the warp kernel's occupancy allows
  int pipe_per_sm = 0;           // ... and the pipelined warp kernel's
  int tune_w64_bps = 0;
  int tune_sp_bps[kSpBuckets] = {0, 0, 0, 0};
  int tune_sp_stage[kSpBuckets] = {-1, -1, -1, -1};
  // timing of the passes of one batch (autotuner)
  bool timing = false;
  cudaEvent_t tev[2][1 + kSpBuckets] = {};
  bool tev_used[1 + kSpBuckets] = {};
  DevBuf deferred, overflow_list, large_list, sp_fail_list, sp_fail_list2, order;
  // the warp kernel's root slots and their ready flags (root -> search hand-over)
  DevBuf roots, ready;
  // staging for host-pointer calls
  DevBuf voff, eoff, rowptr, col, color, ooff, dense, roff, rows, label, stats, status;
};

// Per-graph time budget of the search loop (GCL_GRAPH_BUDGET_S, default
// 600 s); a graph that exceeds it reports GCL_ERR_TIMEOUT instead of holding
// its warp forever.
static uint64_t graph_budget_ns() {
  const char* e = std::getenv("GCL_GRAPH_BUDGET_S");
  double s = e ? std::atof(e) : 600.0;
  if (!(s > 0)) return 0;
  return (uint64_t)(s * 1e9);
}

// Device memory the per-warp workspaces of one pass may take
// (GCL_WORKSPACE_GB, default 4 GiB).
static uint64_t workspace_budget() {
  const char* e = std::getenv("GCL_WORKSPACE_GB");
  double g = e ? std::atof(e) : 4.0;
  if (!(g > 0)) g = 4.0;
  return (uint64_t)(g * (1ull << 30));
}

static uint64_t ctx_workspace(const gcl_context* c) {
  return c->workspace_bytes ? c->workspace_bytes : workspace_budget();
}

static_assert(kBatchSmallN == kW64MaxN, "the host checks and the warp kernel agree on small n");

// the items kernel of the wide search: with or without work sharing, with
// or without its counters
static void (*wide_items_fn(bool share, bool count))(WideArgs) {
  if (share) return count ? wide_items_kernel<true, true> : wide_items_kernel<true, false>;
  return count ? wide_items_kernel<false, true> : wide_items_kernel<false, false>;
}

static int cuda_status(cudaError_t e) {
  if (e == cudaSuccess) return GCL_OK;
  if (e == cudaErrorMemoryAllocation) return GCL_ERR_NOMEM;
  return GCL_ERR_CUDA;
}
#define GCL_TRY(x)                          \
  do {                                      \
    cudaError_t e_ = (x);                   \
    if (e_ != cudaSuccess) return cuda_status(e_); \
  } while (0)

extern "C" {

const char* gcl_status_string(int s) {
  switch (s) {
    case GCL_OK: return "ok";
    case GCL_ERR_ARG: return "invalid argument";
    case GCL_ERR_CUDA: return "CUDA error";
    case GCL_ERR_NOMEM: return "out of memory";
    case GCL_ERR_BAD_INPUT: return "bad input graph (loop, duplicate or one-directional edge)";
    case GCL_ERR_TOO_LARGE: return "graph too large";
    case GCL_ERR_TIMEOUT: return "bounded device wait timed out";
    default: return "internal error";
  }
}

int gcl_version(void) { return 100; }

int gcl_create(int device, gcl_context** out) try {
  if (!out) return GCL_ERR_ARG;
  *out = nullptr;
  int ndev = 0;
  GCL_TRY(cudaGetDeviceCount(&ndev));
  if (device < 0 || device >= ndev) return GCL_ERR_ARG;
  GCL_TRY(cudaSetDevice(device));
  gcl_context* c = new (std::nothrow) gcl_context();
  if (!c) return GCL_ERR_NOMEM;
  c->device = device;
  cudaError_t e = cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) {
    c->each_buf([&](DevBuf& b) { b.stream = c->stream; });
    // keep freed stream-ordered memory in the device's default pool instead
    // of returning it at every synchronization (it is reused by the next
    // allocation of this process)
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
      uint64_t keep = ~0ull;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    // an optional setting: a failure above must not surface in a later
    // launch check as the thread's last error
    (void)cudaGetLastError();
  }
  int per_sm = 0;
  if (e == cudaSuccess)
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, w64_batch_kernel, kW64Threads, 0);
  if (e == cudaSuccess) {
    // GCL_W64_BLOCKS_PER_SM caps the resident blocks of the warp kernel (fewer
    // warps per SM run each graph faster; more hide more latency)
    const char* cap_env = std::getenv("GCL_W64_BLOCKS_PER_SM");
    if (cap_env && std::atoi(cap_env) > 0) per_sm = std::min(per_sm, std::atoi(cap_env));
    c->w64_per_sm = std::max(per_sm, 1);
    c->w64_grid = c->sms * std::max(per_sm, 1);
    int pipe = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&pipe, w64_pipe_kernel, kW64Threads, 0);
    c->pipe_per_sm = std::max(std::min(pipe, c->w64_per_sm), 1);
  }
  if (e == cudaSuccess) e = c->deferred.ensure(sizeof(Deferred));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(sp_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             kSpSmemPerBlock);
  for (int share = 0; share < 2 && e == cudaSuccess; ++share)
    for (int count = 0; count < 2 && e == cudaSuccess; ++count)
      e = cudaFuncSetAttribute(wide_items_fn(share != 0, count != 0),
                               cudaFuncAttributeMaxDynamicSharedMemorySize, kSpSmemPerBlock);
  if (e != cudaSuccess) {
    c->deferred.release();
    if (c->stream) {
      cudaStreamSynchronize(c->stream);
      cudaStreamDestroy(c->stream);
    }
    delete c;
    return cuda_status(e);
  }
  *out = c;
  return GCL_OK;
} GCL_CATCH_ALL

int gcl_destroy(gcl_context* c) {
  if (!c) return GCL_ERR_ARG;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->peer) gcl_destroy(c->peer);
  c->peer = nullptr;
  cudaSetDevice(c->device);
  if (c->split_ev) cudaEventDestroy(c->split_ev);
  for (auto& row : c->tev)
    for (cudaEvent_t& ev : row)
      if (ev) cudaEventDestroy(ev);
  c->each_buf([](DevBuf& b) { b.release(); });
  if (c->stream) {
    cudaStreamSynchronize(c->stream);
    cudaStreamDestroy(c->stream);
  }
  for (const auto& h : c->mapped) cudaFreeHost(h.p);
  delete c;
  return GCL_OK;
}

void* gcl_stream(gcl_context* c) { return c ? (void*)c->stream : nullptr; }

int gcl_sync(gcl_context* c) {
  if (!c) return GCL_ERR_ARG;
  GCL_TRY(cudaStreamSynchronize(c->stream));
  return GCL_OK;
}

int gcl_wide_counters(gcl_context* c, int64_t* out, int cap) {
  if (!c || !out || cap < 0) return GCL_ERR_ARG;
  if (!c->counted || !c->wide_sh.p) return GCL_ERR_ARG;  // no counted search yet
  // the header is the first region of the search's device block (offset 0)
  GCL_TRY(cudaSetDevice(c->device));
  unsigned long long v[kWideCounters];
  GCL_TRY(cudaMemcpyAsync(v, (const uint8_t*)c->wide_sh.p + offsetof(WideHdr, cnt), sizeof v,
                          cudaMemcpyDeviceToHost, c->stream));
  GCL_TRY(cudaStreamSynchronize(c->stream));
  const int k = cap < (int)kWideCounters ? cap : (int)kWideCounters;
  for (int i = 0; i < k; ++i) out[i] = (int64_t)v[i];
  return k;
}

int gcl_canon_batch_device_async(gcl_context* c, int count, const int64_t* d_voff,
                                 const int64_t* d_eoff, const int32_t* d_rowptr,
                                 const int32_t* d_col, const int32_t* d_color, int max_aut,
                                 int max_n, int64_t max_m2, uint8_t* d_out_dense,
                                 const int64_t* d_ooff, uint64_t* d_out_rows,
                                 const int64_t* d_roff,
                                 int32_t* d_out_label, int64_t* d_out_stats,
                                 int32_t* d_out_status) try {
  if (!c || count < 0 || max_aut <= 0 || !d_voff || !d_eoff || !d_rowptr || !d_out_status ||
      (d_out_dense && !d_ooff) || (d_out_rows && !d_roff) || max_n < 0 || max_n > GCL_MAX_N)
    return GCL_ERR_ARG;
  if (count == 0) return GCL_OK;
  GCL_TRY(cudaSetDevice(c->device));
  const uint32_t maut = (uint32_t)max_aut;
  const uint32_t cap = std::min<uint32_t>(maut, kW64AutCap);
  const uint64_t slot_bytes = w64_slot_bytes(cap);
  const uint64_t slots = (uint64_t)c->w64_grid * kW64Warps;
  GCL_TRY(c->work.ensure(slots * slot_bytes));
  GCL_TRY(c->overflow_list.ensure((size_t)count * sizeof(int)));
  GCL_TRY(c->large_list.ensure((size_t)count * kSpBuckets * sizeof(int)));
  GCL_TRY(c->order.ensure((size_t)count * sizeof(int)));
  if (max_n > 0) {
    GCL_TRY(c->roots.ensure((size_t)count * w64_root_slot_bytes()));
    GCL_TRY(c->ready.ensure((size_t)count * sizeof(int)));
    GCL_TRY(cudaMemsetAsync(c->ready.p, 0, (size_t)count * sizeof(int), c->stream));
  }
  GCL_TRY(cudaMemsetAsync(c->deferred.p, 0, sizeof(Deferred), c->stream));
  order_by_size_kernel<<<1, kOrderThreads, 0, c->stream>>>(count, d_voff, (int*)c->order.p);
  GCL_TRY(cudaGetLastError());

  BatchArgs A;
  std::memset(&A, 0, sizeof A);
  A.count = count;
  A.voff = d_voff;
  A.eoff = d_eoff;
  A.rowptr = d_rowptr;
  A.col = d_col;
  A.color = d_color;
  A.order = (const int32_t*)c->order.p;
  A.max_aut = maut;
  A.aut_cap = cap;
  A.out_dense = d_out_dense;
  A.ooff = d_ooff;
  A.out_rows = d_out_rows;
  A.roff = d_roff;
  A.out_label = d_out_label;
  A.out_stats = d_out_stats;
  A.status = d_out_status;
  A.work = (uint8_t*)c->work.p;
  A.slot_bytes = slot_bytes;
  A.budget_ns = c->budget_override_ns ? c->budget_override_ns : graph_budget_ns();
  Deferred* D = (Deferred*)c->deferred.p;
  const int64_t w64_grid = c->tune_w64_bps > 0
                               ? (int64_t)c->sms * std::min(c->tune_w64_bps, c->w64_per_sm)
                               : (int64_t)c->w64_grid;
  const int grid1 = (int)std::min<int64_t>(w64_grid, ((int64_t)count + kW64Warps - 1) / kW64Warps);
  if (c->timing) {
    for (int k = 0; k <= kSpBuckets; ++k) c->tev_used[k] = false;
    GCL_TRY(cudaEventRecord(c->tev[0][0], c->stream));
  }
  if (max_n > 0) {
    // root refinements, then the searches below the roots that are not
    // discrete, in one launch
    const int pipe_bps = c->tune_w64_bps > 0 ? std::min(c->tune_w64_bps, c->pipe_per_sm)
                                             : c->pipe_per_sm;
    const int gridp = (int)std::min<int64_t>((int64_t)c->sms * pipe_bps,
                                             ((int64_t)count + kW64Warps - 1) / kW64Warps);
    w64_pipe_kernel<<<gridp, kW64Threads, 0, c->stream>>>(A, D, (int*)c->large_list.p,
                                                          (int*)c->overflow_list.p,
                                                          (uint8_t*)c->roots.p,
                                                          (int*)c->ready.p);
  } else {
    // a batch of empty graphs (max_n 0): one pass, no hand-over buffers
    w64_batch_kernel<<<grid1, kW64Threads, 0, c->stream>>>(A, D, (int*)c->overflow_list.p,
                                                           (int*)c->large_list.p, 0);
  }
  GCL_TRY(cudaGetLastError());
  if (c->timing) {
    GCL_TRY(cudaEventRecord(c->tev[1][0], c->stream));
    c->tev_used[0] = true;
  }

  if (cap < maut) {
    // graphs whose ring outgrew `cap`: rerun with the full ring
    if (c->work_big_aut < maut || !c->work_big.p) {
      // few graphs outgrow the first ring (at most n - 1 = 63 automorphisms
      // were stored on every graph of up to 64 vertices tried), so a few
      // blocks take them: the full-size ring costs about 0.7 MB per warp
      c->big_slots = std::min(std::max(c->sms, 1), 16);
      GCL_TRY(c->work_big.ensure((uint64_t)c->big_slots * kW64Warps * w64_slot_bytes(maut)));
      c->work_big_aut = maut;
    }
    BatchArgs B = A;
    B.aut_cap = maut;
    B.work = (uint8_t*)c->work_big.p;
    B.slot_bytes = w64_slot_bytes(maut);
    w64_batch_kernel<<<c->big_slots, kW64Threads, 0, c->stream>>>(
        B, D, (int*)c->overflow_list.p, (int*)c->large_list.p, 1);
    GCL_TRY(cudaGetLastError());
  }

  if (max_n > kW64MaxN) {
    // graphs with n > 64: one sparse pass per size bucket, then a rerun of
    // the graphs that outgrew the first passes' orbit pool or ring
    const uint64_t m2max = (uint64_t)std::max<int64_t>(max_m2, 1);
    const uint32_t cap1 = std::min<uint32_t>(maut, max_n <= 4096 ? kSpAutCap : kSpAutCapHuge);
    const uint32_t pool1 = max_n <= 4096 ? kSpPool : kSpPoolHuge;
    const uint64_t budget = ctx_workspace(c);
    GCL_TRY(c->sp_fail_list.ensure((size_t)count * sizeof(int)));
    GCL_TRY(c->sp_fail_list2.ensure((size_t)count * sizeof(int)));
    for (int bk = 0; bk < kSpBuckets; ++bk) {
      const uint32_t lo = bk == 0 ? (uint32_t)kW64MaxN + 1 : kSpBucketHi[bk - 1] + 1;
      if ((uint32_t)max_n < lo) break;
      const uint32_t nmax = std::min<uint32_t>((uint32_t)max_n, kSpBucketHi[bk]);
      const uint64_t sb1 = sp_layout(nmax, m2max, pool1, cap1).bytes;
      const bool stage = c->tune_sp_stage[bk] >= 0 ? c->tune_sp_stage[bk] != 0 : c->smem_stage;
      uint64_t smw = stage ? sp_smem_bytes(nmax) : 0;
      if (smw * kSpWarps > (uint64_t)kSpSmemPerBlock) smw = 0;  // device memory only
      int per_sm = 0;
      GCL_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sp_batch_kernel, kSpThreads,
                                                            (size_t)(smw * kSpWarps)));
      if (c->tune_sp_bps[bk] > 0) per_sm = std::min(per_sm, c->tune_sp_bps[bk]);
      int64_t slots = std::min<int64_t>((int64_t)c->sms * std::max(per_sm, 1) * kSpWarps,
                                        std::max<int64_t>(kSpWarps, (int64_t)(budget / sb1)));
      slots = std::min<int64_t>(slots, ((int64_t)count + kSpWarps - 1) / kSpWarps * kSpWarps);
      slots = std::max<int64_t>(kSpWarps, slots / kSpWarps * kSpWarps);
      DevBuf& wb = c->sp_work[bk];
      GCL_TRY(wb.ensure((size_t)(slots * sb1)));
      BatchArgs Sa = A;
      Sa.work = (uint8_t*)wb.p;
      if (c->timing) GCL_TRY(cudaEventRecord(c->tev[0][1 + bk], c->stream));
      sp_batch_kernel<<<(int)(slots / kSpWarps), kSpThreads, (size_t)(smw * kSpWarps),
                        c->stream>>>(Sa, (const int*)c->large_list.p + (int64_t)bk * count,
                                     &D->large_count[bk], &D->next_large[bk],
                                     (int*)c->sp_fail_list.p, &D->sp_fail_count, nmax, m2max,
                                     pool1, cap1, sb1, smw);
      GCL_TRY(cudaGetLastError());
      if (c->timing) {
        GCL_TRY(cudaEventRecord(c->tev[1][1 + bk], c->stream));
        c->tev_used[1 + bk] = true;
      }
    }
    // middle rerun: a larger pool and ring, still many warps
    const uint32_t nmax = (uint32_t)max_n;
    {
      const uint32_t poolm = std::min<uint32_t>(nmax + 2, kSpPoolMid);
      const uint32_t capm = std::min<uint32_t>(maut, kSpAutCapMid);
      const uint64_t sbm = sp_layout(nmax, m2max, poolm, capm).bytes;
      int per_sm = 0;
      GCL_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sp_batch_kernel, kSpThreads, 0));
      int64_t slotsm = std::min<int64_t>((int64_t)c->sms * std::max(per_sm, 1) * kSpWarps,
                                         (int64_t)(budget / sbm));
      slotsm = std::min<int64_t>(slotsm, ((int64_t)count + kSpWarps - 1) / kSpWarps * kSpWarps);
      slotsm = std::max<int64_t>(kSpWarps, slotsm / kSpWarps * kSpWarps);
      GCL_TRY(c->sp_work_mid.ensure((size_t)(slotsm * sbm)));
      BatchArgs Sm = A;
      Sm.work = (uint8_t*)c->sp_work_mid.p;
      sp_batch_kernel<<<(int)(slotsm / kSpWarps), kSpThreads, 0, c->stream>>>(
          Sm, (const int*)c->sp_fail_list.p, &D->sp_fail_count, &D->next_sp_fail,
          (int*)c->sp_fail_list2.p, &D->sp_fail2_count, nmax, m2max, poolm, capm, sbm, 0);
      GCL_TRY(cudaGetLastError());
    }
    // last rerun with a representative array per level and the full ring
    const uint32_t pool2 = nmax + 2;
    const uint64_t sb2 = sp_layout(nmax, m2max, pool2, maut).bytes;
    int64_t slots2 = std::max<int64_t>(1, std::min<int64_t>((int64_t)c->sms,
                                                          (int64_t)(budget / (sb2 * kSpWarps))));
    GCL_TRY(c->sp_work_big.ensure((size_t)(slots2 * kSpWarps * sb2)));
    BatchArgs Sb = A;
    Sb.work = (uint8_t*)c->sp_work_big.p;
    sp_batch_kernel<<<(int)slots2, kSpThreads, 0, c->stream>>>(
        Sb, (const int*)c->sp_fail_list2.p, &D->sp_fail2_count, &D->next_sp_fail2, nullptr,
        nullptr,
        nmax, m2max, pool2, maut, sb2, 0);
    GCL_TRY(cudaGetLastError());
  }
  return GCL_OK;
} GCL_CATCH_ALL

int gcl_set_option(gcl_context* c, int option, int64_t value) {
  if (!c) return GCL_ERR_ARG;
  switch (option) {
    case GCL_OPT_WIDE_MIN_N:
      if (value < 1) return GCL_ERR_ARG;
      c->wide_min_n = value;
      return GCL_OK;
    case GCL_OPT_WORKSPACE_BYTES:
      if (value < 0) return GCL_ERR_ARG;
      c->workspace_bytes = (uint64_t)value;
      return GCL_OK;
    case GCL_OPT_WIDE_MAX_WARPS:
      if (value < 0) return GCL_ERR_ARG;
      c->wide_max_warps = value;
      return GCL_OK;
    case GCL_OPT_SMEM_STAGE:
      if (value != 0 && value != 1) return GCL_ERR_ARG;
      c->smem_stage = value != 0;
      return GCL_OK;
    case GCL_OPT_WIDE_GATE:
      if (value < 0 || value > 2) return GCL_ERR_ARG;
      c->wide_gate = (int)value;
      return GCL_OK;
    case GCL_OPT_WIDE_SHARE:
      if (value != 0 && value != 1) return GCL_ERR_ARG;
      c->wide_share = value != 0;
      return GCL_OK;
    case GCL_OPT_COUNTERS:
      if (value != 0 && value != 1) return GCL_ERR_ARG;
      c->wide_count = value != 0;
      return GCL_OK;
    case GCL_OPT_WIDE_PROBE:
      if (value != 0 && value != 1) return GCL_ERR_ARG;
      c->wide_probe = value != 0;
      return GCL_OK;
    case GCL_OPT_BATCH_HANDOFF_MS:
      if (value < 0) return GCL_ERR_ARG;
      c->handoff_ns = (uint64_t)value * 1000000ull;
      return GCL_OK;
    case GCL_OPT_BATCH_SPLIT:
      if (value != 0 && value != 1) return GCL_ERR_ARG;
      c->batch_split = value != 0;
      return GCL_OK;
    case GCL_OPT_STREAM_PRIORITY: {
      if (value != 0 && value != 1) return GCL_ERR_ARG;
      int lo = 0, hi = 0;
      GCL_TRY(cudaSetDevice(c->device));
      GCL_TRY(cudaDeviceGetStreamPriorityRange(&lo, &hi));
      cudaStream_t s2 = nullptr;
      GCL_TRY(cudaStreamCreateWithPriority(&s2, cudaStreamNonBlocking, value ? hi : lo));
      // work and stream-ordered frees issued so far finish on the old stream
      cudaStreamSynchronize(c->stream);
      cudaStreamDestroy(c->stream);
      c->stream = s2;
      c->each_buf([&](DevBuf& b) { b.stream = s2; });
      if (c->peer) return gcl_set_option(c->peer, GCL_OPT_STREAM_PRIORITY, value);
      return GCL_OK;
    }
    default:
      return GCL_ERR_ARG;
  }
}

int gcl_canon_wide_device_async(gcl_context* c, const int32_t* d_rowptr, const int32_t* d_col,
                                const int32_t* d_color, int n, int64_t m, int max_aut,
                                uint8_t* d_out_dense, uint64_t* d_out_rows,
                                int32_t* d_out_label, int64_t* d_out_stats,
                                int32_t* d_out_status) try {
  if (!c || n < 1 || m < 0 || max_aut <= 0 || !d_rowptr || (m > 0 && !d_col) || !d_out_status)
    return GCL_ERR_ARG;
  if (n > GCL_MAX_N) return GCL_ERR_TOO_LARGE;
  GCL_TRY(cudaSetDevice(c->device));
  const uint32_t un = (uint32_t)n;
  const uint64_t m2 = (uint64_t)std::max<int64_t>(m, 1);
  const uint32_t cap = wide_store_cap(un, max_aut);
  // work sharing: a queue of handed-over subtrees, never recycled within a
  // search, of at most 65,536 entries and 256 MiB
  const uint32_t qcap = c->wide_share
                            ? (uint32_t)std::min<uint64_t>(65536, kGiftMaxWords / wide_gift_words(un))
                            : 0u;
  const WideLayout WL = wide_layout(un, m2, cap, qcap);
  const uint32_t pool = std::min<uint32_t>(c->wide_pool, un + 2);
  const SpLayout Lo = sp_layout(un, m2, pool, 0, std::min<uint32_t>(cap, kWideFixCap));
  uint64_t smw = c->smem_stage ? sp_smem_bytes(un) : 0;
  if (smw * kSpWarps > (uint64_t)kSpSmemPerBlock) smw = 0;
  int per_sm = 0;
  GCL_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &per_sm, wide_items_fn(c->wide_share, c->wide_count), kSpThreads, (size_t)(smw * kSpWarps)));
  const uint64_t budget = ctx_workspace(c);
  int64_t warps = std::min<int64_t>((int64_t)c->sms * std::max(per_sm, 1) * kSpWarps,
                                    std::max<int64_t>(kSpWarps, (int64_t)(budget / Lo.bytes)));
  // no more warps than the largest possible number of work items
  warps = std::min<int64_t>(warps, ((int64_t)n * 2 + kSpWarps - 1) / kSpWarps * kSpWarps);
  if (c->wide_max_warps > 0) warps = std::min<int64_t>(warps, c->wide_max_warps);
  warps = std::max<int64_t>(kSpWarps, warps / kSpWarps * kSpWarps);
  GCL_TRY(c->wide_sh.ensure(WL.bytes));
  GCL_TRY(c->wide_slots.ensure((size_t)(warps * Lo.bytes)));
  WideArgs WA;
  std::memset(&WA, 0, sizeof WA);
  WA.rp = d_rowptr;
  WA.col = d_col;
  WA.color = d_color;
  WA.n = un;
  WA.m = m;
  WA.sh = (uint8_t*)c->wide_sh.p;
  WA.WL = WL;
  WA.slots = (uint8_t*)c->wide_slots.p;
  WA.Lo = Lo;
  WA.slot_bytes = Lo.bytes;
  WA.pool = pool;
  WA.gate = (uint32_t)c->wide_gate;
  WA.probe = c->wide_probe ? 1u : 0u;
  WA.smem_per_warp = smw;
  WA.budget_ns = graph_budget_ns();
  WA.out_dense = d_out_dense;
  WA.out_rows = d_out_rows;
  WA.out_label = d_out_label;
  WA.out_stats = d_out_stats;
  WA.out_status = d_out_status;
  cudaStream_t s = c->stream;
  // the store's completion flags start clear: the buffer is reused across
  // searches (and comes from the pool uninitialised), and a flag left set
  // would let a reader take a slot that a writer has claimed but not filled
  GCL_TRY(cudaMemsetAsync(WA.sh + WL.ready, 0, 4ull * cap, s));
  if (qcap) GCL_TRY(cudaMemsetAsync(WA.sh + WL.gready, 0, 4ull * qcap, s));
  c->counted = false;
  if (c->wide_count)
    GCL_TRY(cudaMemsetAsync(WA.sh + WL.hdr + offsetof(WideHdr, cnt), 0,
                            sizeof(((WideHdr*)nullptr)->cnt), s));
  wide_first_kernel<<<1, 32, 0, s>>>(WA);
  GCL_TRY(cudaGetLastError());
  const int grid = (int)(warps / kSpWarps);
  const size_t smem = (size_t)(smw * kSpWarps);
  if (c->wide_share) {
    if (c->wide_count)
      wide_items_kernel<true, true><<<grid, kSpThreads, smem, s>>>(WA);
    else
      wide_items_kernel<true, false><<<grid, kSpThreads, smem, s>>>(WA);
  } else {
    if (c->wide_count)
      wide_items_kernel<false, true><<<grid, kSpThreads, smem, s>>>(WA);
    else
      wide_items_kernel<false, false><<<grid, kSpThreads, smem, s>>>(WA);
  }
  GCL_TRY(cudaGetLastError());
  c->counted = c->wide_count;
  // a warp per canonical row, up to 8 blocks of 4 warps per SM
  const int64_t finish_warps_per_block = kWideFinishThreads / 32;
  const int finish_blocks = (int)std::max<int64_t>(
      1, std::min<int64_t>(((int64_t)n + finish_warps_per_block - 1) / finish_warps_per_block,
                           (int64_t)std::max(c->sms, 1) * 8));
  wide_finish_kernel<<<finish_blocks, kWideFinishThreads, 0, s>>>(WA);
  GCL_TRY(cudaGetLastError());
  return GCL_OK;
} GCL_CATCH_ALL

}  // extern "C"

namespace gcl {
int context_device(const gcl_context* c) { return c->device; }
}  // namespace gcl

// ---------------------------------------------------------------------------
// Host-pointer entry points.
// ---------------------------------------------------------------------------
namespace {

std::once_flag g_default_once;
gcl_context* g_default = nullptr;
int g_default_rc = GCL_OK;
// calls through the process-wide context hold this lock: a context serves
// one call at a time, and callers of the NULL context may be on any thread
std::mutex g_default_mu;

int default_context(gcl_context** out) {
  std::call_once(g_default_once, [] { g_default_rc = gcl_create(0, &g_default); });
  *out = g_default;
  return g_default_rc;
}

int graph_status_to_rc(int32_t s) {
  switch (s) {
    case kOk: return GCL_OK;
    case kBadInput: return GCL_ERR_BAD_INPUT;
    case kTooLarge: return GCL_ERR_TOO_LARGE;
    case kTimeout: return GCL_ERR_TIMEOUT;
    default: return GCL_ERR_INTERNAL;
  }
}

// The device address of [p, p + count) when that range lies whole in one of
// the context's mapped host buffers (gcl_host_alloc); null otherwise.
template <typename T>
T* mapped_alias(const gcl_context* c, const T* p, size_t count) {
  if (!p) return nullptr;
  const uintptr_t b = (uintptr_t)p;
  const size_t bytes = count * sizeof(T);
  for (const auto& h : c->mapped) {
    const uintptr_t lo = (uintptr_t)h.p, hi = lo + h.bytes;
    if (b >= lo && b <= hi && bytes <= hi - b) return (T*)(h.dev + (b - lo));
  }
  return nullptr;
}

// Wide search of one graph given in host memory; the dense matrix (out_nxn)
// or the packed rows (out_rows) and the statistics come back to the host.
// GCL_ERR_INTERNAL: no result (workspace outgrown or an internal check), the
// caller falls back.
int canon_wide_host(gcl_context* c, const int32_t* rowptr, const int32_t* col,
                    const int32_t* color, int n, int max_aut, uint8_t* out_nxn,
                    uint64_t* out_rows, int64_t* st) {
  const int64_t m = rowptr[n];
  if (rowptr[0] != 0 || m < 0) return GCL_ERR_BAD_INPUT;
  if (m > 0 && !col) return GCL_ERR_ARG;
  GCL_TRY(cudaSetDevice(c->device));
  cudaStream_t s = c->stream;
  DrainOnExit drain(s);
  GCL_TRY(c->rowptr.ensure(((size_t)n + 1) * sizeof(int32_t)));
  GCL_TRY(c->col.ensure(std::max<size_t>((size_t)m, 1) * sizeof(int32_t)));
  const size_t row_words = (size_t)n * (((size_t)n + 63) / 64);
  if (out_nxn) GCL_TRY(c->dense.ensure(std::max<size_t>((size_t)n * n, 1)));
  if (out_rows) GCL_TRY(c->rows.ensure(std::max<size_t>(row_words, 1) * sizeof(uint64_t)));
  GCL_TRY(c->stats.ensure(2 * sizeof(int64_t)));
  GCL_TRY(c->status.ensure(sizeof(int32_t)));
  GCL_TRY(cudaMemcpyAsync(c->rowptr.p, rowptr, ((size_t)n + 1) * sizeof(int32_t),
                          cudaMemcpyHostToDevice, s));
  if (m) GCL_TRY(cudaMemcpyAsync(c->col.p, col, (size_t)m * sizeof(int32_t), cudaMemcpyHostToDevice, s));
  int32_t* d_color = nullptr;
  if (color) {
    GCL_TRY(c->color.ensure((size_t)n * sizeof(int32_t)));
    GCL_TRY(cudaMemcpyAsync(c->color.p, color, (size_t)n * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    d_color = (int32_t*)c->color.p;
  }
  int rc = gcl_canon_wide_device_async(
      c, (int32_t*)c->rowptr.p, (int32_t*)c->col.p, d_color, n, m, max_aut,
      out_nxn ? (uint8_t*)c->dense.p : nullptr, out_rows ? (uint64_t*)c->rows.p : nullptr,
      nullptr, (int64_t*)c->stats.p, (int32_t*)c->status.p);
  if (rc != GCL_OK) return rc == GCL_ERR_NOMEM ? GCL_ERR_INTERNAL : rc;
  int32_t status = 0;
  GCL_TRY(cudaMemcpyAsync(&status, c->status.p, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  GCL_TRY(cudaMemcpyAsync(st, c->stats.p, 2 * sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  GCL_TRY(cudaStreamSynchronize(s));
  if (status == kAutOverflow) return GCL_ERR_INTERNAL;
  if (status != kOk) return graph_status_to_rc(status);
  if (out_nxn)
    GCL_TRY(cudaMemcpyAsync(out_nxn, c->dense.p, (size_t)n * n, cudaMemcpyDeviceToHost, s));
  if (out_rows)
    GCL_TRY(cudaMemcpyAsync(out_rows, c->rows.p, row_words * sizeof(uint64_t),
                            cudaMemcpyDeviceToHost, s));
  GCL_TRY(cudaStreamSynchronize(s));
  drain.done = true;
  return GCL_OK;
}

// gcl_canon_one with the dense matrix (out_nxn) or the packed rows (out_rows)
int canon_one(gcl_context* c, const int32_t* rowptr, const int32_t* col, const int32_t* color,
              int n, int max_aut, uint8_t* out_nxn, uint64_t* out_rows, int64_t* node_count,
              int64_t* num_aut) {
  std::unique_lock<std::mutex> shared_ctx;
  if (!c) {
    int rc = default_context(&c);
    if (rc != GCL_OK) return rc;
    shared_ctx = std::unique_lock<std::mutex>(g_default_mu);
  }
  if (n == 0) {  // the reference's search visits the (discrete) root only
    if (node_count) *node_count = 1;
    if (num_aut) *num_aut = 0;
    return GCL_OK;
  }
  int64_t st[2] = {0, 0};
  if ((int64_t)n >= c->wide_min_n && n <= GCL_MAX_N) {
    const int rcw = canon_wide_host(c, rowptr, col, color, n, max_aut, out_nxn, out_rows, st);
    if (rcw != GCL_ERR_INTERNAL) {  // no result for want of workspace: sequential search
      if (rcw == GCL_OK) {
        if (num_aut) *num_aut = st[0];
        if (node_count) *node_count = st[1];
      }
      return rcw;
    }
  }
  const int64_t voff[2] = {0, n};
  const int64_t eoff[2] = {0, rowptr[n]};
  const int64_t ooff[2] = {0, (int64_t)n * n};
  const int64_t roff[2] = {0, (int64_t)n * (((int64_t)n + 63) / 64)};
  int32_t status = 0;
  int rc = gcl_canon_batch(c, 1, voff, eoff, rowptr, col, color, max_aut, out_nxn,
                           out_nxn ? ooff : nullptr, out_rows, out_rows ? roff : nullptr, nullptr,
                           st, &status);
  if (rc != GCL_OK) return rc;
  if (num_aut) *num_aut = st[0];
  if (node_count) *node_count = st[1];
  return GCL_OK;
}


// The graphs (n > 64) of a host batch that ran past the hand-off budget in
// their batch warp (gcl_canon_batch with GCL_OPT_BATCH_HANDOFF_MS): the wide
// search, one graph at a time on the context (the smallest first), each
// within the per-graph budget and all within `hard_ns` (0 = no limit).  A
// graph it finishes gets
// the wide search's results in place of the timeout: the same canonical
// form, a labeling that is one of the equivalent best leaves, and the wide
// search's own statistics; one it does not finish keeps its timeout.
int batch_handoff(gcl_context* c, int count, const int64_t* voff, const int64_t* eoff,
                  const int32_t* d_color, int max_aut, const int64_t* ooff, const int64_t* roff,
                  uint8_t* out_dense, uint64_t* out_rows, int32_t* out_label,
                  int64_t* out_stats, int32_t* out_status, uint8_t* d_dense, uint64_t* d_rows,
                  int32_t* d_label, int64_t* d_stats, uint64_t hard_ns) {
  cudaStream_t s = c->stream;
  const auto t0 = std::chrono::steady_clock::now();
  const int32_t* d_rp = (const int32_t*)c->rowptr.p;
  const int32_t* d_col = (const int32_t*)c->col.p;
  int32_t* d_status = (int32_t*)c->status.p;
  std::vector<int> todo;
  for (int g = 0; g < count; ++g)
    if (out_status[g] == kTimeout && voff[g + 1] - voff[g] > kW64MaxN) todo.push_back(g);
  std::stable_sort(todo.begin(), todo.end(),
                   [&](int a, int b) { return voff[a + 1] - voff[a] < voff[b + 1] - voff[b]; });
  for (const int g : todo) {
    const int64_t n = voff[g + 1] - voff[g];
    if (hard_ns && (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
                       std::chrono::steady_clock::now() - t0).count() > hard_ns)
      break;
    const int64_t vo = voff[g], eo = eoff[g];
    const int rc = gcl_canon_wide_device_async(
        c, d_rp + vo + g, d_col + eo, d_color ? d_color + vo : nullptr, (int)n, eoff[g + 1] - eo,
        max_aut, d_dense ? d_dense + ooff[g] : nullptr, d_rows ? d_rows + roff[g] : nullptr,
        d_label ? d_label + vo : nullptr, d_stats ? d_stats + 2 * g : nullptr, d_status + g);
    if (rc != GCL_OK) return rc;
    int32_t st = 0;
    GCL_TRY(cudaMemcpyAsync(&st, d_status + g, sizeof st, cudaMemcpyDeviceToHost, s));
    GCL_TRY(cudaStreamSynchronize(s));
    if (st != kOk) continue;  // keeps the batch's timeout
    if (out_dense && n)
      GCL_TRY(cudaMemcpyAsync(out_dense + ooff[g], d_dense + ooff[g], (size_t)(n * n),
                              cudaMemcpyDeviceToHost, s));
    if (out_rows && n)
      GCL_TRY(cudaMemcpyAsync(out_rows + roff[g], d_rows + roff[g],
                              (size_t)(roff[g + 1] - roff[g]) * sizeof(uint64_t),
                              cudaMemcpyDeviceToHost, s));
    if (d_label)
      GCL_TRY(cudaMemcpyAsync(out_label + vo, d_label + vo, (size_t)n * sizeof(int32_t),
                              cudaMemcpyDeviceToHost, s));
    if (d_stats)
      GCL_TRY(cudaMemcpyAsync(out_stats + 2 * g, d_stats + 2 * g, 2 * sizeof(int64_t),
                              cudaMemcpyDeviceToHost, s));
    GCL_TRY(cudaStreamSynchronize(s));
    out_status[g] = kOk;
  }
  return GCL_OK;
}

}  // namespace

extern "C" {

// Batches of at least this many graphs of up to 64 vertices run as two
// halves on two streams (GCL_OPT_BATCH_SPLIT).
constexpr int kSplitMinGraphs = 4096;

// gcl_canon_batch in two halves: graphs [0, h) on the context's stream,
// [h, count) on the companion context's.  The offsets of the arena are
// absolute, so each half is the same arrays seen from its first graph: the
// uploads, the kernels and the downloads of a half touch its own ranges only.
// Returns GCL_OK or an error code; the caller maps per-graph statuses.
static int canon_batch_halves(gcl_context* c, const BatchShape& B, int count,
                              const int64_t* voff, const int64_t* eoff, const int32_t* rowptr,
                              const int32_t* col, const int32_t* color, int max_aut,
                              uint8_t* out_dense, const int64_t* ooff, uint64_t* out_rows,
                              const int64_t* roff, int32_t* out_label, int64_t* out_stats,
                              int32_t* out_status) {
  if (!c->peer) {
    gcl_context* q = nullptr;
    const int rc = gcl_create(c->device, &q);
    if (rc != GCL_OK) return rc;
    c->peer = q;
    GCL_TRY(cudaSetDevice(c->device));
    // the same stream priority as the context's (GCL_OPT_STREAM_PRIORITY)
    int pr = 0, lo = 0, hi = 0;
    if (cudaStreamGetPriority(c->stream, &pr) == cudaSuccess &&
        cudaDeviceGetStreamPriorityRange(&lo, &hi) == cudaSuccess && lo != hi && pr == hi) {
      const int rp = gcl_set_option(q, GCL_OPT_STREAM_PRIORITY, 1);
      if (rp != GCL_OK) return rp;
    }
    (void)cudaGetLastError();
  }
  gcl_context* q = c->peer;
  q->tune_w64_bps = c->tune_w64_bps;
  q->workspace_bytes = c->workspace_bytes;
  if (!c->split_ev) GCL_TRY(cudaEventCreateWithFlags(&c->split_ev, cudaEventDisableTiming));
  const size_t cnt = (size_t)count;
  GCL_TRY(c->voff.ensure((cnt + 1) * sizeof(int64_t)));
  GCL_TRY(c->eoff.ensure((cnt + 1) * sizeof(int64_t)));
  GCL_TRY(c->rowptr.ensure(B.nrp * sizeof(int32_t)));
  GCL_TRY(c->col.ensure(std::max<size_t>(B.ne, 1) * sizeof(int32_t)));
  GCL_TRY(c->status.ensure(cnt * sizeof(int32_t)));
  if (color && B.nv) GCL_TRY(c->color.ensure(B.nv * sizeof(int32_t)));
  if (out_dense) {
    GCL_TRY(c->ooff.ensure((cnt + 1) * sizeof(int64_t)));
    GCL_TRY(c->dense.ensure(std::max<size_t>(B.dense_bytes, 1)));
  }
  if (out_rows) {
    GCL_TRY(c->roff.ensure((cnt + 1) * sizeof(int64_t)));
    GCL_TRY(c->rows.ensure(std::max<size_t>(B.rows_words, 1) * sizeof(uint64_t)));
  }
  if (out_label && B.nv) GCL_TRY(c->label.ensure(B.nv * sizeof(int32_t)));
  if (out_stats) GCL_TRY(c->stats.ensure(2 * cnt * sizeof(int64_t)));
  int64_t* d_voff = (int64_t*)c->voff.p;
  int64_t* d_eoff = (int64_t*)c->eoff.p;
  int32_t* d_rowptr = (int32_t*)c->rowptr.p;
  int32_t* d_col = (int32_t*)c->col.p;
  int32_t* d_color = color && B.nv ? (int32_t*)c->color.p : nullptr;
  int64_t* d_ooff = out_dense ? (int64_t*)c->ooff.p : nullptr;
  uint8_t* d_dense = out_dense ? (uint8_t*)c->dense.p : nullptr;
  int64_t* d_roff = out_rows ? (int64_t*)c->roff.p : nullptr;
  uint64_t* d_rows = out_rows ? (uint64_t*)c->rows.p : nullptr;
  int32_t* d_label = out_label && B.nv ? (int32_t*)c->label.p : nullptr;
  int64_t* d_stats = out_stats ? (int64_t*)c->stats.p : nullptr;
  int32_t* d_status = (int32_t*)c->status.p;
  cudaStream_t s0 = c->stream, s1 = q->stream;
  DrainOnExit drain0(s0), drain1(s1);
  // the buffers were (re)allocated in the context's stream order: the
  // companion stream starts after that
  GCL_TRY(cudaEventRecord(c->split_ev, s0));
  GCL_TRY(cudaStreamWaitEvent(s1, c->split_ev, 0));
  auto h2d = [](void* dst, const void* src, size_t bytes, cudaStream_t s) {
    return bytes ? cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s) : cudaSuccess;
  };
  auto d2h = [](void* dst, const void* src, size_t bytes, cudaStream_t s) {
    return bytes ? cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s) : cudaSuccess;
  };
  // graphs [g0, g1): their offsets, CSR rows (n + 1 entries per graph from
  // voff[g] + g), neighbours, colours and output offsets
  auto upload = [&](int g0, int g1, cudaStream_t s) -> cudaError_t {
    const size_t k = (size_t)(g1 - g0) + 1;
    const size_t r0 = (size_t)(voff[g0] + g0), r1 = (size_t)(voff[g1] + g1);
    cudaError_t e = h2d(d_voff + g0, voff + g0, k * sizeof(int64_t), s);
    if (e == cudaSuccess) e = h2d(d_eoff + g0, eoff + g0, k * sizeof(int64_t), s);
    if (e == cudaSuccess) e = h2d(d_rowptr + r0, rowptr + r0, (r1 - r0) * sizeof(int32_t), s);
    if (e == cudaSuccess)
      e = h2d(d_col + eoff[g0], col + eoff[g0], (size_t)(eoff[g1] - eoff[g0]) * sizeof(int32_t), s);
    if (e == cudaSuccess && d_color)
      e = h2d(d_color + voff[g0], color + voff[g0], (size_t)(voff[g1] - voff[g0]) * sizeof(int32_t), s);
    if (e == cudaSuccess && d_ooff) e = h2d(d_ooff + g0, ooff + g0, k * sizeof(int64_t), s);
    if (e == cudaSuccess && d_roff) e = h2d(d_roff + g0, roff + g0, k * sizeof(int64_t), s);
    return e;
  };
  auto download = [&](int g0, int g1, cudaStream_t s) -> cudaError_t {
    cudaError_t e = cudaSuccess;
    if (d_dense)
      e = d2h(out_dense + ooff[g0], d_dense + ooff[g0], (size_t)(ooff[g1] - ooff[g0]), s);
    if (e == cudaSuccess && d_rows)
      e = d2h(out_rows + roff[g0], d_rows + roff[g0], (size_t)(roff[g1] - roff[g0]) * sizeof(uint64_t), s);
    if (e == cudaSuccess && d_label)
      e = d2h(out_label + voff[g0], d_label + voff[g0], (size_t)(voff[g1] - voff[g0]) * sizeof(int32_t), s);
    if (e == cudaSuccess && d_stats)
      e = d2h(out_stats + 2 * (size_t)g0, d_stats + 2 * (size_t)g0, 2 * (size_t)(g1 - g0) * sizeof(int64_t), s);
    if (e == cudaSuccess)
      e = d2h(out_status + g0, d_status + g0, (size_t)(g1 - g0) * sizeof(int32_t), s);
    return e;
  };
  const int h = count / 2;
  GCL_TRY(upload(0, h, s0));
  int rc = gcl_canon_batch_device_async(c, h, d_voff, d_eoff, d_rowptr, d_col, d_color, max_aut,
                                        B.max_n, B.max_m2, d_dense, d_ooff, d_rows, d_roff, d_label,
                                        d_stats, d_status);
  if (rc != GCL_OK) return rc;
  GCL_TRY(upload(h, count, s1));
  rc = gcl_canon_batch_device_async(q, count - h, d_voff + h, d_eoff + h, d_rowptr + h, d_col,
                                    d_color, max_aut, B.max_n, B.max_m2, d_dense,
                                    d_ooff ? d_ooff + h : nullptr, d_rows,
                                    d_roff ? d_roff + h : nullptr, d_label,
                                    d_stats ? d_stats + 2 * (size_t)h : nullptr, d_status + h);
  GCL_TRY(cudaSetDevice(c->device));
  if (rc != GCL_OK) return rc;
  GCL_TRY(download(0, h, s0));
  GCL_TRY(download(h, count, s1));
  GCL_TRY(cudaStreamSynchronize(s0));
  GCL_TRY(cudaStreamSynchronize(s1));
  drain0.done = drain1.done = true;
  return GCL_OK;
}

int gcl_canon_batch(gcl_context* c, int count, const int64_t* voff, const int64_t* eoff,
                    const int32_t* rowptr, const int32_t* col, const int32_t* color, int max_aut,
                    uint8_t* out_dense, const int64_t* ooff, uint64_t* out_rows,
                    const int64_t* roff, int32_t* out_label, int64_t* out_stats,
                    int32_t* out_status) try {
  if (!c || count < 0 || max_aut <= 0 || !voff || !eoff || !rowptr || !out_status ||
      (out_dense && !ooff) || (out_rows && !roff))
    return GCL_ERR_ARG;
  if (count == 0) return GCL_OK;
  BatchShape B;
  const int rcb = check_batch(count, voff, eoff, rowptr, col, out_dense ? ooff : nullptr,
                              out_rows ? roff : nullptr, &B);
  if (rcb != GCL_OK) return rcb;
  const int max_n = B.max_n;
  const int64_t max_m2 = B.max_m2;
  GCL_TRY(cudaSetDevice(c->device));
  if (c->batch_split && count >= kSplitMinGraphs && max_n <= kW64MaxN && !c->timing) {
    const int rs = canon_batch_halves(c, B, count, voff, eoff, rowptr, col, color, max_aut,
                                      out_dense, ooff, out_rows, roff, out_label, out_stats,
                                      out_status);
    if (rs != GCL_OK) return rs;
    for (int g = 0; g < count; ++g)
      if (out_status[g] != kOk) return graph_status_to_rc(out_status[g]);
    return GCL_OK;
  }
  const size_t nv = B.nv, ne = B.ne;
  const size_t cnt = (size_t)count;  // byte counts in size_t, not int
  const size_t nrp = B.nrp;
  GCL_TRY(c->voff.ensure((cnt + 1) * sizeof(int64_t)));
  GCL_TRY(c->eoff.ensure((cnt + 1) * sizeof(int64_t)));
  GCL_TRY(c->rowptr.ensure(nrp * sizeof(int32_t)));
  GCL_TRY(c->col.ensure(std::max<size_t>(ne, 1) * sizeof(int32_t)));
  GCL_TRY(c->status.ensure(cnt * sizeof(int32_t)));
  cudaStream_t s = c->stream;
  DrainOnExit drain(s);
  GCL_TRY(cudaMemcpyAsync(c->voff.p, voff, (cnt + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, s));
  GCL_TRY(cudaMemcpyAsync(c->eoff.p, eoff, (cnt + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, s));
  GCL_TRY(cudaMemcpyAsync(c->rowptr.p, rowptr, nrp * sizeof(int32_t), cudaMemcpyHostToDevice, s));
  if (ne) GCL_TRY(cudaMemcpyAsync(c->col.p, col, ne * sizeof(int32_t), cudaMemcpyHostToDevice, s));
  int32_t* d_color = nullptr;
  if (color && nv) {
    GCL_TRY(c->color.ensure(nv * sizeof(int32_t)));
    GCL_TRY(cudaMemcpyAsync(c->color.p, color, nv * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    d_color = (int32_t*)c->color.p;
  }
  uint8_t* d_dense = nullptr;
  int64_t* d_ooff = nullptr;
  size_t dense_bytes = 0;
  if (out_dense) {
    dense_bytes = (size_t)ooff[count];
    GCL_TRY(c->ooff.ensure((cnt + 1) * sizeof(int64_t)));
    GCL_TRY(c->dense.ensure(std::max<size_t>(dense_bytes, 1)));
    GCL_TRY(cudaMemcpyAsync(c->ooff.p, ooff, (cnt + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, s));
    d_dense = (uint8_t*)c->dense.p;
    d_ooff = (int64_t*)c->ooff.p;
  }
  uint64_t* d_rows = nullptr;
  int64_t* d_roff = nullptr;
  size_t rows_words = 0;
  if (out_rows) {
    rows_words = (size_t)roff[count];
    GCL_TRY(c->roff.ensure((cnt + 1) * sizeof(int64_t)));
    GCL_TRY(c->rows.ensure(std::max<size_t>(rows_words, 1) * sizeof(uint64_t)));
    GCL_TRY(cudaMemcpyAsync(c->roff.p, roff, (cnt + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, s));
    d_rows = (uint64_t*)c->rows.p;
    d_roff = (int64_t*)c->roff.p;
  }
  int32_t* d_label = nullptr;
  if (out_label && nv) {
    GCL_TRY(c->label.ensure(nv * sizeof(int32_t)));
    d_label = (int32_t*)c->label.p;
  }
  int64_t* d_stats = nullptr;
  if (out_stats) {
    GCL_TRY(c->stats.ensure(2 * cnt * sizeof(int64_t)));
    d_stats = (int64_t*)c->stats.p;
  }
  // with a hand-off budget, graphs above 64 vertices whose batch warp runs
  // past it are searched again by the wide search below
  const uint64_t hard_ns = graph_budget_ns();
  const bool handoff = c->handoff_ns > 0 && max_n > kW64MaxN && (hard_ns == 0 || c->handoff_ns < hard_ns);
  if (handoff) c->budget_override_ns = c->handoff_ns;
  int rc = gcl_canon_batch_device_async(c, count, (int64_t*)c->voff.p, (int64_t*)c->eoff.p,
                                        (int32_t*)c->rowptr.p, (int32_t*)c->col.p, d_color,
                                        max_aut, max_n, max_m2, d_dense, d_ooff, d_rows, d_roff,
                                        d_label, d_stats,
                                        (int32_t*)c->status.p);
  c->budget_override_ns = 0;
  if (rc != GCL_OK) return rc;
  if (out_dense && dense_bytes)
    GCL_TRY(cudaMemcpyAsync(out_dense, d_dense, dense_bytes, cudaMemcpyDeviceToHost, s));
  if (out_rows && rows_words)
    GCL_TRY(cudaMemcpyAsync(out_rows, d_rows, rows_words * sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
  if (d_label) GCL_TRY(cudaMemcpyAsync(out_label, d_label, nv * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  if (d_stats)
    GCL_TRY(cudaMemcpyAsync(out_stats, d_stats, 2 * cnt * sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  GCL_TRY(cudaMemcpyAsync(out_status, c->status.p, cnt * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  GCL_TRY(cudaStreamSynchronize(s));
  if (handoff) {
    const int rh = batch_handoff(c, count, voff, eoff, d_color, max_aut, ooff, roff, out_dense,
                                 out_rows, out_label, out_stats, out_status, d_dense, d_rows,
                                 d_label, d_stats, hard_ns);
    if (rh != GCL_OK) return rh;
  }
  drain.done = true;
  for (int g = 0; g < count; ++g)
    if (out_status[g] != kOk) return graph_status_to_rc(out_status[g]);
  return GCL_OK;
} GCL_CATCH_ALL

int gcl_canon_one(gcl_context* c, const int32_t* rowptr, const int32_t* col, const int32_t* color,
                  int n, int max_aut, uint8_t* out_nxn, int64_t* node_count, int64_t* num_aut) try {
  if (n < 0 || !rowptr || max_aut <= 0 || (n > 0 && !out_nxn)) return GCL_ERR_ARG;
  return canon_one(c, rowptr, col, color, n, max_aut, out_nxn, nullptr, node_count, num_aut);
} GCL_CATCH_ALL

int gcl_canon_one_rows(gcl_context* c, const int32_t* rowptr, const int32_t* col,
                       const int32_t* color, int n, int max_aut, uint64_t* out_rows,
                       int64_t* node_count, int64_t* num_aut) try {
  if (n < 0 || !rowptr || max_aut <= 0 || (n > 0 && !out_rows)) return GCL_ERR_ARG;
  return canon_one(c, rowptr, col, color, n, max_aut, nullptr, out_rows, node_count, num_aut);
} GCL_CATCH_ALL

int gcl_host_alloc(gcl_context* c, size_t bytes, void** out) try {
  if (!c || !out || bytes == 0) return GCL_ERR_ARG;
  *out = nullptr;
  GCL_TRY(cudaSetDevice(c->device));
  void *p = nullptr, *dev = nullptr;
  GCL_TRY(mapped_alloc(&p, &dev, bytes));
  try {
    c->mapped.push_back({(uint8_t*)p, bytes, (uint8_t*)dev});
  } catch (...) {
    cudaFreeHost(p);
    throw;
  }
  *out = p;
  return GCL_OK;
} GCL_CATCH_ALL

int gcl_host_free(gcl_context* c, void* p) try {
  if (!c || !p) return GCL_ERR_ARG;
  for (size_t i = 0; i < c->mapped.size(); ++i) {
    if (c->mapped[i].p != (uint8_t*)p) continue;
    cudaStreamSynchronize(c->stream);  // no kernel of the context still uses it
    cudaFreeHost(p);
    c->mapped.erase(c->mapped.begin() + (std::ptrdiff_t)i);
    return GCL_OK;
  }
  return GCL_ERR_ARG;
} GCL_CATCH_ALL

int gcl_canon_batch_mapped(gcl_context* c, int count, const int64_t* voff, const int64_t* eoff,
                           const int32_t* rowptr, const int32_t* col, const int32_t* color,
                           int max_aut, uint8_t* out_dense, const int64_t* ooff,
                           uint64_t* out_rows, const int64_t* roff, int32_t* out_label,
                           int64_t* out_stats, int32_t* out_status) try {
  if (!c || count < 0 || max_aut <= 0 || !voff || !eoff || !rowptr || !out_status ||
      (out_dense && !ooff) || (out_rows && !roff))
    return GCL_ERR_ARG;
  if (count == 0) return GCL_OK;
  const size_t cnt = (size_t)count;
  // the offsets first: the host checks below read the arrays they delimit
  if (!mapped_alias(c, voff, cnt + 1) || !mapped_alias(c, eoff, cnt + 1) ||
      (out_dense && !mapped_alias(c, ooff, cnt + 1)) ||
      (out_rows && !mapped_alias(c, roff, cnt + 1)))
    return GCL_ERR_ARG;
  // ascending vertex offsets keep every rowptr index the checks read below
  // voff[count] + count, the extent checked here
  for (int g = 0; g < count; ++g)
    if (voff[g + 1] < voff[g]) return GCL_ERR_ARG;
  if (voff[0] != 0 || !mapped_alias(c, rowptr, (size_t)voff[count] + cnt)) return GCL_ERR_ARG;
  BatchShape B;
  const int rcb = check_batch(count, voff, eoff, rowptr, col, out_dense ? ooff : nullptr,
                              out_rows ? roff : nullptr, &B);
  if (rcb != GCL_OK) return rcb;
  // every array whole in the context's mapped buffers: the kernels read and
  // write them in place
  const int64_t* d_voff = mapped_alias(c, voff, cnt + 1);
  const int64_t* d_eoff = mapped_alias(c, eoff, cnt + 1);
  const int32_t* d_rowptr = mapped_alias(c, rowptr, B.nrp);
  const int32_t* d_col = B.ne ? mapped_alias(c, col, B.ne) : nullptr;
  const int32_t* d_color = color && B.nv ? mapped_alias(c, color, B.nv) : nullptr;
  uint8_t* d_dense = out_dense ? mapped_alias(c, out_dense, B.dense_bytes) : nullptr;
  const int64_t* d_ooff = out_dense ? mapped_alias(c, ooff, cnt + 1) : nullptr;
  uint64_t* d_rows = out_rows ? mapped_alias(c, out_rows, B.rows_words) : nullptr;
  const int64_t* d_roff = out_rows ? mapped_alias(c, roff, cnt + 1) : nullptr;
  int32_t* d_label = out_label && B.nv ? mapped_alias(c, out_label, B.nv) : nullptr;
  int64_t* d_stats = out_stats ? mapped_alias(c, out_stats, 2 * cnt) : nullptr;
  int32_t* d_status = mapped_alias(c, out_status, cnt);
  if (!d_rowptr || (B.ne && !d_col) || (color && B.nv && !d_color) || (out_dense && !d_dense) ||
      (out_rows && !d_rows) || (out_label && B.nv && !d_label) || (out_stats && !d_stats) ||
      !d_status)
    return GCL_ERR_ARG;
  // the kernels for larger graphs read the CSR again at every refinement
  // step: those batches go through device copies (DMA from the same buffers)
  if (B.max_n > kW64MaxN)
    return gcl_canon_batch(c, count, voff, eoff, rowptr, col, color, max_aut, out_dense, ooff,
                           out_rows, roff, out_label, out_stats, out_status);
  GCL_TRY(cudaSetDevice(c->device));
  cudaStream_t s = c->stream;
  DrainOnExit drain(s);
  if (!d_col) {  // no edges: a valid address all the same
    GCL_TRY(c->col.ensure(sizeof(int32_t)));
    d_col = (const int32_t*)c->col.p;
  }
  const int rc = gcl_canon_batch_device_async(c, count, d_voff, d_eoff, d_rowptr, d_col, d_color,
                                              max_aut, B.max_n, B.max_m2, d_dense, d_ooff,
                                              d_rows, d_roff, d_label, d_stats, d_status);
  if (rc != GCL_OK) return rc;
  GCL_TRY(cudaStreamSynchronize(s));
  drain.done = true;
  for (int g = 0; g < count; ++g)
    if (out_status[g] != kOk) return graph_status_to_rc(out_status[g]);
  return GCL_OK;
} GCL_CATCH_ALL

int gcl_iso(gcl_context* c, const int32_t* rp1, const int32_t* col1, const int32_t* color1, int n1,
            const int32_t* rp2, const int32_t* col2, const int32_t* color2, int n2, int max_aut,
            int* verdict) try {
  if (!verdict || n1 < 0 || n2 < 0 || !rp1 || !rp2 || max_aut <= 0) return GCL_ERR_ARG;
  std::unique_lock<std::mutex> shared_ctx;
  if (!c) {
    int rc = default_context(&c);
    if (rc != GCL_OK) return rc;
    shared_ctx = std::unique_lock<std::mutex>(g_default_mu);
  }
  // packed canonical rows: equal upper triangles (main.cpp:73-90) of
  // symmetric matrices with a zero diagonal are equal rows
  std::vector<uint64_t> a((size_t)n1 * (((size_t)n1 + 63) / 64) + 1);
  std::vector<uint64_t> b((size_t)n2 * (((size_t)n2 + 63) / 64) + 1);
  int rc = canon_one(c, rp1, col1, color1, n1, max_aut, nullptr, a.data(), nullptr, nullptr);
  if (rc == GCL_OK)
    rc = canon_one(c, rp2, col2, color2, n2, max_aut, nullptr, b.data(), nullptr, nullptr);
  if (rc != GCL_OK) return rc;
  *verdict = n1 == n2 && a == b;
  return GCL_OK;
} GCL_CATCH_ALL

int gcl_group_order(gcl_context* c, const int32_t* rowptr, const int32_t* col,
                    const int32_t* color, int n, double* log10_order, char* digits,
                    int digits_cap, int64_t* generators, int* checked) try {
  if (n < 0 || !rowptr || !log10_order || (digits && digits_cap < 2)) return GCL_ERR_ARG;
  if (n > GCL_MAX_N) return GCL_ERR_TOO_LARGE;
  std::unique_lock<std::mutex> shared_ctx;
  if (!c) {
    int rc = default_context(&c);
    if (rc != GCL_OK) return rc;
    shared_ctx = std::unique_lock<std::mutex>(g_default_mu);
  }
  if (checked) *checked = 0;
  auto put = [&](const std::string& d, double lg, int64_t ng, int chk) {
    *log10_order = lg;
    if (generators) *generators = ng;
    if (checked) *checked = chk;
    if (!digits) return GCL_OK;
    if ((int)d.size() + 1 > digits_cap) return GCL_ERR_ARG;
    std::memcpy(digits, d.c_str(), d.size() + 1);
    return GCL_OK;
  };
  if (n <= 1) return put("1", 0.0, 0, 1);
  // a wide search whose store takes every automorphism it finds
  const int64_t m = rowptr[n];
  if (rowptr[0] != 0 || m < 0) return GCL_ERR_BAD_INPUT;
  if (m > 0 && !col) return GCL_ERR_ARG;
  GCL_TRY(cudaSetDevice(c->device));
  cudaStream_t s = c->stream;
  DrainOnExit drain(s);
  GCL_TRY(c->rowptr.ensure(((size_t)n + 1) * sizeof(int32_t)));
  GCL_TRY(c->col.ensure(std::max<size_t>((size_t)m, 1) * sizeof(int32_t)));
  GCL_TRY(c->stats.ensure(2 * sizeof(int64_t)));
  GCL_TRY(c->status.ensure(sizeof(int32_t)));
  GCL_TRY(cudaMemcpyAsync(c->rowptr.p, rowptr, ((size_t)n + 1) * sizeof(int32_t),
                          cudaMemcpyHostToDevice, s));
  if (m) GCL_TRY(cudaMemcpyAsync(c->col.p, col, (size_t)m * sizeof(int32_t), cudaMemcpyHostToDevice, s));
  int32_t* d_color = nullptr;
  if (color) {
    GCL_TRY(c->color.ensure((size_t)n * sizeof(int32_t)));
    GCL_TRY(cudaMemcpyAsync(c->color.p, color, (size_t)n * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    d_color = (int32_t*)c->color.p;
  }
  const int max_aut = 0x7fffffff;
  int32_t status = 0;
  int64_t st[2] = {0, 0};
  // A warp whose item goes deeper than its per-level orbit arrays reach
  // ends the search with kAutOverflow (the canonizing calls then rerun the
  // graph sequentially); the group order needs this search's automorphisms,
  // so it reruns the wide search with an orbit array for every level.
  for (int attempt = 0; attempt < 2; ++attempt) {
    const uint32_t saved_pool = c->wide_pool;
    if (attempt) c->wide_pool = (uint32_t)n + 2;
    const int rc = gcl_canon_wide_device_async(c, (int32_t*)c->rowptr.p, (int32_t*)c->col.p,
                                               d_color, n, m, max_aut, nullptr, nullptr, nullptr,
                                               (int64_t*)c->stats.p, (int32_t*)c->status.p);
    c->wide_pool = saved_pool;
    if (rc != GCL_OK) return rc;
    GCL_TRY(cudaMemcpyAsync(&status, c->status.p, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    GCL_TRY(cudaMemcpyAsync(st, c->stats.p, 2 * sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    GCL_TRY(cudaStreamSynchronize(s));
    if (status != kAutOverflow) break;
  }
  if (status != kOk) return graph_status_to_rc(status);
  const uint32_t un = (uint32_t)n;
  const uint32_t cap = wide_store_cap(un, max_aut);
  if ((uint64_t)st[0] > cap) return GCL_ERR_TOO_LARGE;  // the store lost generators
  const WideLayout WL = wide_layout(un, (uint64_t)std::max<int64_t>(m, 1), cap);
  std::vector<uint16_t> auts((size_t)st[0] * WL.stride + 1);
  if (st[0])
    GCL_TRY(cudaMemcpyAsync(auts.data(), (const uint8_t*)c->wide_sh.p + WL.auts,
                            (size_t)st[0] * WL.stride * sizeof(uint16_t),
                            cudaMemcpyDeviceToHost, s));
  GCL_TRY(cudaStreamSynchronize(s));
  // the first path's individualized vertices are a base of Aut(G): an
  // automorphism fixing them fixes the first leaf's discrete partition
  const uint8_t* sh = (const uint8_t*)c->wide_sh.p;
  uint32_t D = 0;
  GCL_TRY(cudaMemcpyAsync(&D, sh + WL.hdr + offsetof(WideHdr, D), sizeof(uint32_t),
                          cudaMemcpyDeviceToHost, s));
  GCL_TRY(cudaStreamSynchronize(s));
  if (D < 1 || D > un) return GCL_ERR_INTERNAL;
  std::vector<uint32_t> base(D);
  if (D > 1)
    GCL_TRY(cudaMemcpyAsync(base.data(), sh + WL.fseq, (size_t)(D - 1) * sizeof(uint32_t),
                            cudaMemcpyDeviceToHost, s));
  GCL_TRY(cudaStreamSynchronize(s));
  // the product of the basic orbits, checked by Schreier-Sims where that
  // finishes within its work budget (its order wins a disagreement)
  double lg = 0;
  std::string d;
  int chk = 0;
  const int rg = group_order_of_search(un, auts.data(), (uint64_t)st[0], WL.stride, base.data(),
                                       D - 1, kGroupCheckCap, &lg, &d, &chk);
  if (rg != kOrderOk) {
    // the first path is no base (an internal inconsistency): the general
    // completion alone, with the full budget
    uint64_t base_len = 0;
    if (!group_order(un, auts.data(), (uint64_t)st[0], WL.stride, kGroupWorkCap, &lg, &d,
                     &base_len))
      return GCL_ERR_INTERNAL;
    chk = 1;
  }
  drain.done = true;
  return put(d, lg, st[0], chk);
} GCL_CATCH_ALL

int gcl_perm_group_order(int n, const uint16_t* perms, int64_t count, double* log10_order,
                         char* digits, int digits_cap) try {
  if (n < 0 || n > GCL_MAX_N || count < 0 || (count > 0 && !perms) || !log10_order ||
      (digits && digits_cap < 2))
    return GCL_ERR_ARG;
  for (int64_t a = 0; a < count; ++a) {  // each row must be a permutation
    std::vector<char> seen((size_t)n, 0);
    for (int x = 0; x < n; ++x) {
      const uint16_t y = perms[a * n + x];
      if (y >= n || seen[y]) return GCL_ERR_ARG;
      seen[y] = 1;
    }
  }
  double lg = 0;
  std::string d = "1";
  uint64_t base_len = 0;
  if (n > 1 && !group_order((uint32_t)n, perms, (uint64_t)count, (uint64_t)n, kGroupWorkCap, &lg,
                            &d, &base_len))
    return GCL_ERR_TIMEOUT;
  *log10_order = lg;
  if (digits) {
    if ((int)d.size() + 1 > digits_cap) return GCL_ERR_ARG;
    std::memcpy(digits, d.c_str(), d.size() + 1);
  }
  return GCL_OK;
} GCL_CATCH_ALL

int gcl_set_tuning(gcl_context* c, const gcl_tuning* t) {
  if (!c || !t) return GCL_ERR_ARG;
  c->tune_w64_bps = std::max(t->w64_blocks_per_sm, 0);
  for (int bk = 0; bk < kSpBuckets; ++bk) {
    c->tune_sp_bps[bk] = std::max(t->sp_blocks_per_sm[bk], 0);
    c->tune_sp_stage[bk] = t->sp_stage[bk] < 0 ? -1 : (t->sp_stage[bk] ? 1 : 0);
  }
  return GCL_OK;
}

int gcl_autotune(gcl_context* c, int count, const int64_t* voff, const int64_t* eoff,
                 const int32_t* rowptr, const int32_t* col, const int32_t* color, int max_aut,
                 int repeats, gcl_tuning* out) try {
  if (!c || count <= 0 || !voff || !eoff || !rowptr || !out || max_aut <= 0) return GCL_ERR_ARG;
  if (repeats < 1) repeats = 2;
  GCL_TRY(cudaSetDevice(c->device));
  for (auto& row : c->tev)
    for (cudaEvent_t& ev : row)
      if (!ev) GCL_TRY(cudaEventCreate(&ev));
  std::vector<int64_t> roff(count + 1, 0);
  for (int g = 0; g < count; ++g) {
    const int64_t n = voff[g + 1] - voff[g];
    roff[g + 1] = roff[g] + n * ((n + 63) / 64);
  }
  std::vector<uint64_t> rows((size_t)std::max<int64_t>(roff[count], 1));
  std::vector<int32_t> status(count);
  // one timed batch per candidate and repeat: the best pass time per bucket
  auto run = [&](float* ms) -> int {
    for (int k = 0; k <= kSpBuckets; ++k) ms[k] = -1.f;
    c->timing = true;
    int rc = gcl_canon_batch(c, count, voff, eoff, rowptr, col, color, max_aut, nullptr, nullptr,
                             rows.data(), roff.data(), nullptr, nullptr, status.data());
    c->timing = false;
    if (rc != GCL_OK) return rc;
    for (int k = 0; k <= kSpBuckets; ++k)
      if (c->tev_used[k]) GCL_TRY(cudaEventElapsedTime(&ms[k], c->tev[0][k], c->tev[1][k]));
    return GCL_OK;
  };
  const int saved_w64 = c->tune_w64_bps;
  int saved_bps[kSpBuckets], saved_stage[kSpBuckets];
  for (int bk = 0; bk < kSpBuckets; ++bk) {
    saved_bps[bk] = c->tune_sp_bps[bk];
    saved_stage[bk] = c->tune_sp_stage[bk];
  }
  float ms[1 + kSpBuckets];
  int rc = run(ms);  // warm-up (workspace allocation, first launches)
  // the warp kernel: resident blocks per SM
  float best_w64 = 1e30f;
  int w64_choice = 0;
  const int w64_cands[] = {1, 2, 3, 4, 6, 8, 12, 16};
  for (int ci = 0; rc == GCL_OK && ci < 8; ++ci) {
    if (w64_cands[ci] > c->w64_per_sm) break;
    c->tune_w64_bps = w64_cands[ci];
    float best = 1e30f;
    for (int r = 0; r < repeats && rc == GCL_OK; ++r) {
      rc = run(ms);
      if (ms[0] >= 0) best = std::min(best, ms[0]);
    }
    if (best < best_w64) {
      best_w64 = best;
      w64_choice = w64_cands[ci];
    }
  }
  c->tune_w64_bps = w64_choice;
  // the sparse buckets: shared-memory staging and resident blocks per SM,
  // one candidate for every bucket per batch (the passes are independent)
  float best_sp[kSpBuckets];
  int bps_choice[kSpBuckets], stage_choice[kSpBuckets];
  for (int bk = 0; bk < kSpBuckets; ++bk) {
    best_sp[bk] = 1e30f;
    bps_choice[bk] = 0;
    stage_choice[bk] = -1;
  }
  const int sp_bps[] = {1, 2, 4, 0};
  for (int stage = 1; stage >= 0 && rc == GCL_OK; --stage)
    for (int bi = 0; bi < 4 && rc == GCL_OK; ++bi) {
      for (int bk = 0; bk < kSpBuckets; ++bk) {
        c->tune_sp_stage[bk] = stage;
        c->tune_sp_bps[bk] = sp_bps[bi];
      }
      float best[kSpBuckets];
      for (int bk = 0; bk < kSpBuckets; ++bk) best[bk] = 1e30f;
      for (int r = 0; r < repeats && rc == GCL_OK; ++r) {
        rc = run(ms);
        for (int bk = 0; bk < kSpBuckets; ++bk)
          if (ms[1 + bk] >= 0) best[bk] = std::min(best[bk], ms[1 + bk]);
      }
      for (int bk = 0; bk < kSpBuckets; ++bk)
        if (best[bk] < best_sp[bk]) {
          best_sp[bk] = best[bk];
          bps_choice[bk] = sp_bps[bi];
          stage_choice[bk] = stage;
        }
    }
  if (rc != GCL_OK) {  // leave the context as it was
    c->tune_w64_bps = saved_w64;
    for (int bk = 0; bk < kSpBuckets; ++bk) {
      c->tune_sp_bps[bk] = saved_bps[bk];
      c->tune_sp_stage[bk] = saved_stage[bk];
    }
    return rc;
  }
  out->w64_blocks_per_sm = w64_choice;
  out->w64_ms = best_w64 < 1e30f ? best_w64 : -1.f;
  for (int bk = 0; bk < kSpBuckets; ++bk) {
    const bool seen = best_sp[bk] < 1e30f;
    out->sp_blocks_per_sm[bk] = seen ? bps_choice[bk] : 0;
    out->sp_stage[bk] = seen ? stage_choice[bk] : -1;
    out->sp_ms[bk] = seen ? best_sp[bk] : -1.f;
  }
  return gcl_set_tuning(c, out);
} GCL_CATCH_ALL

}  // extern "C"
