// gcl_files.cu -- canonize DIMACS files with parsing overlapped with the GPU
// (host code on top of the batched entry point).
//
// Files are taken in chunks.  Host threads parse chunk k (gcl_dimacs.h:
// CSRGraph::fromDIMACS semantics, CSRGraph.cpp:40-119) while the GPU
// canonizes chunk k-1; when chunk k-1's copies back have landed its results
// go to the caller's callback, in file order, on the calling thread, and
// chunk k is packed into the pinned arena of its slot and launched.  Two
// slots alternate.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstring>
#include <thread>
#include <utility>
#include <vector>

#include "../../include/gcl.h"
#include "gcl_alloc.h"
#include "gcl_dimacs.h"
#include "gcl_guard.h"

namespace {

struct FGraph : gcl::DimacsGraph {
  int32_t status = 0;  // GCL_GRAPH_OK once parsed
};

// One file through the shared reader; any rejection is bad input, except a
// vertex count above GCL_MAX_N, which is too large.
FGraph parse_file(const char* path) {
  FGraph g;
  const int rc = gcl::read_dimacs_file(path, GCL_MAX_N, &g);
  if (rc != gcl::kDimacsOk) g.status = rc == gcl::kDimacsTooLarge ? GCL_GRAPH_TOO_LARGE : GCL_GRAPH_BAD_INPUT;
  return g;
}

struct Pinned {
  void* p = nullptr;
  size_t cap = 0;
  cudaError_t ensure(size_t b) {
    if (b <= cap && p) return cudaSuccess;
    if (p) cudaFreeHost(p);  // slots are idle when they grow
    p = nullptr;
    cap = 0;
    const size_t want = std::max<size_t>(b + b / 2, 4096);
    cudaError_t e = gcl::pinned_alloc(&p, want);
    if (e == cudaSuccess) cap = want;
    return e;
  }
  ~Pinned() {
    if (p) cudaFreeHost(p);
  }
};

struct Dev {
  void* p = nullptr;
  size_t cap = 0;
  cudaStream_t s = nullptr;
  cudaError_t ensure(size_t b) {
    if (b <= cap && p) return cudaSuccess;
    if (p) cudaFreeAsync(p, s);
    p = nullptr;
    cap = 0;
    const size_t want = std::max<size_t>(b + b / 2, 4096);
    cudaError_t e = gcl::device_alloc(&p, want, s);
    if (e == cudaSuccess) cap = want;
    return e;
  }
  void release() {
    if (p) cudaFreeAsync(p, s);
    p = nullptr;
    cap = 0;
  }
};

struct Slot {
  int64_t first = 0;  // index of the chunk's first file
  std::vector<FGraph> graphs;
  std::vector<int> batch;  // position in the batch of each parsed graph, -1 = bad input
  int count = 0;           // graphs in the batch
  Pinned voff, eoff, rp, col, color, roff, rows, label, stats, status;
  Dev d_voff, d_eoff, d_rp, d_col, d_color, d_roff, d_rows, d_label, d_stats, d_status;
  cudaEvent_t done = nullptr;
  bool busy = false;
  void bind(cudaStream_t s) {
    Dev* ds[] = {&d_voff, &d_eoff, &d_rp, &d_col, &d_color, &d_roff,
                 &d_rows, &d_label, &d_stats, &d_status};
    for (Dev* d : ds) d->s = s;
  }
  void release() {
    Dev* ds[] = {&d_voff, &d_eoff, &d_rp, &d_col, &d_color, &d_roff,
                 &d_rows, &d_label, &d_stats, &d_status};
    for (Dev* d : ds) d->release();
  }
};

int rc_of(cudaError_t e) {
  if (e == cudaSuccess) return GCL_OK;
  return e == cudaErrorMemoryAllocation ? GCL_ERR_NOMEM : GCL_ERR_CUDA;
}

// Parses paths[first, first + cnt) into the slot with up to `threads` host
// threads.  GCL_ERR_NOMEM when a parser ran out of host memory.
int parse_chunk(Slot& sl, const char* const* paths, int64_t first, int64_t cnt, int threads) {
  sl.first = first;
  sl.graphs.assign((size_t)cnt, FGraph());
  std::atomic<int64_t> next{0};
  std::atomic<bool> failed{false};
  auto work = [&] {
    for (int64_t i = next++; i < cnt && !failed.load(); i = next++) {
      try {
        sl.graphs[i] = parse_file(paths[first + i]);
      } catch (...) {
        failed.store(true);
      }
    }
  };
  std::vector<std::thread> pool;
  try {
    pool.reserve((size_t)std::max(threads - 1, 0));
    for (int t = 1; t < threads; ++t) pool.emplace_back(work);
  } catch (...) {
    // fewer helper threads than asked for: the calling thread still parses
  }
  work();
  for (auto& th : pool) th.join();
  return failed.load() ? GCL_ERR_NOMEM : GCL_OK;
}

// pack the chunk's good graphs into the slot's pinned arena and enqueue copy
// in, the batched search and copy out on the context stream
int launch_chunk(gcl_context* c, Slot& sl, int max_aut) {
  cudaStream_t s = (cudaStream_t)gcl_stream(c);
  sl.batch.assign(sl.graphs.size(), -1);
  int count = 0;
  int64_t nv = 0, ne = 0, words = 0;
  int max_n = 0;
  int64_t max_m2 = 0;
  bool colored = false;
  for (size_t i = 0; i < sl.graphs.size(); ++i) {
    const FGraph& g = sl.graphs[i];
    if (g.status) continue;
    sl.batch[i] = count++;
    nv += g.n;
    ne += (int64_t)g.col.size();
    words += (int64_t)g.n * ((g.n + 63) / 64);
    max_n = std::max(max_n, g.n);
    if (g.n > 64) max_m2 = std::max<int64_t>(max_m2, (int64_t)g.col.size());
    colored |= g.colored;
  }
  sl.count = count;
  if (count == 0) return GCL_OK;
  cudaError_t e = cudaSuccess;
  auto ens = [&](Pinned& h, Dev& d, size_t b) {
    if (e == cudaSuccess) e = h.ensure(b);
    if (e == cudaSuccess) e = d.ensure(b);
  };
  ens(sl.voff, sl.d_voff, (count + 1) * 8);
  ens(sl.eoff, sl.d_eoff, (count + 1) * 8);
  ens(sl.rp, sl.d_rp, (size_t)(nv + count) * 4);
  ens(sl.col, sl.d_col, (size_t)std::max<int64_t>(ne, 1) * 4);
  ens(sl.color, sl.d_color, (size_t)std::max<int64_t>(nv, 1) * 4);
  ens(sl.roff, sl.d_roff, (count + 1) * 8);
  ens(sl.rows, sl.d_rows, (size_t)std::max<int64_t>(words, 1) * 8);
  ens(sl.label, sl.d_label, (size_t)std::max<int64_t>(nv, 1) * 4);
  ens(sl.stats, sl.d_stats, (size_t)count * 16);
  ens(sl.status, sl.d_status, (size_t)count * 4);
  if (e != cudaSuccess) return rc_of(e);
  int64_t* voff = (int64_t*)sl.voff.p;
  int64_t* eoff = (int64_t*)sl.eoff.p;
  int64_t* roff = (int64_t*)sl.roff.p;
  int32_t* rp = (int32_t*)sl.rp.p;
  int32_t* col = (int32_t*)sl.col.p;
  int32_t* color = (int32_t*)sl.color.p;
  voff[0] = eoff[0] = roff[0] = 0;
  int b = 0;
  for (const FGraph& g : sl.graphs) {
    if (g.status) continue;
    const int64_t m = (int64_t)g.col.size();
    std::memcpy(rp + voff[b] + b, g.rowptr.data(), (g.n + 1) * sizeof(int32_t));
    if (m) std::memcpy(col + eoff[b], g.col.data(), m * sizeof(int32_t));
    if (colored) std::memcpy(color + voff[b], g.color.data(), g.n * sizeof(int32_t));
    voff[b + 1] = voff[b] + g.n;
    eoff[b + 1] = eoff[b] + m;
    roff[b + 1] = roff[b] + (int64_t)g.n * ((g.n + 63) / 64);
    ++b;
  }
  auto h2d = [&](Dev& d, const Pinned& h, size_t bytes) {
    if (e == cudaSuccess && bytes) e = cudaMemcpyAsync(d.p, h.p, bytes, cudaMemcpyHostToDevice, s);
  };
  h2d(sl.d_voff, sl.voff, (count + 1) * 8);
  h2d(sl.d_eoff, sl.eoff, (count + 1) * 8);
  h2d(sl.d_rp, sl.rp, (size_t)(nv + count) * 4);
  h2d(sl.d_col, sl.col, (size_t)ne * 4);
  if (colored) h2d(sl.d_color, sl.color, (size_t)nv * 4);
  h2d(sl.d_roff, sl.roff, (count + 1) * 8);
  if (e != cudaSuccess) return rc_of(e);
  int rc = gcl_canon_batch_device_async(
      c, count, (int64_t*)sl.d_voff.p, (int64_t*)sl.d_eoff.p, (int32_t*)sl.d_rp.p,
      (int32_t*)sl.d_col.p, colored ? (int32_t*)sl.d_color.p : nullptr, max_aut, max_n, max_m2,
      nullptr, nullptr, (uint64_t*)sl.d_rows.p, (int64_t*)sl.d_roff.p, (int32_t*)sl.d_label.p,
      (int64_t*)sl.d_stats.p, (int32_t*)sl.d_status.p);
  if (rc != GCL_OK) return rc;
  auto d2h = [&](Pinned& h, const Dev& d, size_t bytes) {
    if (e == cudaSuccess && bytes) e = cudaMemcpyAsync(h.p, d.p, bytes, cudaMemcpyDeviceToHost, s);
  };
  d2h(sl.rows, sl.d_rows, (size_t)words * 8);
  d2h(sl.label, sl.d_label, (size_t)nv * 4);
  d2h(sl.stats, sl.d_stats, (size_t)count * 16);
  d2h(sl.status, sl.d_status, (size_t)count * 4);
  if (e == cudaSuccess) e = cudaEventRecord(sl.done, s);
  sl.busy = e == cudaSuccess;
  return rc_of(e);
}

int deliver(Slot& sl, gcl_file_result_fn cb, void* user) {
  if (sl.busy) {
    cudaError_t e = cudaEventSynchronize(sl.done);
    sl.busy = false;
    if (e != cudaSuccess) return rc_of(e);
  }
  const int64_t* voff = (const int64_t*)sl.voff.p;
  const int64_t* roff = (const int64_t*)sl.roff.p;
  for (size_t i = 0; i < sl.graphs.size(); ++i) {
    const int b = sl.batch.empty() ? -1 : sl.batch[i];
    if (b < 0) {
      cb(user, sl.first + (int64_t)i, sl.graphs[i].status ? sl.graphs[i].status : GCL_GRAPH_BAD_INPUT,
         0, nullptr, nullptr, 0, 0);
      continue;
    }
    const int64_t* st = (const int64_t*)sl.stats.p + 2 * b;
    const int32_t status = ((const int32_t*)sl.status.p)[b];
    cb(user, sl.first + (int64_t)i, status, sl.graphs[i].n,
       status ? nullptr : (const uint64_t*)sl.rows.p + roff[b],
       status ? nullptr : (const int32_t*)sl.label.p + voff[b], st[0], st[1]);
  }
  sl.graphs.clear();
  return GCL_OK;
}

}  // namespace

extern "C" int gcl_canon_files(gcl_context* c, int64_t count, const char* const* paths,
                               int max_aut, int chunk, int threads, gcl_file_result_fn cb,
                               void* user) {
  if (!c || count < 0 || (count > 0 && !paths) || max_aut <= 0 || !cb) return GCL_ERR_ARG;
  if (count == 0) return GCL_OK;
  if (chunk <= 0) chunk = 4096;
  if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
  cudaStream_t s = (cudaStream_t)gcl_stream(c);
  Slot slot[2];
  int rc = GCL_OK;
  for (Slot& sl : slot) {
    sl.bind(s);
    if (rc == GCL_OK) rc = rc_of(cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming));
  }
  try {
    int64_t k = 0;
    for (int64_t first = 0; rc == GCL_OK && first < count; first += chunk, ++k) {
      Slot& cur = slot[k & 1];
      Slot& prev = slot[(k + 1) & 1];
      // parse this chunk while the GPU works on the previous one
      rc = parse_chunk(cur, paths, first, std::min<int64_t>(chunk, count - first), threads);
      if (rc == GCL_OK && k > 0) rc = deliver(prev, cb, user);
      if (rc == GCL_OK) rc = launch_chunk(c, cur, max_aut);
    }
    if (rc == GCL_OK && k > 0) rc = deliver(slot[(k - 1) & 1], cb, user);
  } catch (...) {
    rc = gcl::exception_status();
  }
  // copies in flight read and write the slots' pinned buffers
  cudaStreamSynchronize(s);
  for (Slot& sl : slot) {
    sl.release();
    if (sl.done) cudaEventDestroy(sl.done);
  }
  cudaStreamSynchronize(s);
  return rc;
}
