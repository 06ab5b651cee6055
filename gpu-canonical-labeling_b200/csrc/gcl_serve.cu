// gcl_serve.cu -- the serving loop of include/gcl.h: continuous batching
// over several device contexts, a device canonical-hash table and a host
// memo of exact repeats.
//
// One dispatcher thread forms the batches and hands out the results; each
// lane is a gcl_context (its own stream and workspace) with its own launch
// thread.  When a lane is free the dispatcher takes the queued requests that
// fit the lane (graph count, device-memory footprint) and passes them to the
// lane's thread, which packs them into the lane's pinned arena and enqueues
// copy-in, the batched search, the table kernel and copy-out on the lane's
// stream; a host callback at the end of the stream wakes the dispatcher,
// which hands the results to pollers.  Lanes run concurrently, so batches
// formed while others are on the GPU overlap with them, and a lane whose
// enqueueing is slow (a workspace that grows for a larger graph) holds up
// no other lane.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <new>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/gcl.h"
#include "gcl_alloc.h"
#include "gcl_device.cuh"
#include "gcl_guard.h"

namespace gcl {

// ---- device canonical-hash table ----------------------------------------
constexpr uint32_t kNoStore = 0xffffffffu;  // key present, form not stored
constexpr int kTableProbes = 64;
constexpr uint32_t kTableSpin = 1u << 20;  // polls for a form being written

__device__ __forceinline__ uint64_t mix64(uint64_t x) {  // splitmix64 finaliser
  x ^= x >> 30;
  x *= 0xbf58476d1ce4e5b9ull;
  x ^= x >> 27;
  x *= 0x94d049bb133111ebull;
  x ^= x >> 31;
  return x;
}

struct TableArgs {
  int count;
  const int64_t* voff;
  const int64_t* roff;
  const uint64_t* rows;
  const int32_t* status;
  unsigned long long* keys;
  uint32_t* vals;  // 0 = form being written, kNoStore, else store offset + 1
  uint64_t mask;
  uint64_t* store;
  unsigned long long* store_top;
  uint64_t store_words;
  uint64_t* out_hash;
  int64_t* out_class;
  int32_t* out_seen;
};

// One warp per graph: hash the packed canonical rows, then find or insert
// the form.  A key match is confirmed by comparing the stored form in full;
// a different form under the same key probes on.
__global__ void __launch_bounds__(256) canon_table_kernel(TableArgs T) {
  const int warp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int nwarps = (int)((gridDim.x * blockDim.x) >> 5);
  const uint32_t lane = lane_id();
  for (int g = warp; g < T.count; g += nwarps) {
    if (T.status[g] != 0) {
      if (lane == 0) {
        T.out_hash[g] = 0;
        T.out_class[g] = -1;
        T.out_seen[g] = 0;
      }
      continue;
    }
    const uint64_t n = (uint64_t)(T.voff[g + 1] - T.voff[g]);
    const uint64_t words = (uint64_t)(T.roff[g + 1] - T.roff[g]);
    const uint64_t* r = T.rows + T.roff[g];
    uint64_t h = 0;
    for (uint64_t i = lane; i < words; i += 32) h += mix64(r[i] ^ mix64(i + 0x9e3779b97f4a7c15ull));
    for (int o = 16; o > 0; o >>= 1) h += bcast64(h, (int)(lane ^ (uint32_t)o));
    h = mix64(h ^ mix64(n + 0x632be59bd9b4e019ull));
    if (h == 0) h = 1;
    int64_t cls = -1;
    int seen = 0;
    uint64_t slot = h & T.mask;
    for (int p = 0; p < kTableProbes; ++p, slot = (slot + 1) & T.mask) {
      unsigned long long k = 0;
      if (lane == 0) k = atomicCAS(&T.keys[slot], 0ull, (unsigned long long)h);
      k = bcast64(k, 0);
      if (k == 0) {  // claimed: a new class, keep its form
        unsigned long long off = 0;
        if (lane == 0) off = atomicAdd(T.store_top, (unsigned long long)(words + 1));
        off = bcast64(off, 0);
        const bool fits = off + words + 1 <= T.store_words && off + 1 < kNoStore;
        if (fits) {
          for (uint64_t i = lane; i < words; i += 32) T.store[off + 1 + i] = r[i];
          if (lane == 0) T.store[off] = n;
        }
        __threadfence();
        __syncwarp();
        if (lane == 0) atomicExch(&T.vals[slot], fits ? (uint32_t)(off + 1) : kNoStore);
        cls = (int64_t)slot;
        break;
      }
      if (k != h) continue;
      uint32_t v = 0;
      if (lane == 0) {
        for (uint32_t s = 0; s < kTableSpin; ++s) {
          v = *(volatile uint32_t*)&T.vals[slot];
          if (v) break;
          __nanosleep(128);
        }
        __threadfence();
      }
      v = __shfl_sync(GCL_FULL, v, 0);
      if (v == 0 || v == kNoStore) break;  // unconfirmable: class unknown
      const uint64_t* st = T.store + (v - 1);
      bool eq = __ldcg((const unsigned long long*)st) == n;
      for (uint64_t i = lane; eq && i < words; i += 32)
        eq = __ldcg((const unsigned long long*)st + 1 + i) == r[i];
      if (__all_sync(GCL_FULL, eq)) {
        cls = (int64_t)slot;
        seen = 1;
        break;
      }
    }
    if (lane == 0) {
      T.out_hash[g] = h;
      T.out_class[g] = cls;
      T.out_seen[g] = seen;
    }
  }
}

}  // namespace gcl

using namespace gcl;

namespace {

using Clock = std::chrono::steady_clock;

// Pinned host buffer.  Freeing pinned memory waits for the whole device, so
// a buffer that grows keeps its old allocation until the server is
// destroyed (growth is geometric, so the retired ones add up to less than
// twice the final size).
struct HostBuf {
  void* p = nullptr;
  size_t cap = 0;
  std::vector<void*> retired;
  cudaError_t ensure(size_t bytes) {
    if (bytes <= cap && p) return cudaSuccess;
    const size_t want = std::max<size_t>(std::max<size_t>(bytes, 4096), 2 * cap);
    void* q = nullptr;
    cudaError_t e = pinned_alloc(&q, want);
    if (e != cudaSuccess) return e;
    if (p) retired.push_back(p);
    p = q;
    cap = want;
    return cudaSuccess;
  }
  void release() {
    for (void* q : retired) cudaFreeHost(q);
    retired.clear();
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
  }
  template <typename T>
  T* as() const {
    return (T*)p;
  }
};

// Device buffer allocated in stream order on its lane's stream (no wait for
// the other lanes when it grows).
struct DevMem {
  void* p = nullptr;
  size_t cap = 0;
  cudaStream_t stream = nullptr;
  cudaError_t ensure(size_t bytes) {
    if (bytes <= cap && p) return cudaSuccess;
    const size_t want = std::max<size_t>(std::max<size_t>(bytes, 4096), 2 * cap);
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
  template <typename T>
  T* as() const {
    return (T*)p;
  }
};

struct Graph {
  int n = 0;
  std::vector<int32_t> rp, col, color;  // color empty = uncoloured
};

uint64_t fnv_mix(uint64_t h, uint64_t x) {
  h ^= x + 0x9e3779b97f4a7c15ull + (h << 6) + (h >> 2);
  return h * 0x100000001b3ull;
}

uint64_t input_key(const Graph& g) {
  uint64_t h = fnv_mix(0xcbf29ce484222325ull, (uint64_t)g.n);
  for (int32_t x : g.rp) h = fnv_mix(h, (uint32_t)x);
  for (int32_t x : g.col) h = fnv_mix(h, (uint32_t)x);
  h = fnv_mix(h, g.color.empty() ? 0 : 1);
  for (int32_t x : g.color) h = fnv_mix(h, (uint32_t)x);
  return h;
}

bool same_input(const Graph& a, const Graph& b) {
  return a.n == b.n && a.rp == b.rp && a.col == b.col && a.color == b.color;
}

struct Req {
  int64_t id = 0;
  int kind = GCL_REQ_CANON;
  int ng = 1;
  Graph g[2];
  uint64_t key[2] = {0, 0};
  uint64_t* out_rows = nullptr;
  int32_t* out_label = nullptr;
  Clock::time_point t0, t_admit, t_launch;
};

struct MemoEntry {
  Graph in;
  std::vector<uint64_t> rows;
  std::vector<int32_t> label;
  int64_t cls = -1;
  uint64_t hash = 0;
};

// Request classes by the larger graph's n: small (the warp kernel for
// n <= 64, microseconds), mid and big (the sparse warp kernel: milliseconds,
// tenths of seconds), large (the wide search).  Each class has its own
// queue, lanes and batch-size cap, so a batch never waits for a graph of a
// slower class.
enum { kSmall = 0, kMid = 1, kBig = 2, kLarge = 3, kClasses = 4 };

struct Lane {
  Clock::time_point t_launch;
  // the lane's launch thread: the dispatcher sets `go` (under the server's
  // lock) once the batch is in `reqs`; a failed enqueue leaves its status in
  // launch_rc and marks the lane ready
  std::thread worker;
  std::condition_variable cv_go;
  bool go = false, quit = false;
  int launch_rc = GCL_OK;
  std::pair<gcl_server*, Lane*> cbarg{nullptr, nullptr};
  std::atomic<int64_t> t_gpu_done{0};  // steady-clock ns when the stream reached the batch's end
  gcl_context* ctx = nullptr;
  cudaStream_t s = nullptr;
  int cls = kSmall;
  bool large = false;
  bool busy = false;
  std::atomic<bool> ready{false};
  std::vector<Req*> reqs;
  std::vector<int> first;  // graph index of each request in the batch
  int count = 0;
  int err = GCL_OK;
  HostBuf h_voff, h_eoff, h_rp, h_col, h_color, h_roff, h_rows, h_label, h_status, h_hash, h_class,
      h_seen;
  DevMem d_voff, d_eoff, d_rp, d_col, d_color, d_roff, d_rows, d_label, d_status, d_hash, d_class,
      d_seen;
  void release() {
    HostBuf* hb[] = {&h_voff, &h_eoff, &h_rp, &h_col, &h_color, &h_roff, &h_rows, &h_label,
                     &h_status, &h_hash, &h_class, &h_seen};
    DevMem* db[] = {&d_voff, &d_eoff, &d_rp, &d_col, &d_color, &d_roff, &d_rows, &d_label,
                    &d_status, &d_hash, &d_class, &d_seen};
    for (auto* b : hb) b->release();
    for (auto* b : db) b->release();
  }
};

int rc_of(cudaError_t e) {
  if (e == cudaSuccess) return GCL_OK;
  return e == cudaErrorMemoryAllocation ? GCL_ERR_NOMEM : GCL_ERR_CUDA;
}

int graph_rc(int32_t s) {
  switch (s) {
    case 0: return GCL_OK;
    case 3: return GCL_ERR_BAD_INPUT;
    case 2: return GCL_ERR_TOO_LARGE;
    case 5: return GCL_ERR_TIMEOUT;
    default: return GCL_ERR_INTERNAL;
  }
}

// Device bytes a graph holds while its batch runs: CSR in, packed rows and
// labeling out, and one search slot of the sparse kernel for n > 64.
int64_t footprint(const Graph& g) {
  const int64_t n = g.n, m = (int64_t)g.col.size();
  int64_t b = 4 * (2 * n + 1 + m) + 8 * n * ((n + 63) / 64) + 4 * n + 64;
  if (n > 64) b += 4 * (25 * (n + 2)) + 12 * (m + 1) + 8 * 32 * ((n + 63) / 64 + 2);
  return b;
}

}  // namespace

struct gcl_server {
  int device = 0;
  gcl_serve_config cfg{};
  std::vector<Lane*> lanes;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Req*> q[kClasses];
  int max_batch[kClasses] = {0, 0, 0, 1};
  std::deque<gcl_serve_result> done;
  std::thread th;
  bool stop = false;
  // device table
  DevMem keys, vals, store, top;
  // host memo of exact repeats
  std::mutex memo_mu;
  std::unordered_map<uint64_t, MemoEntry> memo;
  std::deque<uint64_t> memo_fifo;
  int64_t memo_used = 0;
  gcl_serve_stats st{};
};

namespace {

void CUDART_CB lane_done_cb(void* arg) {
  auto* pr = (std::pair<gcl_server*, Lane*>*)arg;
  pr->second->t_gpu_done.store(
      std::chrono::duration_cast<std::chrono::nanoseconds>(Clock::now().time_since_epoch()).count());
  {
    std::lock_guard<std::mutex> lk(pr->first->mu);
    pr->second->ready.store(true);
  }
  pr->first->cv_work.notify_one();
}

void push_done(gcl_server* S, const gcl_serve_result& r) {
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->done.push_back(r);
    S->st.completed += 1;
  }
  S->cv_done.notify_all();
}

void memo_put(gcl_server* S, const Graph& g, uint64_t key, const uint64_t* rows, size_t words,
              const int32_t* label, int64_t cls, uint64_t hash) {
  if (S->cfg.memo_bytes <= 0) return;
  const int64_t bytes = (int64_t)(4 * (g.rp.size() + g.col.size() + g.color.size()) +
                                  8 * words + 4 * (size_t)g.n + 128);
  if (bytes > S->cfg.memo_bytes / 4) return;
  std::lock_guard<std::mutex> lk(S->memo_mu);
  if (S->memo.count(key)) return;
  while (S->memo_used + bytes > S->cfg.memo_bytes && !S->memo_fifo.empty()) {
    auto it = S->memo.find(S->memo_fifo.front());
    S->memo_fifo.pop_front();
    if (it != S->memo.end()) {
      const MemoEntry& e = it->second;
      S->memo_used -= (int64_t)(4 * (e.in.rp.size() + e.in.col.size() + e.in.color.size()) +
                                8 * e.rows.size() + 4 * e.label.size() + 128);
      S->memo.erase(it);
    }
  }
  try {
    MemoEntry e;
    e.in = g;
    e.rows.assign(rows, rows + words);
    e.label.assign(label, label + g.n);
    e.cls = cls;
    e.hash = hash;
    auto ins = S->memo.emplace(key, std::move(e));
    try {
      S->memo_fifo.push_back(key);
    } catch (...) {
      S->memo.erase(ins.first);
      throw;
    }
    S->memo_used += bytes;
  } catch (...) {
    // the memo is a cache: an entry that finds no host memory is not kept
  }
}

bool memo_get(gcl_server* S, const Graph& g, uint64_t key, MemoEntry* out) {
  if (S->cfg.memo_bytes <= 0) return false;
  std::lock_guard<std::mutex> lk(S->memo_mu);
  auto it = S->memo.find(key);
  if (it == S->memo.end() || !same_input(it->second.in, g)) return false;
  *out = it->second;
  return true;
}

// Requests for a free lane: FIFO from the lane's queue while the batch stays
// within max_batch graphs and the lane's device-memory budget (a large lane
// takes one request).  Called with S->mu held.
std::vector<Req*> take_batch(gcl_server* S, Lane* L) {
  std::vector<Req*> out;
  std::deque<Req*>& q = S->q[L->cls];
  int graphs = 0;
  int64_t bytes = 0;
  while (!q.empty()) {
    Req* r = q.front();
    int64_t b = 0;
    for (int i = 0; i < r->ng; ++i) b += footprint(r->g[i]);
    if (!out.empty() &&
        (graphs + r->ng > S->max_batch[L->cls] || bytes + b > S->cfg.lane_bytes))
      break;
    q.pop_front();
    out.push_back(r);
    graphs += r->ng;
    bytes += b;
    if (L->large) break;
  }
  return out;
}

// Sizes a lane's host and device buffers up front for batches of `graphs`
// graphs with `verts` vertices, `edges` CSR entries and `words` packed-row
// words in all, so that serving does not allocate pinned memory: pinning
// pages takes the driver's lock, and every other lane's CUDA calls waited
// behind it (hundreds of ms under load).  Larger batches still grow them.
cudaError_t lane_reserve(Lane* L, int64_t graphs, int64_t verts, int64_t edges, int64_t words) {
  cudaError_t e = cudaSuccess;
  auto ens = [&](HostBuf& h, DevMem& d, size_t bytes) {
    if (e == cudaSuccess) e = h.ensure(bytes);
    if (e == cudaSuccess) e = d.ensure(bytes);
  };
  ens(L->h_voff, L->d_voff, (size_t)(graphs + 1) * 8);
  ens(L->h_eoff, L->d_eoff, (size_t)(graphs + 1) * 8);
  ens(L->h_rp, L->d_rp, (size_t)(verts + graphs) * 4);
  ens(L->h_col, L->d_col, (size_t)edges * 4);
  ens(L->h_color, L->d_color, (size_t)verts * 4);
  ens(L->h_roff, L->d_roff, (size_t)(graphs + 1) * 8);
  ens(L->h_rows, L->d_rows, (size_t)words * 8);
  ens(L->h_label, L->d_label, (size_t)verts * 4);
  ens(L->h_status, L->d_status, (size_t)graphs * 4);
  ens(L->h_hash, L->d_hash, (size_t)graphs * 8);
  ens(L->h_class, L->d_class, (size_t)graphs * 8);
  ens(L->h_seen, L->d_seen, (size_t)graphs * 4);
  return e;
}

int launch(gcl_server* S, Lane* L) {
  int count = 0;
  int64_t nv = 0, ne = 0, words = 0;
  int max_n = 0;
  int64_t max_m2 = 0;
  bool colored = false;
  L->first.clear();
  for (Req* r : L->reqs) {
    L->first.push_back(count);
    for (int i = 0; i < r->ng; ++i) {
      const Graph& g = r->g[i];
      ++count;
      nv += g.n;
      ne += (int64_t)g.col.size();
      words += (int64_t)g.n * ((g.n + 63) / 64);
      max_n = std::max(max_n, g.n);
      if (g.n > 64) max_m2 = std::max<int64_t>(max_m2, (int64_t)g.col.size());
      colored |= !g.color.empty();
    }
  }
  L->count = count;
  cudaError_t e = cudaSuccess;
  int64_t part[6] = {0, 0, 0, 0, 0, 0};
  auto since = [](Clock::time_point t) {
    return std::chrono::duration_cast<std::chrono::nanoseconds>(Clock::now() - t).count();
  };
  auto ens = [&](HostBuf& h, DevMem& d, size_t bytes) {
    Clock::time_point t = Clock::now();
    if (e == cudaSuccess) e = h.ensure(bytes);
    part[0] += since(t);
    t = Clock::now();
    if (e == cudaSuccess) e = d.ensure(bytes);
    part[1] += since(t);
  };
  auto report = [&] {
    std::lock_guard<std::mutex> lk(S->mu);
    for (int k = 0; k < 6; ++k)
      S->st.enqueue_part_max_ns[k] = std::max(S->st.enqueue_part_max_ns[k], part[k]);
  };
  ens(L->h_voff, L->d_voff, (count + 1) * 8);
  ens(L->h_eoff, L->d_eoff, (count + 1) * 8);
  ens(L->h_rp, L->d_rp, (size_t)(nv + count) * 4);
  ens(L->h_col, L->d_col, (size_t)std::max<int64_t>(ne, 1) * 4);
  ens(L->h_color, L->d_color, (size_t)std::max<int64_t>(nv, 1) * 4);
  ens(L->h_roff, L->d_roff, (count + 1) * 8);
  ens(L->h_rows, L->d_rows, (size_t)std::max<int64_t>(words, 1) * 8);
  ens(L->h_label, L->d_label, (size_t)std::max<int64_t>(nv, 1) * 4);
  ens(L->h_status, L->d_status, (size_t)count * 4);
  ens(L->h_hash, L->d_hash, (size_t)count * 8);
  ens(L->h_class, L->d_class, (size_t)count * 8);
  ens(L->h_seen, L->d_seen, (size_t)count * 4);
  if (e != cudaSuccess) return rc_of(e);
  Clock::time_point tp = Clock::now();
  int64_t* voff = L->h_voff.as<int64_t>();
  int64_t* eoff = L->h_eoff.as<int64_t>();
  int64_t* roff = L->h_roff.as<int64_t>();
  int32_t* rp = L->h_rp.as<int32_t>();
  int32_t* col = L->h_col.as<int32_t>();
  int32_t* color = L->h_color.as<int32_t>();
  voff[0] = eoff[0] = roff[0] = 0;
  int gi = 0;
  for (Req* r : L->reqs)
    for (int i = 0; i < r->ng; ++i, ++gi) {
      const Graph& g = r->g[i];
      const int64_t m = (int64_t)g.col.size();
      std::memcpy(rp + voff[gi] + gi, g.rp.data(), (g.n + 1) * sizeof(int32_t));
      if (m) std::memcpy(col + eoff[gi], g.col.data(), m * sizeof(int32_t));
      if (colored) {
        if (g.color.empty())
          std::memset(color + voff[gi], 0, g.n * sizeof(int32_t));
        else
          std::memcpy(color + voff[gi], g.color.data(), g.n * sizeof(int32_t));
      }
      voff[gi + 1] = voff[gi] + g.n;
      eoff[gi + 1] = eoff[gi] + m;
      roff[gi + 1] = roff[gi] + (int64_t)g.n * ((g.n + 63) / 64);
    }
  part[2] = since(tp);
  tp = Clock::now();
  cudaStream_t s = L->s;
  auto h2d = [&](DevMem& d, const HostBuf& h, size_t bytes) {
    if (e == cudaSuccess && bytes) e = cudaMemcpyAsync(d.p, h.p, bytes, cudaMemcpyHostToDevice, s);
  };
  h2d(L->d_voff, L->h_voff, (count + 1) * 8);
  h2d(L->d_eoff, L->h_eoff, (count + 1) * 8);
  h2d(L->d_rp, L->h_rp, (size_t)(nv + count) * 4);
  h2d(L->d_col, L->h_col, (size_t)ne * 4);
  if (colored) h2d(L->d_color, L->h_color, (size_t)nv * 4);
  h2d(L->d_roff, L->h_roff, (count + 1) * 8);
  if (e != cudaSuccess) return rc_of(e);
  part[3] = since(tp);
  tp = Clock::now();
  int rc = GCL_OK;
  const int32_t* d_color = colored ? L->d_color.as<int32_t>() : nullptr;
  if (L->large) {
    // one request: each graph through the wide search
    for (int g = 0; g < count && rc == GCL_OK; ++g) {
      const int n = (int)(voff[g + 1] - voff[g]);
      if (n == 0) {
        e = cudaMemsetAsync(L->d_status.as<int32_t>() + g, 0, 4, s);
        continue;
      }
      rc = gcl_canon_wide_device_async(
          L->ctx, L->d_rp.as<int32_t>() + voff[g] + g, L->d_col.as<int32_t>() + eoff[g],
          d_color ? d_color + voff[g] : nullptr, n, eoff[g + 1] - eoff[g], S->cfg.max_aut,
          nullptr, L->d_rows.as<uint64_t>() + roff[g], L->d_label.as<int32_t>() + voff[g],
          nullptr, L->d_status.as<int32_t>() + g);
    }
  } else {
    rc = gcl_canon_batch_device_async(L->ctx, count, L->d_voff.as<int64_t>(),
                                      L->d_eoff.as<int64_t>(), L->d_rp.as<int32_t>(),
                                      L->d_col.as<int32_t>(), d_color, S->cfg.max_aut, max_n,
                                      max_m2, nullptr, nullptr, L->d_rows.as<uint64_t>(),
                                      L->d_roff.as<int64_t>(), L->d_label.as<int32_t>(), nullptr,
                                      L->d_status.as<int32_t>());
  }
  part[4] = since(tp);
  tp = Clock::now();
  if (rc != GCL_OK) return rc;
  if (e != cudaSuccess) return rc_of(e);
  TableArgs T;
  T.count = count;
  T.voff = L->d_voff.as<int64_t>();
  T.roff = L->d_roff.as<int64_t>();
  T.rows = L->d_rows.as<uint64_t>();
  T.status = L->d_status.as<int32_t>();
  T.keys = S->keys.as<unsigned long long>();
  T.vals = S->vals.as<uint32_t>();
  T.mask = (uint64_t)S->cfg.table_slots - 1;
  T.store = S->store.as<uint64_t>();
  T.store_top = S->top.as<unsigned long long>();
  T.store_words = (uint64_t)S->cfg.store_bytes / 8;
  T.out_hash = L->d_hash.as<uint64_t>();
  T.out_class = L->d_class.as<int64_t>();
  T.out_seen = L->d_seen.as<int32_t>();
  const int blocks = std::min(1024, (count + 7) / 8);
  canon_table_kernel<<<blocks, 256, 0, s>>>(T);
  e = cudaGetLastError();
  auto d2h = [&](HostBuf& h, const DevMem& d, size_t bytes) {
    if (e == cudaSuccess && bytes) e = cudaMemcpyAsync(h.p, d.p, bytes, cudaMemcpyDeviceToHost, s);
  };
  d2h(L->h_rows, L->d_rows, (size_t)words * 8);
  d2h(L->h_label, L->d_label, (size_t)nv * 4);
  d2h(L->h_status, L->d_status, (size_t)count * 4);
  d2h(L->h_hash, L->d_hash, (size_t)count * 8);
  d2h(L->h_class, L->d_class, (size_t)count * 8);
  d2h(L->h_seen, L->d_seen, (size_t)count * 4);
  part[5] = since(tp);
  report();
  if (e != cudaSuccess) return rc_of(e);
  return GCL_OK;
}

void complete(gcl_server* S, Lane* L) {
  const int64_t* voff = L->h_voff.as<int64_t>();
  const int64_t* roff = L->h_roff.as<int64_t>();
  const int32_t* status = L->h_status.as<int32_t>();
  const uint64_t* hash = L->h_hash.as<uint64_t>();
  const int64_t* cls = L->h_class.as<int64_t>();
  const int32_t* seen = L->h_seen.as<int32_t>();
  const uint64_t* rows = L->h_rows.as<uint64_t>();
  const int32_t* label = L->h_label.as<int32_t>();
  const Clock::time_point now = Clock::now();
  const Clock::time_point t_gpu{std::chrono::duration_cast<Clock::duration>(
      std::chrono::nanoseconds(L->t_gpu_done.load()))};
  int64_t repeats = 0, classes = 0;
  for (size_t k = 0; k < L->reqs.size(); ++k) {
    Req* r = L->reqs[k];
    const int g = L->first[k];
    if (L->large && L->err == GCL_OK) {
      // a wide search that ran out of per-warp orbit storage (or failed an
      // internal check) has no result: the request goes to lanes of the
      // batched sequential search (big, or mid when the big lanes are wide),
      // which reruns it with full storage
      bool retry = false;
      for (int i = 0; i < r->ng; ++i) retry |= status[g + i] == 1 || status[g + i] == 4;
      if (retry) {
        std::lock_guard<std::mutex> lk(S->mu);
        S->q[S->cfg.big_wide ? kMid : kBig].push_back(r);
        continue;
      }
    }
    gcl_serve_result res;
    std::memset(&res, 0, sizeof res);
    res.id = r->id;
    res.verdict = -1;
    res.batch = L->count;
    res.class_id = -1;
    int rc = L->err;
    for (int i = 0; rc == GCL_OK && i < r->ng; ++i) rc = graph_rc(status[g + i]);
    res.status = rc;
    if (rc == GCL_OK) {
      res.class_id = cls[g];
      res.canon_hash = hash[g];
      res.repeat = seen[g] ? 1 : 0;
      for (int i = 0; i < r->ng; ++i) {
        if (seen[g + i]) ++repeats;
        else if (cls[g + i] >= 0) ++classes;
      }
      const size_t w0 = (size_t)(roff[g + 1] - roff[g]);
      if (r->kind == GCL_REQ_CANON) {
        if (r->out_rows) std::memcpy(r->out_rows, rows + roff[g], w0 * 8);
        if (r->out_label) std::memcpy(r->out_label, label + voff[g], (size_t)r->g[0].n * 4);
        memo_put(S, r->g[0], r->key[0], rows + roff[g], w0, label + voff[g], cls[g], hash[g]);
      } else {
        const size_t w1 = (size_t)(roff[g + 2] - roff[g + 1]);
        res.verdict = r->g[0].n == r->g[1].n && hash[g] == hash[g + 1] && w0 == w1 &&
                      std::memcmp(rows + roff[g], rows + roff[g + 1], w0 * 8) == 0;
        for (int i = 0; i < 2; ++i)
          memo_put(S, r->g[i], r->key[i], rows + roff[g + i], (size_t)(roff[g + i + 1] - roff[g + i]),
                   label + voff[g + i], cls[g + i], hash[g + i]);
      }
    }
    res.latency_s = std::chrono::duration<double>(now - r->t0).count();
    res.admit_s = std::chrono::duration<double>(r->t_admit - r->t0).count();
    res.launch_s = std::chrono::duration<double>(r->t_launch - r->t0).count();
    res.gpu_done_s = std::chrono::duration<double>(t_gpu - r->t0).count();
    push_done(S, res);
    delete r;
  }
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->st.batches += 1;
    S->st.class_batches[L->cls] += 1;
    S->st.class_batch_ns[L->cls] +=
        std::chrono::duration_cast<std::chrono::nanoseconds>(now - L->t_launch).count();
    S->st.graphs += L->count;
    S->st.class_repeats += repeats;
    S->st.classes += classes;
    if (L->large) S->st.large_graphs += L->count;
  }
  L->reqs.clear();
  L->busy = false;
  L->ready.store(false);
}

void fail_batch(gcl_server* S, Lane* L, int rc) {
  L->err = rc;
  // nothing usable was produced: report the error for every request
  const Clock::time_point now = Clock::now();
  for (Req* r : L->reqs) {
    gcl_serve_result res;
    std::memset(&res, 0, sizeof res);
    res.id = r->id;
    res.status = rc;
    res.verdict = -1;
    res.class_id = -1;
    res.latency_s = std::chrono::duration<double>(now - r->t0).count();
    push_done(S, res);
    delete r;
  }
  L->reqs.clear();
  L->busy = false;
  L->err = GCL_OK;
}

// A lane's launch thread: packs and enqueues each batch the dispatcher hands
// it.  The requests' enqueue time is stamped before the completion callback
// is enqueued, since the dispatcher may finish (and free) them as soon as
// the callback has run.
void lane_worker(gcl_server* S, Lane* L) {
  cudaSetDevice(S->device);
  while (true) {
    {
      std::unique_lock<std::mutex> lk(S->mu);
      L->cv_go.wait(lk, [&] { return L->go || L->quit; });
      if (!L->go) break;
      L->go = false;
    }
    int rc = launch(S, L);
    const Clock::time_point tl = Clock::now();
    for (Req* r : L->reqs) r->t_launch = tl;
    const int64_t dt =
        std::chrono::duration_cast<std::chrono::nanoseconds>(tl - L->t_launch).count();
    {
      std::lock_guard<std::mutex> lk(S->mu);
      S->st.class_max_launch_ns[L->cls] = std::max(S->st.class_max_launch_ns[L->cls], dt);
    }
    if (rc == GCL_OK) {
      const cudaError_t e = cudaLaunchHostFunc(L->s, lane_done_cb, &L->cbarg);
      if (e != cudaSuccess) rc = rc_of(e);
    }
    if (rc != GCL_OK) {
      {
        std::lock_guard<std::mutex> lk(S->mu);
        L->launch_rc = rc;
        L->ready.store(true);
      }
      S->cv_work.notify_one();
    }
  }
}

void dispatcher(gcl_server* S) {
  cudaSetDevice(S->device);
  while (true) {
    bool progress = false;
    for (size_t i = 0; i < S->lanes.size(); ++i) {
      Lane* L = S->lanes[i];
      if (L->busy && L->ready.load()) {
        const Clock::time_point tc = Clock::now();
        const int cls = L->cls;
        if (L->launch_rc != GCL_OK) {
          // the enqueue failed: drain what was queued, report the error
          cudaStreamSynchronize(L->s);
          const int rc = L->launch_rc;
          L->launch_rc = GCL_OK;
          fail_batch(S, L, rc);
        } else if (cudaStreamQuery(L->s) == cudaSuccess) {
          complete(S, L);
        } else {
          cudaError_t e = cudaStreamSynchronize(L->s);
          if (e == cudaSuccess)
            complete(S, L);
          else
            fail_batch(S, L, rc_of(e));
        }
        const int64_t dt =
            std::chrono::duration_cast<std::chrono::nanoseconds>(Clock::now() - tc).count();
        {
          std::lock_guard<std::mutex> lk(S->mu);
          S->st.class_max_complete_ns[cls] = std::max(S->st.class_max_complete_ns[cls], dt);
        }
        progress = true;
      }
    }
    for (size_t i = 0; i < S->lanes.size(); ++i) {
      Lane* L = S->lanes[i];
      if (L->busy) continue;
      {
        std::lock_guard<std::mutex> lk(S->mu);
        L->reqs = take_batch(S, L);
      }
      if (L->reqs.empty()) continue;
      L->busy = true;
      L->t_launch = Clock::now();
      {
        int64_t q = 0;
        for (Req* r : L->reqs) {
          r->t_admit = L->t_launch;
          q += std::chrono::duration_cast<std::chrono::nanoseconds>(L->t_launch - r->t0).count();
        }
        std::lock_guard<std::mutex> lk(S->mu);
        S->st.class_queue_ns[L->cls] += q / (int64_t)L->reqs.size();
      }
      L->ready.store(false);
      L->t_gpu_done.store(0);
      {
        std::lock_guard<std::mutex> lk(S->mu);
        L->launch_rc = GCL_OK;
        L->go = true;
      }
      L->cv_go.notify_one();
      progress = true;
    }
    std::unique_lock<std::mutex> lk(S->mu);
    bool any_busy = false, any_ready = false;
    for (Lane* L : S->lanes) {
      any_busy |= L->busy;
      any_ready |= L->busy && L->ready.load();
    }
    bool queued = false;
    for (auto& q : S->q) queued |= !q.empty();
    if (S->stop && !any_busy && !queued) break;
    if (progress || any_ready) continue;
    bool can_launch = false;
    for (Lane* L : S->lanes)
      if (!L->busy && !S->q[L->cls].empty()) can_launch = true;
    if (can_launch) continue;
    S->cv_work.wait_for(lk, std::chrono::milliseconds(2));
  }
}

void submit_done_now(gcl_server* S, Req* r, const gcl_serve_result& res) {
  gcl_serve_result x = res;
  x.latency_s = std::chrono::duration<double>(Clock::now() - r->t0).count();
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->st.memo_hits += 1;
  }
  push_done(S, x);
}

bool copy_graph(Graph& g, const int32_t* rp, const int32_t* col, const int32_t* color, int n) {
  if (n < 0 || n > GCL_MAX_N || !rp) return false;
  const int64_t m = rp[n];
  if (rp[0] != 0 || m < 0 || (m > 0 && !col)) return false;
  g.n = n;
  g.rp.assign(rp, rp + n + 1);
  g.col.assign(col ? col : rp, col ? col + m : rp);
  if (color)
    g.color.assign(color, color + n);
  else
    g.color.clear();
  return true;
}

// Frees the lanes (each on its own stream, before its context goes), the
// device table and the server itself.  The dispatcher must not be running;
// the lanes' launch threads are stopped here.
void teardown(gcl_server* S) {
  cudaSetDevice(S->device);
  for (Lane* L : S->lanes) {
    {
      std::lock_guard<std::mutex> lk(S->mu);
      L->quit = true;
    }
    L->cv_go.notify_all();
    if (L->worker.joinable()) L->worker.join();
  }
  for (Lane* L : S->lanes) {
    if (L->s) cudaStreamSynchronize(L->s);
    L->release();
    if (L->ctx) gcl_destroy(L->ctx);
    delete L;
  }
  S->keys.release();
  S->vals.release();
  S->store.release();
  S->top.release();
  cudaDeviceSynchronize();
  delete S;
}

}  // namespace

extern "C" {

int gcl_serve_create(int device, const gcl_serve_config* cfg, gcl_server** out) try {
  if (!out) return GCL_ERR_ARG;
  *out = nullptr;
  gcl_serve_config c{};
  if (cfg) c = *cfg;
  if (c.lanes <= 0) c.lanes = 3;
  if (c.mid_lanes <= 0) c.mid_lanes = 3;
  if (c.big_lanes <= 0) c.big_lanes = 8;
  if (c.large_lanes <= 0) c.large_lanes = 4;
  if (c.max_batch <= 0) c.max_batch = 8192;
  if (c.mid_batch <= 0) c.mid_batch = 512;
  if (c.big_batch <= 0) c.big_batch = 8;
  if (c.mid_n <= 0) c.mid_n = 65;
  if (c.big_n <= 0) c.big_n = 257;
  if (c.large_n <= 0) c.large_n = 2049;
  if (c.max_aut <= 0) c.max_aut = 10000;
  if (c.lane_bytes <= 0) c.lane_bytes = 256ll << 20;
  if (c.table_slots <= 0) c.table_slots = 1ll << 20;
  if (c.store_bytes <= 0) c.store_bytes = 256ll << 20;
  if (c.memo_bytes == 0) c.memo_bytes = 64ll << 20;
  if (c.memo_bytes < 0) c.memo_bytes = 0;  // off
  if ((c.table_slots & (c.table_slots - 1)) != 0 || c.big_n < c.mid_n || c.large_n < c.big_n)
    return GCL_ERR_ARG;
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return rc_of(e);
  gcl_server* S = new (std::nothrow) gcl_server();
  if (!S) return GCL_ERR_NOMEM;
  S->device = device;
  S->cfg = c;
  S->max_batch[kSmall] = c.max_batch;
  S->max_batch[kMid] = c.mid_batch;
  S->max_batch[kBig] = c.big_wide ? 1 : c.big_batch;
  S->max_batch[kLarge] = 1;
  int rc = GCL_OK;
  int dev_sms = 0;
  cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, device);
  const int nl[kClasses] = {c.lanes, c.mid_lanes, c.big_lanes, c.large_lanes};
  try {
    S->lanes.reserve((size_t)(nl[0] + nl[1] + nl[2] + nl[3]));
  } catch (...) {
    delete S;
    throw;
  }
  for (int i = 0; i < nl[0] + nl[1] + nl[2] + nl[3] && rc == GCL_OK; ++i) {
    Lane* L = new (std::nothrow) Lane();
    if (!L) {
      rc = GCL_ERR_NOMEM;
      break;
    }
    L->cls = i < nl[0] ? kSmall : i < nl[0] + nl[1] ? kMid : i < nl[0] + nl[1] + nl[2] ? kBig : kLarge;
    // lanes whose requests go through the wide search one at a time
    L->large = L->cls == kLarge || (c.big_wide && L->cls == kBig);
    S->lanes.push_back(L);
    rc = gcl_create(device, &L->ctx);
    // short work first: small and mid lanes get high-priority streams
    if (rc == GCL_OK)
      rc = gcl_set_option(L->ctx, GCL_OPT_STREAM_PRIORITY,
                          L->cls == kSmall || L->cls == kMid ? 1 : 0);
    if (rc == GCL_OK) {
      L->s = (cudaStream_t)gcl_stream(L->ctx);
      DevMem* db[] = {&L->d_voff, &L->d_eoff, &L->d_rp, &L->d_col, &L->d_color, &L->d_roff,
                      &L->d_rows, &L->d_label, &L->d_status, &L->d_hash, &L->d_class, &L->d_seen};
      for (DevMem* b : db) b->stream = L->s;
      if (!L->large) rc = gcl_set_option(L->ctx, GCL_OPT_WORKSPACE_BYTES, c.lane_bytes);
      // a wide search takes one block per SM, leaving room on every SM for
      // the batches of the other lanes
      else if (L->cls == kLarge)
        rc = gcl_set_option(L->ctx, GCL_OPT_WIDE_MAX_WARPS, (int64_t)std::max(dev_sms, 1) * 4);
      // a big graph's search has at most a few hundred items (trees: about
      // one per first-path level), which 128 warps cover
      else rc = gcl_set_option(L->ctx, GCL_OPT_WIDE_MAX_WARPS, 128);
      if (rc == GCL_OK && L->large && c.big_wide)
        rc = gcl_set_option(L->ctx, GCL_OPT_WIDE_GATE, 2);
      // searches of big and large graphs run for long: their blocks keep
      // their per-step arrays in device memory so that they never fill an
      // SM's shared memory and lock the small lanes' kernels out
      if (rc == GCL_OK && (L->cls == kBig || L->large))
        rc = gcl_set_option(L->ctx, GCL_OPT_SMEM_STAGE, 0);
    }
  }
  // each lane's buffers for a full batch of its class (mean degree 8; the
  // large lanes for a pair of 8,192-vertex graphs)
  for (Lane* L : S->lanes) {
    if (rc != GCL_OK) break;
    int64_t g = 0, nmax = 0;
    switch (L->cls) {
      case kSmall: g = c.max_batch, nmax = 64; break;
      case kMid: g = c.mid_batch, nmax = 256; break;
      case kBig: g = S->max_batch[kBig], nmax = 2048; break;
      default: g = 2, nmax = 8192; break;
    }
    const int64_t v = g * nmax;
    rc = rc_of(lane_reserve(L, g, v, v * 8, v * ((nmax + 63) / 64)));
  }
  if (rc == GCL_OK) rc = rc_of(S->keys.ensure((size_t)c.table_slots * 8));
  if (rc == GCL_OK) rc = rc_of(S->vals.ensure((size_t)c.table_slots * 4));
  if (rc == GCL_OK) rc = rc_of(S->store.ensure((size_t)c.store_bytes));
  if (rc == GCL_OK) rc = rc_of(S->top.ensure(8));
  if (rc == GCL_OK) rc = rc_of(cudaMemset(S->keys.p, 0, (size_t)c.table_slots * 8));
  if (rc == GCL_OK) rc = rc_of(cudaMemset(S->vals.p, 0, (size_t)c.table_slots * 4));
  if (rc == GCL_OK) rc = rc_of(cudaMemset(S->top.p, 0, 8));
  if (rc == GCL_OK) rc = rc_of(cudaDeviceSynchronize());
  if (rc != GCL_OK) {
    teardown(S);
    return rc;
  }
  try {
    for (Lane* L : S->lanes) {
      L->cbarg = {S, L};
      L->worker = std::thread(lane_worker, S, L);
    }
    S->th = std::thread(dispatcher, S);
  } catch (...) {
    teardown(S);
    throw;
  }
  *out = S;
  return GCL_OK;
} GCL_CATCH_ALL

int gcl_serve_destroy(gcl_server* S) {
  if (!S) return GCL_ERR_ARG;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stop = true;
  }
  S->cv_work.notify_all();
  if (S->th.joinable()) S->th.join();
  for (auto& q : S->q)
    for (Req* r : q) delete r;
  teardown(S);
  return GCL_OK;
}

int gcl_serve_submit(gcl_server* S, int64_t id, int kind, const int32_t* rowptr,
                     const int32_t* col, const int32_t* color, int n, const int32_t* rowptr2,
                     const int32_t* col2, const int32_t* color2, int n2, uint64_t* out_rows,
                     int32_t* out_label) try {
  if (!S || (kind != GCL_REQ_CANON && kind != GCL_REQ_ISO)) return GCL_ERR_ARG;
  std::unique_ptr<Req> r(new (std::nothrow) Req());
  if (!r) return GCL_ERR_NOMEM;
  r->t0 = Clock::now();
  r->id = id;
  r->kind = kind;
  r->ng = kind == GCL_REQ_ISO ? 2 : 1;
  if (!copy_graph(r->g[0], rowptr, col, color, n) ||
      (r->ng == 2 && !copy_graph(r->g[1], rowptr2, col2, color2, n2)))
    return GCL_ERR_ARG;
  if (kind == GCL_REQ_CANON) {
    r->out_rows = out_rows;
    r->out_label = out_label;
  }
  // exact repeats: answer from the memo without a launch
  bool all_hit = S->cfg.memo_bytes > 0;
  MemoEntry e[2];
  for (int i = 0; i < r->ng; ++i) {
    r->key[i] = input_key(r->g[i]);
    if (all_hit) all_hit = memo_get(S, r->g[i], r->key[i], &e[i]);
  }
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->st.submitted += 1;
  }
  if (all_hit) {
    gcl_serve_result res;
    std::memset(&res, 0, sizeof res);
    res.id = id;
    res.status = GCL_OK;
    res.repeat = 2;
    res.class_id = e[0].cls;
    res.canon_hash = e[0].hash;
    res.verdict = -1;
    if (kind == GCL_REQ_CANON) {
      if (out_rows) std::memcpy(out_rows, e[0].rows.data(), e[0].rows.size() * 8);
      if (out_label) std::memcpy(out_label, e[0].label.data(), e[0].label.size() * 4);
    } else {
      res.verdict = e[0].in.n == e[1].in.n && e[0].rows == e[1].rows;
    }
    submit_done_now(S, r.get(), res);
    return GCL_OK;
  }
  const int nmax = std::max(r->g[0].n, r->ng == 2 ? r->g[1].n : 0);
  const int cls = nmax >= S->cfg.large_n ? kLarge
                  : nmax >= S->cfg.big_n ? kBig
                  : nmax >= S->cfg.mid_n ? kMid
                                         : kSmall;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->q[cls].push_back(r.get());
    r.release();  // owned by the queue
  }
  S->cv_work.notify_one();
  return GCL_OK;
} GCL_CATCH_ALL

int gcl_serve_poll(gcl_server* S, gcl_serve_result* out, int max, int timeout_ms) try {
  if (!S || !out || max < 0) return GCL_ERR_ARG;
  std::unique_lock<std::mutex> lk(S->mu);
  if (S->done.empty() && timeout_ms != 0) {
    auto pred = [&] { return !S->done.empty(); };
    if (timeout_ms < 0)
      S->cv_done.wait(lk, pred);
    else
      S->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), pred);
  }
  int k = 0;
  while (k < max && !S->done.empty()) {
    out[k++] = S->done.front();
    S->done.pop_front();
  }
  return k;
} GCL_CATCH_ALL

int gcl_serve_stats_get(gcl_server* S, gcl_serve_stats* out) try {
  if (!S || !out) return GCL_ERR_ARG;
  std::lock_guard<std::mutex> lk(S->mu);
  *out = S->st;
  return GCL_OK;
} GCL_CATCH_ALL

int gcl_serve_replay(gcl_server* S, int nreq, const double* arrival_s, const int32_t* kind,
                     const int32_t* g1, const int32_t* g2, int count, const int64_t* voff,
                     const int64_t* eoff, const int32_t* rowptr, const int32_t* col,
                     const int32_t* color, double timeout_s, gcl_serve_result* results) try {
  if (!S || nreq < 0 || !arrival_s || !kind || !g1 || !voff || !eoff || !rowptr || !results)
    return GCL_ERR_ARG;
  for (int i = 0; i < nreq; ++i) {
    if (g1[i] < 0 || g1[i] >= count) return GCL_ERR_ARG;
    if (kind[i] == GCL_REQ_ISO && (!g2 || g2[i] < 0 || g2[i] >= count)) return GCL_ERR_ARG;
    if (i > 0 && arrival_s[i] < arrival_s[i - 1]) return GCL_ERR_ARG;
  }
  std::vector<double> lag(nreq, 0.0);   // actual submit - scheduled arrival
  std::vector<char> got(nreq, 0);
  std::atomic<int> submit_rc{GCL_OK};
  const Clock::time_point start = Clock::now();
  auto graph_ptrs = [&](int g, const int32_t** rp, const int32_t** cl, const int32_t** co, int* n) {
    *n = (int)(voff[g + 1] - voff[g]);
    *rp = rowptr + voff[g] + g;
    *cl = col + eoff[g];
    *co = color ? color + voff[g] : nullptr;
  };
  std::vector<gcl_serve_result> buf(256);  // allocated before the thread starts
  std::thread gen([&] {
    for (int i = 0; i < nreq; ++i) {
      const Clock::time_point due =
          start + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double>(arrival_s[i]));
      Clock::time_point now = Clock::now();
      if (due - now > std::chrono::microseconds(300)) std::this_thread::sleep_until(due - std::chrono::microseconds(200));
      while (Clock::now() < due) {
      }
      const int32_t *rp1, *cl1, *co1, *rp2 = nullptr, *cl2 = nullptr, *co2 = nullptr;
      int n1, n2 = 0;
      graph_ptrs(g1[i], &rp1, &cl1, &co1, &n1);
      if (kind[i] == GCL_REQ_ISO) graph_ptrs(g2[i], &rp2, &cl2, &co2, &n2);
      lag[i] = std::chrono::duration<double>(Clock::now() - due).count();
      const int rc = gcl_serve_submit(S, i, kind[i], rp1, cl1, co1, n1, rp2, cl2, co2, n2,
                                      nullptr, nullptr);
      if (rc != GCL_OK) {
        submit_rc.store(rc);
        break;
      }
    }
  });
  int have = 0, rc = GCL_OK;
  while (have < nreq) {
    const int k = gcl_serve_poll(S, buf.data(), (int)buf.size(), 5);
    for (int j = 0; j < k; ++j) {
      const int64_t i = buf[j].id;
      if (i < 0 || i >= nreq || got[i]) continue;
      got[i] = 1;
      results[i] = buf[j];
      ++have;
    }
    if (submit_rc.load() != GCL_OK) {
      rc = submit_rc.load();
      break;
    }
    if (timeout_s > 0 && std::chrono::duration<double>(Clock::now() - start).count() > timeout_s) {
      rc = GCL_ERR_TIMEOUT;
      break;
    }
  }
  gen.join();
  if (rc == GCL_OK)
    for (int i = 0; i < nreq; ++i) {
      results[i].latency_s += lag[i];
      if (results[i].batch) {
        results[i].admit_s += lag[i];
        results[i].launch_s += lag[i];
        results[i].gpu_done_s += lag[i];
      }
    }
  return rc;
} GCL_CATCH_ALL

}  // extern "C"
