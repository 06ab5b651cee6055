// canon_wide.cuh -- many warps search the tree of one graph.
//
// The reference's GPU path (nauty_parallel.cu, BWDWorkList.cuh) spreads one
// graph's search tree over thread blocks that share the automorphism store
// and the best leaf.  This is the B200 form of that idea, built on the
// sparse warp machinery of canon_sparse.cuh:
//
//   1. one warp walks the first path (first_path_node, sequential.cpp:216-257)
//      to the first leaf and records, per level, the target cell's position
//      range, the path's codes and the leaf's partition;
//   2. the siblings of the first path -- every member of every level's target
//      cell except the first-path vertex -- become work items, deepest level
//      first.  A persistent grid of warps takes items from an atomic counter;
//      a warp rebuilds the item's parent node by backtracking a copy of the
//      first leaf's partition (cells never move vertices across their
//      boundaries, so reconstruct_at_level gives the node back), drops the
//      item if the vertex is not the least of its orbit under the stored
//      automorphisms that fix the path prefix, and otherwise runs the
//      reference's DFS (other_path_node / classify_node, sequential.cpp:304-624)
//      over the item's subtree;
//   3. automorphisms go to one device-wide append-only store, the best leaf
//      to one device-wide record guarded by a lock; each warp prunes against
//      its private copy of the best leaf, which is never better than the
//      shared one, and publishes under the lock when it finds a better leaf.
//
// The reference's leaf order is total -- the trail of codes, then a sentinel,
// then the upper-triangle matrix -- and every pruning rule discards only
// leaves that are worse than, or equivalent to, a leaf that some warp still
// covers, so the best leaf's matrix is the sequential one.  Two rules change
// to keep that true when subtrees finish out of order: a leaf equivalent to
// a best leaf found outside the current item only records the automorphism
// and steps back one level (the sequential jump to the common ancestor
// assumes that ancestor's other subtree is already complete), and a node
// found worse than a newly adopted best is pruned at once.  The stored
// automorphism count and node count are the wide search's own, like the
// reference GPU path's.
#pragma once
#include <cstdint>

#include "canon_sparse.cuh"

namespace gcl {

constexpr uint32_t kWideSpinLimit = 1u << 24;      // lock attempts (~1 s with back-off)
constexpr uint32_t kWideGateSpinLimit = 1u << 26;  // gate polls, up to 32 us apart

struct WideHdr {
  uint32_t D;          // level of the first leaf
  uint32_t nitems;     // work items (first-path siblings)
  uint32_t next_item;  // work counter
  uint32_t naut;       // automorphism slots claimed
  uint32_t lock;       // guards the best leaf
  uint32_t version;    // best-leaf version (0 = the first leaf)
  uint32_t best_level;
  uint32_t best_seqlen;
  int32_t status;
  uint32_t done;       // items finished (the gate of the next level)
  uint32_t orb_lock;   // guards the orbit cache
  int32_t orb_level;   // level index the orbit cache belongs to (-1 = none)
  uint32_t orb_known;  // store entries merged into the orbit cache
  uint32_t gate;       // the items kernel's level gate (1 on), set by the first kernel
  // work sharing (the sharing items kernel only)
  uint32_t busy;       // warps working on an item or a handed-over subtree
  uint32_t hungry;     // warps waiting for a handed-over subtree
  uint32_t qhead;      // handed-over subtrees taken
  uint32_t qtail;      // handed-over subtrees published (slots claimed)
  unsigned long long nodes;
  unsigned long long t0;  // start time (globaltimer ns)
  // how long a level's other items wait for its first item (the probe)
  // before they start anyway: twice the first path's duration
  unsigned long long probe_ns;
  // opt-in counters of the items kernel (GCL_OPT_COUNTERS; zeroed by the
  // host before a counted search, untouched otherwise)
  unsigned long long cnt[16];
};
// the header's region is 256 bytes: the counters move no other region
static_assert(sizeof(WideHdr) <= 256, "WideHdr outgrew its 256-byte region");

// Counters of the items kernel, summed over its warps (gcl_wide_counters):
// events, and clock64 cycles spent in each part of the work.
enum WideCounter : uint32_t {
  kCntItems,           // items searched (not pruned by an orbit)
  kCntItemsPruned,     // items skipped as equivalent to a smaller sibling
  kCntGiftsTaken,      // handed-over subtrees searched or pruned
  kCntGiftsGiven,      // subtrees handed over
  kCntNodes,           // search-tree nodes
  kCntLeaves,          // leaves reached (discrete partitions)
  kCntAutsFirst,       // automorphisms from a leaf equal to the first leaf
  kCntAutsBest,        // automorphisms from a leaf equal to the best leaf
  kCntBestPublished,   // leaves that became the shared best
  kCntPublishRetries,  // publish attempts that met a moved shared best
  kCntRefineCycles,    // individualize + refine
  kCntOrbitCycles,     // orbit tests of items and of target cells
  kCntGateCycles,      // waiting at the level gate
  kCntGiftWaitCycles,  // waiting for a handed-over subtree
  kCntLeafCycles,      // leaf certificates and their comparisons
  kCntWarpCycles,      // the warps' whole time in the kernel
  kWideCounters
};

template <bool kOn>
struct WideCnt {  // counting off: every call compiles to nothing
  __device__ __forceinline__ void add(uint32_t, unsigned long long) {}
  __device__ __forceinline__ unsigned long long now() const { return 0; }
  __device__ __forceinline__ void flush(WideHdr*) {}
};
template <>
struct WideCnt<true> {
  unsigned long long v[kWideCounters] = {};
  __device__ __forceinline__ void add(uint32_t i, unsigned long long x) { v[i] += x; }
  __device__ __forceinline__ unsigned long long now() const { return (unsigned long long)clock64(); }
  __device__ __forceinline__ void flush(WideHdr* H) {
    if (lane_id() == 0)
      for (uint32_t i = 0; i < kWideCounters; ++i)
        if (v[i]) atomicAdd(&H->cnt[i], v[i]);
  }
};

// Byte layout of the device-wide region of one wide search.
struct WideLayout {
  uint64_t hdr, fcode, fseq, flabel, fcert, lelem, linlev, lstb, tcfirst, tclen, cum;
  uint64_t bcode, bseq, blabel, bcert, auts, ready, fixlev, orb, gq, gready, bytes;
  uint32_t cap, stride;
  uint32_t qcap, gstride;  // handed-over subtrees: slots and words per slot (0 = none)
};

// words of one handed-over subtree: its level L, the child v, the parent's
// L-1 individualized vertices and its L codes (L <= n + 1)
__host__ __device__ inline uint32_t wide_gift_words(uint32_t n) {
  return ((2 * (n + 2) + 3) + 3) & ~3u;
}

__host__ __device__ inline WideLayout wide_layout(uint32_t n, uint64_t m2, uint32_t cap,
                                                  uint32_t qcap = 0) {
  WideLayout L{};
  uint64_t o = 0;
  auto take = [&](uint64_t bytes) {
    const uint64_t at = o;
    o = (o + bytes + 255u) & ~255ull;
    return at;
  };
  const uint64_t N1 = (uint64_t)n + 2;
  const uint64_t nw = (n + 63) / 64 + 1;
  L.stride = (uint32_t)N1;
  L.cap = cap;
  L.hdr = take(sizeof(WideHdr));
  L.fcode = take(4 * (N1 + 1));
  L.fseq = take(4 * N1);
  L.flabel = take(4 * N1);
  L.fcert = take(4 * (m2 + 1));
  L.lelem = take(4 * N1);
  L.linlev = take(4 * N1);
  L.lstb = take(8 * nw);
  L.tcfirst = take(4 * N1);
  L.tclen = take(4 * N1);
  L.cum = take(4 * (N1 + 1));
  L.bcode = take(4 * (N1 + 1));
  L.bseq = take(4 * N1);
  L.blabel = take(4 * N1);
  L.bcert = take(4 * (m2 + 1));
  L.auts = take(2ull * cap * N1);
  L.ready = take(4ull * cap);
  L.fixlev = take(4ull * cap);
  L.orb = take(4 * N1);
  L.qcap = qcap;
  L.gstride = qcap ? wide_gift_words(n) : 0;
  L.gq = take(4ull * qcap * L.gstride);
  L.gready = take(4ull * qcap);
  L.bytes = o;
  return L;
}

struct WideArgs {
  const int32_t* rp;
  const int32_t* col;
  const int32_t* color;
  uint32_t n;
  int64_t m;  // CSR entries
  uint8_t* sh;
  WideLayout WL;
  uint8_t* slots;  // per-warp workspace
  SpLayout Lo;
  uint64_t slot_bytes;
  uint32_t pool;
  uint32_t gate;  // level gate: 1 on (a level's items wait for the deeper ones), 0 off, 2 auto
  uint32_t probe;  // under the gate: a level's first item runs before the rest of the level
  uint64_t smem_per_warp;
  uint64_t budget_ns;
  uint8_t* out_dense;    // n*n, or null
  uint64_t* out_rows;    // n * ceil(n/64) words, or null
  int32_t* out_label;    // n, or null
  int64_t* out_stats;    // {num_aut, nodes}, or null
  int32_t* out_status;   // 1
};

struct WidePtrs {
  WideHdr* H;
  int32_t *fcode, *bcode;
  uint32_t *fseq, *flabel, *fcert, *lelem, *linlev, *tcfirst, *tclen, *cum;
  uint32_t *bseq, *blabel, *bcert, *ready, *fixlev, *orb, *gq, *gready;
  uint64_t* lstb;
  uint16_t* auts;
};

__device__ inline WidePtrs wide_ptrs(const WideArgs& A) {
  uint8_t* b = A.sh;
  const WideLayout& L = A.WL;
  WidePtrs P;
  P.H = (WideHdr*)(b + L.hdr);
  P.fcode = (int32_t*)(b + L.fcode);
  P.bcode = (int32_t*)(b + L.bcode);
  P.fseq = (uint32_t*)(b + L.fseq);
  P.flabel = (uint32_t*)(b + L.flabel);
  P.fcert = (uint32_t*)(b + L.fcert);
  P.lelem = (uint32_t*)(b + L.lelem);
  P.linlev = (uint32_t*)(b + L.linlev);
  P.tcfirst = (uint32_t*)(b + L.tcfirst);
  P.tclen = (uint32_t*)(b + L.tclen);
  P.cum = (uint32_t*)(b + L.cum);
  P.bseq = (uint32_t*)(b + L.bseq);
  P.blabel = (uint32_t*)(b + L.blabel);
  P.bcert = (uint32_t*)(b + L.bcert);
  P.ready = (uint32_t*)(b + L.ready);
  P.fixlev = (uint32_t*)(b + L.fixlev);
  P.orb = (uint32_t*)(b + L.orb);
  P.gq = (uint32_t*)(b + L.gq);
  P.gready = (uint32_t*)(b + L.gready);
  P.lstb = (uint64_t*)(b + L.lstb);
  P.auts = (uint16_t*)(b + L.auts);
  return P;
}

__device__ __forceinline__ void wide_fail(WideHdr* H, int32_t status) {
  if (lane_id() == 0) atomicCAS((int*)&H->status, (int)kOk, (int)status);
}

// ---------------------------------------------------------------------------
// 1. First path (one warp).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(32) wide_first_kernel(WideArgs A) {
  const uint32_t lane = lane_id();
  const WidePtrs P = wide_ptrs(A);
  WideHdr* H = P.H;
  SpWarp& W = sp_w();
  const uint32_t n = A.n;
  if (lane == 0) {
    H->D = 0;
    H->nitems = 0;
    H->next_item = 0;
    H->naut = 0;
    H->lock = 0;
    H->version = 0;
    H->best_level = 0;
    H->best_seqlen = 0;
    H->status = kOk;
    H->done = 0;
    H->orb_lock = 0;
    H->orb_level = -1;
    H->orb_known = 0;
    H->busy = 0;
    H->hungry = 0;
    H->qhead = 0;
    H->qtail = 0;
    H->nodes = 1;
    H->t0 = global_ns();
  }
  sp_bind(A.slots, A.Lo, n, A.rp, A.col, nullptr, 0, A.pool, 0, 1);
  __syncwarp();
  if (!sp_check_input(A.m)) {
    wide_fail(H, kBadInput);
    return;
  }
  sp_init_partition(A.color);
  int code = sp_refine(0);
  if (code < 0) {
    wide_fail(H, kInternal);
    return;
  }
  uint32_t level = 1, seqlen = 0;
  unsigned long long nodes = 1;
  if (lane == 0) P.fcode[0] = code;
  __syncwarp();
  while (W.ncells < n) {
    const uint32_t t = level <= n ? sp_first_nonsingleton() : kNone;
    if (t == kNone) {
      wide_fail(H, kInternal);
      return;
    }
    const uint32_t len = sp_cell_end(W, t) - t;
    uint32_t v = kNone;
    for (uint32_t q = t + lane; q < t + len; q += 32) v = min(v, W.elem[q]);
    v = __reduce_min_sync(GCL_FULL, v);  // first representative: the least member
    __syncwarp();
    if (lane == 0) {
      P.tcfirst[level - 1] = t;
      P.tclen[level - 1] = len;
      W.seq[seqlen] = v;
    }
    __syncwarp();
    ++seqlen;
    ++nodes;
    if (!sp_individualize(level, v, t)) {
      wide_fail(H, kInternal);
      return;
    }
    code = sp_refine(level);
    if (code < 0) {
      wide_fail(H, kInternal);
      return;
    }
    ++level;
    __syncwarp();
    if (lane == 0) P.fcode[level - 1] = code;
    __syncwarp();
  }
  // the first leaf: certificate, labeling, partition, and the initial best
  const uint32_t D = level;
  sp_leaf_cert(P.fcert);
  for (uint32_t i = lane; i < n; i += 32) {
    const uint32_t e = W.elem[i];
    P.flabel[i] = e;
    P.blabel[i] = e;
    P.lelem[i] = e;
    P.linlev[i] = W.inlev[i];
  }
  for (uint32_t i = lane; i < seqlen; i += 32) {
    P.fseq[i] = W.seq[i];
    P.bseq[i] = W.seq[i];
  }
  for (uint32_t w = lane; w < W.nw; w += 32) P.lstb[w] = W.stb[w];
  for (int64_t i = lane; i < A.m; i += 32) P.bcert[i] = P.fcert[i];
  for (uint32_t i = lane; i < D; i += 32) P.bcode[i] = P.fcode[i];
  __syncwarp();
  if (lane == 0) {
    P.fcode[D] = kSentinel;
    P.bcode[D] = kSentinel;
    // items of node level L = D-1 .. 1: its target cell minus the first-path
    // vertex, which the first path left at the cell's first position
    uint32_t run = 0;
    P.cum[0] = 0;
    for (uint32_t i = 0; i + 1 < D; ++i) {
      const uint32_t L = D - 1 - i;
      run += P.tclen[L - 1] - 1;
      P.cum[i + 1] = run;
    }
    H->D = D;
    H->best_level = D;
    H->best_seqlen = seqlen;
    H->nodes = nodes;
    // automatic gate: off when the levels hold fewer than 4 items each on
    // average (trees), where it would run the items one after another
    H->gate = A.gate == 2 ? (run >= 4u * (D - 1u) ? 1u : 0u) : (A.gate != 0 ? 1u : 0u);
    H->probe_ns = max(2ull * (global_ns() - H->t0), 20000ull);
    __threadfence();
    H->nitems = run;
  }
}

// ---------------------------------------------------------------------------
// 2. Items (persistent grid, one item per warp at a time).
// ---------------------------------------------------------------------------

// Number of leading automorphism-store entries whose contents are complete.
__device__ __noinline__ uint32_t wide_ready_prefix(const WidePtrs& P, uint32_t known,
                                                   uint32_t cap) {
  uint32_t k = known;
  if (lane_id() == 0) {
    const uint32_t claimed = min(*(volatile uint32_t*)&P.H->naut, cap);
    while (k < claimed && *(volatile uint32_t*)&P.ready[k]) ++k;
    __threadfence();
  }
  return __shfl_sync(GCL_FULL, k, 0);
}

__device__ __noinline__ bool wide_lock(uint32_t* lk) {
  uint32_t got = 0;
  if (lane_id() == 0) {
    for (uint32_t i = 0; i < kWideSpinLimit; ++i) {
      if (atomicCAS(lk, 0u, 1u) == 0u) {
        got = 1;
        break;
      }
      __nanosleep(64);
    }
    __threadfence();
  }
  return __shfl_sync(GCL_FULL, got, 0) != 0;
}

__device__ __noinline__ void wide_unlock(uint32_t* lk) {
  __threadfence();
  __syncwarp();
  if (lane_id() == 0) atomicExch(lk, 0u);
  __syncwarp();
}

__device__ __forceinline__ uint32_t wide_find(const uint32_t* d, uint32_t x, uint32_t n) {
  uint32_t p = __ldcg(d + x);
  for (uint32_t step = 0; p < x && step <= n; ++step) {
    x = p;
    p = __ldcg(d + x);
  }
  return x;
}

// Least vertex of v's orbit under the stored automorphisms that fix the
// first path's first k vertices (subgroup_fixing_sequence +
// compute_orbits_fast, perm_group.cpp:5-116), uniting over the members of
// the level's target cell only (positions [tf, tf+tl) of the first leaf;
// such automorphisms map the cell onto itself).  Only one level's items run at
// a time, so one device-wide union-find serves them all: the first warp of a
// level resets it, every warp merges the store entries that arrived since
// the last merge, under the cache lock.  A root below v without the lock is
// already a proof that v is not the least of its orbit (roots only move
// down).  Sets *ok = false when a wait or a merge gives up.
__device__ __noinline__ uint32_t wide_orbit_min(const WidePtrs& P, uint32_t v, uint32_t li,
                                                uint32_t k, uint32_t tf, uint32_t tl,
                                                uint32_t known, uint32_t stride, bool* ok) {
  SpWarp& W = sp_w();
  const uint32_t lane = lane_id();
  const uint32_t n = W.n;
  WideHdr* H = P.H;
  uint32_t r = kNone;
  if (lane == 0 && *(volatile int32_t*)&H->orb_level == (int32_t)li) {
    const uint32_t merged = *(volatile uint32_t*)&H->orb_known;
    __threadfence();
    const uint32_t x = wide_find(P.orb, v, n);
    if (x < v || merged >= known) r = x;
  }
  r = __shfl_sync(GCL_FULL, r, 0);
  if (r != kNone) return r;
  if (!wide_lock(&H->orb_lock)) {
    *ok = false;
    return v;
  }
  if (*(volatile int32_t*)&H->orb_level != (int32_t)li) {
    for (uint32_t x = lane; x < n; x += 32) P.orb[x] = x;
    __threadfence();
    __syncwarp();
    if (lane == 0) {
      H->orb_known = 0;
      __threadfence();
      *(volatile int32_t*)&H->orb_level = (int32_t)li;
    }
    __syncwarp();
  }
  uint32_t from = *(volatile uint32_t*)&H->orb_known;
  uint32_t* own = W.dsu;
  __syncwarp();
  if (lane == 0) W.dsu = P.orb;
  __syncwarp();
  for (uint32_t a = from; a < known; ++a) {
    if (__ldcg(P.fixlev + a) < k) continue;
    if (!sp_dsu_apply<true>(P.auts + (uint64_t)a * stride, P.lelem + tf, tl, n)) {
      *ok = false;
      break;
    }
  }
  __syncwarp();
  if (lane == 0) W.dsu = own;
  __threadfence();
  __syncwarp();
  if (lane == 0) {
    if (*ok && known > from) H->orb_known = known;
    r = wide_find(P.orb, v, n);
  }
  r = __shfl_sync(GCL_FULL, r, 0);
  wide_unlock(&H->orb_lock);
  return r;
}

// wide_orbit_min for items that do not wait for the deeper levels: items of
// several levels run at once, so the warp unites in its own union-find
// (W.dsu, free between items) instead of the shared one, and stops as soon
// as v has a smaller root.
__device__ __noinline__ uint32_t wide_orbit_min_own(const WidePtrs& P, uint32_t v, uint32_t k,
                                                    uint32_t tf, uint32_t tl, uint32_t known,
                                                    uint32_t stride, bool* ok) {
  SpWarp& W = sp_w();
  const uint32_t lane = lane_id();
  const uint32_t n = W.n;
  const uint32_t* mem = P.lelem + tf;
  for (uint32_t x = lane; x < n; x += 32) W.dsu[x] = x;
  __syncwarp();
  uint32_t r = v;
  for (uint32_t a = 0; a < known && r == v; ++a) {
    if (__ldcg(P.fixlev + a) < k) continue;
    if (!sp_dsu_apply<true>(P.auts + (uint64_t)a * stride, mem, tl, n)) {
      *ok = false;
      break;
    }
    uint32_t x = v;
    if (lane == 0) x = sp_find(W.dsu, v, n);
    r = __shfl_sync(GCL_FULL, x, 0);
  }
  return r;
}

// Append aut[label[j]] = elem[j] to the store with its fixed-prefix length.
template <bool kCgLabel>
__device__ __noinline__ void wide_store_aut(const WidePtrs& P, const uint32_t* label, uint32_t cap,
                                            uint32_t stride, uint32_t D) {
  SpWarp& W = sp_w();
  const uint32_t lane = lane_id();
  uint32_t slot = 0;
  if (lane == 0) slot = atomicAdd(&P.H->naut, 1u);
  slot = __shfl_sync(GCL_FULL, slot, 0);
  if (slot >= cap) return;  // store full: fewer prunes, same result
  uint16_t* pm = P.auts + (uint64_t)slot * stride;
  for (uint32_t j = lane; j < W.n; j += 32) pm[ldx<kCgLabel>(label + j)] = (uint16_t)W.elem[j];
  __syncwarp();
  // leading first-path vertices it fixes
  const uint32_t np = D - 1;
  uint32_t fl = np;
  for (uint32_t i0 = 0; i0 < np; i0 += 32) {
    const uint32_t i = i0 + lane;
    const uint32_t b = __ballot_sync(GCL_FULL, i < np && pm[P.fseq[i]] != P.fseq[i]);
    if (b) {
      fl = i0 + (uint32_t)(__ffs(b) - 1);
      break;
    }
  }
  __threadfence();
  __syncwarp();
  if (lane == 0) {
    P.fixlev[slot] = fl;
    __threadfence();
    *(volatile uint32_t*)&P.ready[slot] = 1u;
  }
  __syncwarp();
}

struct WideBest {
  int canon_level;
  uint32_t best_seqlen;
  uint32_t version;  // even; 0 = the first leaf
};

// Copy the shared best leaf into the warp's private copy.  The shared record
// is a sequence lock: its version is odd while a writer (holding the best
// lock) rewrites it, so a copy taken between two equal even versions is
// whole.  After repeated collisions the copy is taken under the lock.
__device__ __noinline__ bool wide_adopt(const WidePtrs& P, int64_t m, WideBest* out) {
  SpWarp& W = sp_w();
  const uint32_t lane = lane_id();
  WideHdr* H = P.H;
  for (int attempt = 0; attempt < 66; ++attempt) {
    const bool locked = attempt == 65;
    if (locked && !wide_lock(&H->lock)) return false;
    uint32_t v1 = 0, lvl = 0, sl = 0;
    if (lane == 0) {
      v1 = *(volatile uint32_t*)&H->version;
      __threadfence();
      lvl = *(volatile uint32_t*)&H->best_level;
      sl = *(volatile uint32_t*)&H->best_seqlen;
      __threadfence();
    }
    v1 = __shfl_sync(GCL_FULL, v1, 0);
    lvl = __shfl_sync(GCL_FULL, lvl, 0);
    sl = __shfl_sync(GCL_FULL, sl, 0);
    if ((v1 & 1u) && !locked) {
      if (lane == 0) __nanosleep(256);
      __syncwarp();
      continue;
    }
    for (uint32_t i = lane; i <= lvl; i += 32) W.ccode[i] = __ldcg(P.bcode + i);
    for (uint32_t i = lane; i < W.n; i += 32) W.blabel[i] = __ldcg(P.blabel + i);
    for (uint32_t i = lane; i < sl; i += 32) W.bseq[i] = __ldcg(P.bseq + i);
    for (int64_t i = lane; i < m; i += 32) W.bcert[i] = __ldcg(P.bcert + i);
    __threadfence();
    __syncwarp();
    uint32_t v2 = 0;
    if (lane == 0) v2 = *(volatile uint32_t*)&H->version;
    v2 = __shfl_sync(GCL_FULL, v2, 0);
    if (locked) wide_unlock(&H->lock);
    if (v1 == v2 || locked) {
      out->canon_level = (int)lvl;
      out->best_seqlen = sl;
      out->version = v1;
      return true;
    }
  }
  return false;
}

// The path's comparison state against the private best: the first level
// whose code differs (eqlevcanon) and the sign there (comp_canon); a better
// path overwrites the private trail from there on, as classify_node does.
__device__ __noinline__ void wide_recompare(uint32_t Lp, int canon_level, int* eqlevcanon,
                                            int* comp_canon) {
  SpWarp& W = sp_w();
  const uint32_t lane = lane_id();
  const uint32_t lim = min(Lp, (uint32_t)canon_level);
  uint32_t i = lim;
  for (uint32_t j0 = 0; j0 < lim; j0 += 32) {
    const uint32_t j = j0 + lane;
    const uint32_t b = __ballot_sync(GCL_FULL, j < lim && W.pathcode[j] != W.ccode[j]);
    if (b) {
      i = j0 + (uint32_t)(__ffs(b) - 1);
      break;
    }
  }
  if (i == Lp) {
    *eqlevcanon = (int)Lp;
    *comp_canon = 0;
    return;
  }
  *eqlevcanon = (int)i;
  const int bc = (int)i < canon_level ? W.ccode[i] : kSentinel;
  *comp_canon = W.pathcode[i] < bc ? -1 : 1;
  if (*comp_canon > 0) {
    __syncwarp();
    for (uint32_t j = i + lane; j < Lp; j += 32) W.ccode[j] = W.pathcode[j];
  }
  __syncwarp();
}

// The current leaf (level Lv) against the private best: trail of codes, then
// the level (a shorter trail ends in the sentinel and wins), then the upper
// triangle.
__device__ __noinline__ int wide_cmp_private(uint32_t Lv, int canon_level) {
  SpWarp& W = sp_w();
  const uint32_t lane = lane_id();
  const uint32_t lim = min(Lv, (uint32_t)canon_level);
  for (uint32_t j0 = 0; j0 < lim; j0 += 32) {
    const uint32_t j = j0 + lane;
    const int32_t pc = j < lim ? W.pathcode[j] : 0, bc = j < lim ? W.ccode[j] : 0;
    const uint32_t b = __ballot_sync(GCL_FULL, j < lim && pc != bc);
    if (b) {
      const int src = __ffs(b) - 1;
      const int32_t x = __shfl_sync(GCL_FULL, pc, src), y = __shfl_sync(GCL_FULL, bc, src);
      return x < y ? -1 : 1;
    }
  }
  if ((int)Lv < canon_level) return 1;
  if ((int)Lv > canon_level) return -1;
  return sp_cmp_leaf(W.ccert, W.blabel, W.bcert, true);
}

// Make the current leaf, which beats the private best of version
// `best.version`, the shared best.  Returns 1 when it was written, 0 when
// the shared best had moved on (it is then adopted: the caller compares the
// leaf again), -1 when the lock could not be taken.
__device__ __noinline__ int wide_try_publish(const WidePtrs& P, const WideArgs& A, uint32_t Lv,
                                             uint32_t seqlen, WideBest* best) {
  SpWarp& W = sp_w();
  const uint32_t lane = lane_id();
  WideHdr* H = P.H;
  if (!wide_lock(&H->lock)) return -1;
  uint32_t cur = 0;
  if (lane == 0) cur = *(volatile uint32_t*)&H->version;
  cur = __shfl_sync(GCL_FULL, cur, 0);
  if (cur != best->version) {
    wide_unlock(&H->lock);
    return wide_adopt(P, A.m, best) ? 0 : -1;
  }
  if (lane == 0) {
    *(volatile uint32_t*)&H->version = cur + 1;  // odd: being rewritten
    __threadfence();
  }
  __syncwarp();
  for (uint32_t i = lane; i < Lv; i += 32) P.bcode[i] = W.pathcode[i];
  for (uint32_t i = lane; i < W.n; i += 32) P.blabel[i] = W.elem[i];
  for (uint32_t i = lane; i < seqlen; i += 32) P.bseq[i] = W.seq[i];
  for (int64_t i = lane; i < A.m; i += 32) P.bcert[i] = W.ccert[i];
  __threadfence();
  __syncwarp();
  if (lane == 0) {
    P.bcode[Lv] = kSentinel;
    H->best_level = Lv;
    H->best_seqlen = seqlen;
    __threadfence();
    *(volatile uint32_t*)&H->version = cur + 2;
  }
  wide_unlock(&H->lock);
  best->version = cur + 2;
  best->canon_level = (int)Lv;
  best->best_seqlen = seqlen;
  return 1;
}

// Wait until `need` items have finished: a level's items start once every
// item of the deeper levels is done, so their automorphisms prune the level
// as they do in the sequential order.  The items being waited for are held
// by running warps of the same grid; the wait ends with the time budget or a
// recorded error at the latest.
__device__ __noinline__ int32_t wide_gate(WideHdr* H, uint32_t need, uint64_t deadline) {
  int32_t st = kOk;
  if (lane_id() == 0) {
    // back off from 0.5 us to 32 us between polls: many warps may wait on
    // the same counter, and a level lasts far longer than the poll period
    uint32_t sleep_ns = 512;
    for (uint32_t i = 0;; ++i) {
      if (*(volatile uint32_t*)&H->done >= need) break;
      const int32_t hs = *(volatile int32_t*)&H->status;
      if (hs != kOk) {
        st = hs;
        break;
      }
      if (i >= kWideGateSpinLimit || (deadline && (i & 15u) == 0 && global_ns() > deadline)) {
        st = kTimeout;
        break;
      }
      __nanosleep(sleep_ns);
      if (sleep_ns < 32768) sleep_ns <<= 1;
    }
    __threadfence();
  }
  return __shfl_sync(GCL_FULL, st, 0);
}

// The probe's wait: like wide_gate, but past `soft` (globaltimer ns) the
// warp stops waiting and starts its item anyway (kOk): a first item whose
// subtree is large would otherwise hold its whole level back.
__device__ __noinline__ int32_t wide_gate_soft(WideHdr* H, uint32_t need, uint64_t soft,
                                               uint64_t deadline) {
  int32_t st = kOk;
  if (lane_id() == 0) {
    uint32_t sleep_ns = 256;
    for (uint32_t i = 0; i < kWideGateSpinLimit; ++i) {
      if (*(volatile uint32_t*)&H->done >= need) break;
      const int32_t hs = *(volatile int32_t*)&H->status;
      if (hs != kOk) {
        st = hs;
        break;
      }
      const uint64_t now = global_ns();
      if (now > soft) break;
      if (deadline && now > deadline) {
        st = kTimeout;
        break;
      }
      __nanosleep(sleep_ns);
      if (sleep_ns < 8192) sleep_ns <<= 1;
    }
    __threadfence();
  }
  return __shfl_sync(GCL_FULL, st, 0);
}

// Store entries [from, to) become known to this warp: nothing is known yet
// about how they act on its sequence.
__device__ __noinline__ void wide_fix_init(uint32_t from, uint32_t to) {
  SpWarp& W = sp_w();
  to = min(to, W.fixcap);
  for (uint32_t a = from + lane_id(); a < to; a += 32) W.fixst[a] = make_uint2(0u, kNone);
  __syncwarp();
}

// ---------------------------------------------------------------------------
// Work sharing inside items (the sharing items kernel).  A busy warp hands an
// idle one the next untried child at the shallowest level of its item where
// a child's subtree has already finished -- so the automorphisms that subtree
// found prune the siblings before they leave -- and treats it as tried.  A
// handed-over subtree is an entry of a device queue (its level L, the child,
// the parent's vertices and codes); the receiver rebuilds the parent from the
// first leaf and searches the child's subtree as it would an item's.  The
// queue is never reused within a search (slots are taken in order and not
// recycled), so a slot is written once and read once.
// ---------------------------------------------------------------------------
constexpr uint32_t kGiftMaxWords = 1u << 26;  // 256 MiB of queue at most

// Offer the next untried child of a level in [k+2, level) when warps are
// waiting for work and the queue holds fewer entries than them; true when
// a subtree was handed over.
__device__ __noinline__ bool wide_try_donate(const WidePtrs& P, const WideArgs& A, uint32_t k,
                                             uint32_t level, int tcl) {
  SpWarp& W = sp_w();
  const uint32_t lane = lane_id();
  WideHdr* H = P.H;
  const uint32_t n = W.n;
  uint32_t want = 0;
  if (lane == 0) {
    const uint32_t hungry = *(volatile uint32_t*)&H->hungry;
    const uint32_t head = *(volatile uint32_t*)&H->qhead;
    const uint32_t tail = *(volatile uint32_t*)&H->qtail;
    want = hungry > tail - head && tail < A.WL.qcap;
  }
  if (!__shfl_sync(GCL_FULL, want, 0)) return false;
  for (uint32_t Lp = k + 2; Lp < level && (int)Lp <= tcl; ++Lp) {
    const SpTc t = W.tc[Lp - 1];
    if (t.counter >= n) continue;
    // the child tried first is the cell's least vertex: while it is still the
    // path's child at this level, its subtree has not finished
    uint32_t least = kNone;
    for (uint32_t q = lane; q < t.len; q += 32) least = min(least, W.elem[t.first + q]);
    least = __reduce_min_sync(GCL_FULL, least);
    if (W.seq[Lp - 1] == least) continue;
    const uint32_t u = sp_next_rep(t);
    if (u == kNone) continue;
    uint32_t slot = kNone;
    if (lane == 0) {
      for (int tries = 0; tries < 64; ++tries) {
        const uint32_t tl = *(volatile uint32_t*)&H->qtail;
        if (tl >= A.WL.qcap) break;
        if (atomicCAS(&H->qtail, tl, tl + 1) == tl) {
          slot = tl;
          break;
        }
      }
    }
    slot = __shfl_sync(GCL_FULL, slot, 0);
    if (slot == kNone) return false;
    uint32_t* e = P.gq + (uint64_t)slot * A.WL.gstride;
    const uint32_t np = A.n + 2;
    if (lane == 0) {
      e[0] = Lp;
      e[1] = u;
    }
    for (uint32_t i = lane; i + 1 < Lp; i += 32) e[2 + i] = W.seq[i];
    for (uint32_t i = lane; i < Lp; i += 32) e[2 + np + i] = (uint32_t)W.pathcode[i];
    __threadfence();
    __syncwarp();
    if (lane == 0) {
      W.tc[Lp - 1].counter = u + 1;  // tried: the receiver searches it
      *(volatile uint32_t*)&P.gready[slot] = 1u;
    }
    __syncwarp();
    return true;
  }
  return false;
}

// Wait for a handed-over subtree.  1: its slot in *slot (the warp now counts
// as busy); 0: the search is over (no warp busy and the queue empty); else a
// status.  The busy count is read before the queue, so a subtree published by
// a warp that then finished is seen.
__device__ __noinline__ int32_t wide_take_gift(const WidePtrs& P, uint64_t deadline,
                                               uint32_t* slot) {
  WideHdr* H = P.H;
  int32_t st = 0;
  uint32_t got = kNone;
  if (lane_id() == 0) {
    atomicAdd(&H->hungry, 1u);
    uint32_t sleep_ns = 512;
    for (uint32_t i = 0;; ++i) {
      const int32_t hs = *(volatile int32_t*)&H->status;
      if (hs != kOk) {
        st = hs;
        break;
      }
      const uint32_t busy = *(volatile uint32_t*)&H->busy;
      __threadfence();
      const uint32_t head = *(volatile uint32_t*)&H->qhead;
      const uint32_t tail = *(volatile uint32_t*)&H->qtail;
      if (head < tail) {
        if (atomicCAS(&H->qhead, head, head + 1) == head) {
          got = head;
          break;
        }
        continue;
      }
      if (busy == 0) break;  // st = 0: nothing left anywhere
      if (i >= kWideGateSpinLimit || (deadline && (i & 15u) == 0 && global_ns() > deadline)) {
        st = kTimeout;
        break;
      }
      __nanosleep(sleep_ns);
      if (sleep_ns < 32768) sleep_ns <<= 1;
    }
    if (got != kNone) {
      atomicAdd(&H->busy, 1u);
      // the publisher fills the slot after claiming it
      uint32_t j = 0;
      while (!*(volatile uint32_t*)&P.gready[got] && j < kWideSpinLimit) {
        __nanosleep(64);
        ++j;
      }
      if (j >= kWideSpinLimit) st = kTimeout;
      else st = 1;
      __threadfence();
    }
    atomicSub(&H->hungry, 1u);
  }
  st = __shfl_sync(GCL_FULL, st, 0);
  *slot = __shfl_sync(GCL_FULL, got, 0);
  return st;
}

// Rebuild the parent node of a handed-over subtree: the first leaf taken back
// to the level its sequence shares with the first path, the rest of its
// vertices individualized and refined (each code checked against the one the
// giver saw).  Leaves W at the parent (level L = *k + 1) with W.seq, W.pathcode
// and the target-cell headers of the replayed levels; *tf, *tl: the parent's
// target cell; *v: the child; *eqlev: leading codes equal to the first path's.
__device__ __noinline__ int32_t wide_gift_node(const WidePtrs& P, const WideArgs& A, uint32_t slot,
                                               uint32_t D, uint32_t* k, uint32_t* tf,
                                               uint32_t* tl, uint32_t* v, uint32_t* eqlev) {
  SpWarp& W = sp_w();
  const uint32_t lane = lane_id();
  const uint32_t n = W.n, np = n + 2;
  const uint32_t* e = P.gq + (uint64_t)slot * A.WL.gstride;
  const uint32_t L = __ldcg(e), vv = __ldcg(e + 1);
  if (L < 2 || L > n || vv >= n) return kInternal;
  // levels shared with the first path: its first c vertices
  const uint32_t lim = min(L - 1, D - 1);
  uint32_t c = lim;
  for (uint32_t j0 = 0; j0 < lim; j0 += 32) {
    const uint32_t j = j0 + lane;
    const uint32_t b = __ballot_sync(GCL_FULL, j < lim && __ldcg(e + 2 + j) != P.fseq[j]);
    if (b) {
      c = j0 + (uint32_t)(__ffs(b) - 1);
      break;
    }
  }
  for (uint32_t i = lane; i < n; i += 32) {
    const uint32_t x = P.lelem[i];
    W.elem[i] = x;
    W.pos[x] = i;
    W.inlev[i] = P.linlev[i];
  }
  for (uint32_t w = lane; w < W.nw; w += 32) W.stb[w] = P.lstb[w];
  __syncwarp();
  bm_resummarize(W.stb, W.sts, W.nw, W.nsw);
  if (lane == 0) W.ncells = n;
  __syncwarp();
  if (!sp_backtrack(c + 1)) return kInternal;
  for (uint32_t i = lane; i < c; i += 32) W.seq[i] = P.fseq[i];
  for (uint32_t i = lane; i <= c; i += 32) W.pathcode[i] = P.fcode[i];
  __syncwarp();
  for (uint32_t lvl = c + 1; lvl < L; ++lvl) {
    const uint32_t t = sp_first_nonsingleton();
    if (t == kNone) return kInternal;
    const uint32_t len = sp_cell_end(W, t) - t;
    const uint32_t u = __ldcg(e + 2 + (lvl - 1));
    if (u >= n || W.pos[u] < t || W.pos[u] >= t + len) return kInternal;
    __syncwarp();
    if (lane == 0) {
      SpTc h;
      h.first = t;
      h.len = len;
      h.counter = n;
      h.last = 0;
      h.rslot = -1;
      h.pad = 0;
      W.tc[lvl - 1] = h;
      W.seq[lvl - 1] = u;
    }
    __syncwarp();
    if (!sp_individualize(lvl, u, t)) return kInternal;
    const int code = sp_refine(lvl);
    if (code < 0 || (uint32_t)code != __ldcg(e + 2 + np + lvl)) return kInternal;
    __syncwarp();
    if (lane == 0) W.pathcode[lvl] = code;
    __syncwarp();
  }
  const uint32_t t = sp_first_nonsingleton();
  if (t == kNone) return kInternal;
  const uint32_t len = sp_cell_end(W, t) - t;
  if (W.pos[vv] < t || W.pos[vv] >= t + len) return kInternal;
  uint32_t q = min(L, D);
  for (uint32_t j0 = 0; j0 < min(L, D); j0 += 32) {
    const uint32_t j = j0 + lane;
    const uint32_t b = __ballot_sync(GCL_FULL, j < min(L, D) && W.pathcode[j] != W.fcode[j]);
    if (b) {
      q = j0 + (uint32_t)(__ffs(b) - 1);
      break;
    }
  }
  *k = L - 1;
  *tf = t;
  *tl = len;
  *v = vv;
  *eqlev = q;
  return kOk;
}

// Least vertex of v's orbit in the parent's target cell [tf, tf+tl) under the
// known automorphisms that fix the parent's k vertices W.seq[0..k), in the
// warp's own union-find; stops at the first smaller root.
__device__ __noinline__ uint32_t wide_gift_orbit_min(const WidePtrs& P, uint32_t v, uint32_t k,
                                                     uint32_t tf, uint32_t tl, uint32_t known,
                                                     uint32_t stride, bool* ok) {
  SpWarp& W = sp_w();
  const uint32_t lane = lane_id();
  const uint32_t n = W.n;
  for (uint32_t x = lane; x < n; x += 32) W.dsu[x] = x;
  __syncwarp();
  uint32_t r = v;
  for (uint32_t a = 0; a < known && r == v; ++a) {
    const uint16_t* pm = P.auts + (uint64_t)a * stride;
    bool moves = false;
    for (uint32_t i = lane; i < k; i += 32) moves |= __ldcg(pm + W.seq[i]) != W.seq[i];
    if (__any_sync(GCL_FULL, moves)) continue;
    if (!sp_dsu_apply<true>(pm, W.elem + tf, tl, n)) {
      *ok = false;
      break;
    }
    uint32_t x = v;
    if (lane == 0) x = sp_find(W.dsu, v, n);
    r = __shfl_sync(GCL_FULL, x, 0);
  }
  return r;
}

template <bool kShare, bool kCount>
__global__ void __launch_bounds__(kSpThreads) wide_items_kernel(WideArgs A) {
  extern __shared__ __align__(16) uint8_t sp_dyn[];
  const int warp = (int)(threadIdx.x >> 5);
  const uint32_t lane = lane_id();
  const WidePtrs P = wide_ptrs(A);
  WideHdr* H = P.H;
  if (H->status != kOk || H->nitems == 0) return;
  WideCnt<kCount> cnt;
  const unsigned long long t_start = cnt.now();
  SpWarp& W = sp_w();
  const uint32_t n = A.n, D = H->D, nitems = H->nitems, cap = A.WL.cap;
  uint8_t* slot = A.slots + ((uint64_t)blockIdx.x * kSpWarps + (uint64_t)warp) * A.slot_bytes;
  uint8_t* smem = A.smem_per_warp ? sp_dyn + (uint64_t)warp * A.smem_per_warp : nullptr;
  sp_bind(slot, A.Lo, n, A.rp, A.col, smem, A.smem_per_warp, A.pool, 0, cap);
  __syncwarp();
  if (lane == 0) {
    // the first path is shared and read-only; automorphisms go to the store
    W.fcode = P.fcode;
    W.fseq = P.fseq;
    W.flabel = P.flabel;
    W.fcert = P.fcert;
    W.auts = P.auts;
    W.stride = A.WL.stride;
    W.nact = 0;
    W.ntouched = 0;
  }
  __syncwarp();
  // the per-step scratch starts clear; set up once the warp has work (a
  // grid has more warps than most searches have items)
  bool ready = false;
  auto setup = [&] {
    for (uint32_t i = lane; i < n; i += 32) {
      W.cnt[i] = 0;
      W.cellcnt[i] = 0;
      W.fill[i] = 0;
    }
    for (uint32_t w = lane; w < W.nw; w += 32) {
      W.act[w] = 0;
      W.tcb[w] = 0;
    }
    for (uint32_t w = lane; w < W.nsw; w += 32) {
      W.acts[w] = 0;
      W.tcbs[w] = 0;
    }
    __syncwarp();
    ready = true;
  };
  const uint64_t deadline = A.budget_ns ? H->t0 + A.budget_ns : 0;
  WideBest best{0, 0, 0xffffffffu};
  uint32_t known = 0, fix_init = 0, prev_k = 0;
  unsigned long long my_nodes = 0;
  int32_t status = kOk;
  uint64_t iter = 0;
  while (status == kOk) {
    uint32_t it = 0;
    if (lane == 0) it = atomicAdd(&H->next_item, 1u);
    it = __shfl_sync(GCL_FULL, it, 0);
    bool gift = false;
    uint32_t k = 0, tf = 0, tl = 0, v = 0, gift_eq = 0;
    bool skip = false;
    if (it >= nitems) {
      if constexpr (!kShare) {
        break;
      } else {
        // no item left: wait for a subtree another warp hands over
        uint32_t slot = 0;
        unsigned long long tc = cnt.now();
        const int32_t gs = wide_take_gift(P, deadline, &slot);
        cnt.add(kCntGiftWaitCycles, cnt.now() - tc);
        if (gs == 0) break;
        if (gs != 1) {
          status = gs;
          break;
        }
        gift = true;
        cnt.add(kCntGiftsTaken, 1);
        tc = cnt.now();
        if (!ready) setup();
        const int32_t ns = wide_gift_node(P, A, slot, D, &k, &tf, &tl, &v, &gift_eq);
        cnt.add(kCntRefineCycles, cnt.now() - tc);
        if (ns != kOk) {
          status = ns;
          break;
        }
        known = wide_ready_prefix(P, known, cap);
        if (known) {
          bool ok = true;
          tc = cnt.now();
          const uint32_t r = wide_gift_orbit_min(P, v, k, tf, tl, known, A.WL.stride, &ok);
          cnt.add(kCntOrbitCycles, cnt.now() - tc);
          if (!ok) {
            status = kTimeout;
            break;
          }
          skip = r != v;
        }
      }
    }
    if (*(volatile int32_t*)&H->status != kOk) break;
    if (!ready) setup();
    if (!gift) {
      if constexpr (kShare) {
        if (lane == 0) atomicAdd(&H->busy, 1u);
      }
      // item -> level (cum is ascending over levels taken deepest first)
      uint32_t lo = 0, hi = D - 1;  // cum[lo] <= it < cum[hi]
      while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (P.cum[mid] <= it)
          lo = mid;
        else
          hi = mid;
      }
      k = D - 2 - lo;  // parent node level k+1, its target cell index k
      tf = P.tcfirst[k];
      tl = P.tclen[k];
      v = P.lelem[tf + 1 + (it - P.cum[lo])];
      if (H->gate) {
        const unsigned long long tc = cnt.now();
        int32_t gs = wide_gate(H, P.cum[lo], deadline);
        // with the probe, the level's other items also wait for its first
        // item, up to twice the first path's duration: the automorphisms
        // that one finds prune them (it is done when `done` passes the
        // deeper levels' items, since no other item of the level can finish
        // before it)
        if (gs == kOk && A.probe && it != P.cum[lo])
          gs = wide_gate_soft(H, P.cum[lo] + 1u,
                              __shfl_sync(GCL_FULL, lane == 0 ? global_ns() : 0ull, 0) +
                                  *(volatile unsigned long long*)&H->probe_ns,
                              deadline);
        cnt.add(kCntGateCycles, cnt.now() - tc);
        if (gs != kOk) {
          status = gs;
          break;
        }
      }
      known = wide_ready_prefix(P, known, cap);
      if (known) {
        bool ok = true;
        const unsigned long long tc = cnt.now();
        const uint32_t r = H->gate ? wide_orbit_min(P, v, lo, k, tf, tl, known, A.WL.stride, &ok)
                                  : wide_orbit_min_own(P, v, k, tf, tl, known, A.WL.stride, &ok);
        cnt.add(kCntOrbitCycles, cnt.now() - tc);
        if (!ok) {
          status = kTimeout;
          break;
        }
        skip = r != v;  // an equivalent sibling is covered by its orbit's least vertex
      }
      cnt.add(skip ? kCntItemsPruned : kCntItems, 1);
    }
    do {
    if (skip) break;
    if (!gift) {
      // the parent node: the first leaf backtracked to level k+1
      for (uint32_t i = lane; i < n; i += 32) {
        const uint32_t e = P.lelem[i];
        W.elem[i] = e;
        W.pos[e] = i;
        W.inlev[i] = P.linlev[i];
      }
      for (uint32_t w = lane; w < W.nw; w += 32) W.stb[w] = P.lstb[w];
      __syncwarp();
      bm_resummarize(W.stb, W.sts, W.nw, W.nsw);
      if (lane == 0) W.ncells = n;
      __syncwarp();
      if (!sp_backtrack(k + 1) || sp_cell_end(W, tf) - tf != tl) {
        status = kInternal;
        break;
      }
      __syncwarp();
      if (lane == 0) {  // the item's DFS logs its changes from here
        W.utop = 0;
        W.ulog_bad = 0;
      }
      __syncwarp();
      for (uint32_t i = lane; i < k; i += 32) W.seq[i] = P.fseq[i];
      for (uint32_t i = lane; i <= k; i += 32) W.pathcode[i] = P.fcode[i];
      __syncwarp();
    } else {
      if (lane == 0) {  // the subtree's DFS logs its changes from here
        W.utop = 0;
        W.ulog_bad = 0;
      }
      __syncwarp();
    }
    // the previous item's sequence shares the first path's first
    // min(k, prev_k) vertices with this one (a handed-over subtree's
    // sequence may share none)
    sp_fix_clamp(gift ? 0u : min(k, prev_k), fix_init);
    prev_k = gift ? 0u : k;
    if (lane == 0) {
      SpTc h;
      h.first = tf;
      h.len = tl;
      h.counter = n;  // this warp takes no other child of the parent
      h.last = 0;
      h.rslot = -1;
      h.pad = 0;
      W.tc[k] = h;
      W.pool_top = 0;
    }
    __syncwarp();
    // private best: refresh when the shared one has changed
    if (*(volatile uint32_t*)&H->version != best.version && !wide_adopt(P, A.m, &best)) {
      status = kTimeout;
      break;
    }
    // the first leaf anchors gca jumps (not for a handed-over subtree)
    bool best_local = !gift && best.version == 0;
    uint32_t eqlevfirst = gift ? gift_eq : k + 1, seqlen = k, level = k + 1;
    int eqlevcanon = 0, comp_canon = 0, tcl = (int)k + 1;
    wide_recompare(k + 1, best.canon_level, &eqlevcanon, &comp_canon);
    // the item's node
    __syncwarp();
    if (lane == 0) W.seq[seqlen] = v;
    __syncwarp();
    ++seqlen;
    ++my_nodes;
    unsigned long long tr = cnt.now();
    if (!sp_individualize(level, v, tf)) {
      status = kInternal;
      break;
    }
    int code = sp_refine(level);
    cnt.add(kCntRefineCycles, cnt.now() - tr);
    if (code < 0) {
      status = kInternal;
      break;
    }
    ++level;
    bool have_node = true;
    // DFS of the item's subtree (other_path_node / classify_node)
    while (true) {
      if ((++iter & 15) == 0 && deadline &&
          __shfl_sync(GCL_FULL, lane == 0 ? global_ns() : 0ull, 0) > deadline) {
        status = kTimeout;
        break;
      }
      if constexpr (kShare) {
        if (!have_node && (iter & 7) == 0 && wide_try_donate(P, A, k, level, tcl))
          cnt.add(kCntGiftsGiven, 1);
      }
      int bt = -1;
      bool recompare = false;
      if (have_node) {
        have_node = false;
        const uint32_t Lv = level;
        __syncwarp();
        if (lane == 0) W.pathcode[Lv - 1] = code;
        __syncwarp();
        if (eqlevfirst == Lv - 1 && code == W.fcode[Lv - 1]) eqlevfirst = Lv;
        if (eqlevcanon == (int)Lv - 1) {
          const int cc = W.ccode[Lv - 1];
          if (code < cc) {
            comp_canon = -1;
          } else if (code > cc) {
            comp_canon = 1;
          } else {
            comp_canon = 0;
            eqlevcanon = (int)Lv;
          }
        }
        if (comp_canon > 0) {
          __syncwarp();
          if (lane == 0) W.ccode[Lv - 1] = code;
          __syncwarp();
        }
        int dec = 0;
        if (eqlevfirst != Lv && comp_canon < 0) {
          dec = 4;
        } else if (W.ncells == n) {
          cnt.add(kCntLeaves, 1);
          const unsigned long long tc = cnt.now();
          sp_leaf_cert(W.ccert);
          if (eqlevfirst == Lv && sp_cmp_leaf(W.ccert, W.flabel, W.fcert, false) == 0) dec = 1;
          if (dec == 0) {
            if (comp_canon == 0) {
              if ((int)Lv < best.canon_level)
                comp_canon = 1;
              else
                comp_canon = sp_cmp_leaf(W.ccert, W.blabel, W.bcert, true);
            }
            dec = comp_canon == 0 ? 2 : (comp_canon > 0 ? 3 : 4);
          }
          cnt.add(kCntLeafCycles, cnt.now() - tc);
        }
        if (dec == 1) {
          cnt.add(kCntAutsFirst, 1);
          wide_store_aut<false>(P, W.flabel, cap, A.WL.stride, D);
          const int gg = sp_gca(W.fseq, D - 1, seqlen);
          bt = gg >= 0 ? gg : (int)Lv - 1;
        } else if (dec == 2) {
          cnt.add(kCntAutsBest, 1);
          wide_store_aut<false>(P, W.blabel, cap, A.WL.stride, D);
          const int gg = best_local ? sp_gca(W.bseq, best.best_seqlen, seqlen) : -1;
          bt = gg >= 0 ? gg : (int)Lv - 1;
        } else if (dec == 3) {
          // the leaf beats the private best: it becomes the shared best
          // unless the shared best has moved on, in which case that one is
          // adopted and the leaf compared again
          int res = 0;
          for (int tries = 0; tries < 64 && res == 0; ++tries) {
            if (tries) cnt.add(kCntPublishRetries, 1);
            const int r = wide_try_publish(P, A, Lv, seqlen, &best);
            if (r != 0) {
              res = r;
              break;
            }
            const int c = wide_cmp_private(Lv, best.canon_level);
            if (c < 0) res = 4;
            if (c == 0) res = 2;
          }
          if (res == 1) {
            cnt.add(kCntBestPublished, 1);
            // the leaf is the new shared best and the private one
            sp_copy_u32(W.bcert, W.ccert, (uint32_t)A.m);
            sp_copy_u32(W.blabel, W.elem, n);
            sp_copy_u32(W.bseq, W.seq, seqlen);
            sp_copy_u32((uint32_t*)W.ccode, (const uint32_t*)W.pathcode, Lv);
            if (lane == 0) W.ccode[Lv] = kSentinel;
            __syncwarp();
            best_local = true;
            eqlevcanon = (int)Lv;
            comp_canon = 0;
          } else if (res == 2 || res == 4) {
            // equivalent to, or worse than, the adopted best
            if (res == 2) {
              cnt.add(kCntAutsBest, 1);
              wide_store_aut<false>(P, W.blabel, cap, A.WL.stride, D);
            }
            best_local = false;
            recompare = true;
          } else {
            status = kTimeout;
            break;
          }
          bt = (int)Lv - 1;
        } else if (dec == 4) {
          bt = (int)Lv - 1;
        }
      } else {
        const bool disc = W.ncells == n;
        if (!disc && (eqlevfirst == level || comp_canon >= 0)) {
          if (tcl < (int)level) {
            const uint32_t t = sp_first_nonsingleton();
            if (t == kNone) {
              status = kInternal;
              break;
            }
            if (lane == 0) {
              SpTc h;
              h.first = t;
              h.len = sp_cell_end(W, t) - t;
              h.counter = 0;
              h.last = 0;
              h.rslot = -1;
              h.pad = 0;
              W.tc[tcl] = h;
            }
            __syncwarp();
            ++tcl;
          }
          const int idx = (int)level - 1;
          if (W.tc[idx].counter >= n) {
            bt = (int)level - 1;
          } else {
            known = wide_ready_prefix(P, known, cap);
            if (known > fix_init) {
              wide_fix_init(fix_init, known);
              fix_init = known;
            }
            if (known > (uint32_t)W.tc[idx].last) {
              const unsigned long long tc = cnt.now();
              const bool orb_ok = sp_orbits<true>(idx, (int)known, seqlen);
              cnt.add(kCntOrbitCycles, cnt.now() - tc);
              if (!orb_ok) {
                status = W.pool_top >= W.pool_cap ? kAutOverflow : kInternal;
                break;
              }
              __syncwarp();
              if (lane == 0) W.tc[idx].last = (int32_t)known;
              __syncwarp();
            }
            const SpTc t = W.tc[idx];
            const uint32_t u = sp_next_rep(t);
            __syncwarp();
            if (u == kNone) {
              if (lane == 0) W.tc[idx].counter = n;
              __syncwarp();
              bt = (int)level - 1;
            } else {
              if (lane == 0) {
                W.tc[idx].counter = u + 1;
                W.seq[seqlen] = u;
              }
              __syncwarp();
              ++seqlen;
              ++my_nodes;
              tr = cnt.now();
              if (!sp_individualize(level, u, t.first)) {
                status = kInternal;
                break;
              }
              code = sp_refine(level);
              cnt.add(kCntRefineCycles, cnt.now() - tr);
              if (code < 0) {
                status = kInternal;
                break;
              }
              ++level;
              have_node = true;
            }
          }
        } else {
          // worse than the private best and off the first path's trail
          bt = (int)level - 1;
          recompare = true;
        }
      }
      if (bt >= 0) {
        const uint32_t Lv = (uint32_t)bt;
        if (Lv <= k + 1) break;  // the item's subtree is done
        if (!sp_backtrack_log(Lv)) {
          status = kInternal;
          break;
        }
        if (Lv < eqlevfirst) eqlevfirst = Lv;
        if ((int)Lv <= eqlevcanon) {
          eqlevcanon = (int)Lv;
          comp_canon = 0;
        }
        seqlen = Lv - 1;
        tcl = (int)Lv;
        level = Lv;
        sp_fix_clamp(seqlen, fix_init);
        __syncwarp();
        if (lane == 0)
          while (W.pool_top > 0 && W.pool_owner[W.pool_top - 1] >= (int32_t)Lv) W.pool_top -= 1;
        __syncwarp();
        if (recompare) wide_recompare(level, best.canon_level, &eqlevcanon, &comp_canon);
      }
    }
    } while (0);
    if (status != kOk) break;
    __syncwarp();
    if (lane == 0) {
      if (!gift) atomicAdd(&H->done, 1u);  // opens the next level's gate when it is the last
      if constexpr (kShare) {
        __threadfence();  // what this warp handed over is published before it stops counting
        atomicSub(&H->busy, 1u);
      }
    }
    __syncwarp();
  }
  if (status != kOk) wide_fail(H, status);
  if (lane == 0) atomicAdd(&H->nodes, my_nodes);
  cnt.add(kCntNodes, my_nodes);
  cnt.add(kCntWarpCycles, cnt.now() - t_start);
  cnt.flush(H);
}

// ---------------------------------------------------------------------------
// 3. Outputs from the shared best leaf (one warp).
// ---------------------------------------------------------------------------
constexpr int kWideFinishThreads = 128;

// Word w of canonical row i of the best leaf's packed matrix: bit c % 64 for
// every certificate entry c (a neighbour's canonical position) of the row's
// vertex with c / 64 == w.
__host__ __device__ inline uint64_t wide_row_word(const int32_t* rp, const uint32_t* label,
                                                  const uint32_t* cert, uint32_t i, uint32_t w) {
  const uint32_t v = label[i];
  uint64_t x = 0;
  for (int32_t j = rp[v]; j < rp[v + 1]; ++j) {
    const uint32_t c = cert[j];
    if ((c >> 6) == w) x |= 1ull << (c & 63);
  }
  return x;
}

// A warp per canonical row (grid-stride): the row's packed words, each lane
// building whole words from the row's certificate entries, and its dense
// bytes, zeroed and then set -- no two lanes write the same byte or word.
__global__ void __launch_bounds__(kWideFinishThreads) wide_finish_kernel(WideArgs A) {
  const uint32_t lane = lane_id();
  const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const WidePtrs P = wide_ptrs(A);
  const WideHdr* H = P.H;
  const uint32_t n = A.n;
  const int32_t status = H->status;
  if (warp == 0 && lane == 0) {
    A.out_status[0] = status;
    if (A.out_stats) {
      A.out_stats[0] = (int64_t)H->naut;
      A.out_stats[1] = (int64_t)H->nodes;
    }
  }
  if (status != kOk) return;
  if (A.out_label)
    for (uint64_t j = warp * 32 + lane; j < n; j += warps * 32)
      A.out_label[j] = (int32_t)P.blabel[j];
  if (A.out_rows) {
    const uint32_t words = (n + 63) / 64;
    for (uint64_t i = warp; i < n; i += warps) {
      uint64_t* row = A.out_rows + i * words;
      for (uint32_t w = lane; w < words; w += 32)
        row[w] = wide_row_word(A.rp, P.blabel, P.bcert, (uint32_t)i, w);
    }
  }
  if (A.out_dense) {
    for (uint64_t i = warp; i < n; i += warps) {
      uint8_t* row = A.out_dense + i * n;
      for (uint32_t j = lane; j < n; j += 32) row[j] = 0;
      __syncwarp();
      const uint32_t v = P.blabel[i];
      for (int32_t j = A.rp[v] + (int32_t)lane; j < A.rp[v + 1]; j += 32) row[P.bcert[j]] = 1;
      __syncwarp();
    }
  }
}

}  // namespace gcl
